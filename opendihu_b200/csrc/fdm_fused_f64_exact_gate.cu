// Fused-kernel instantiations: HH, double reaction, fdm_math_exact, with onlyComputeIfHasBeenStimulated.
#include "fdm_fused_inst.cuh"

namespace fdm {
cudaError_t launch_fused_hh_f64_exact_gate(int shape, const FusedArgs& a, cudaStream_t s)
{
  return fused_shape<FusedHH, double, fdm_math_exact, true>(shape, a, s);
}
} // namespace fdm
