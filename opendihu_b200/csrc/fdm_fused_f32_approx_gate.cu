// Fused-kernel instantiations: HH, float reaction, fdm_math_approx, with onlyComputeIfHasBeenStimulated.
#include "fdm_fused_inst.cuh"

namespace fdm {
cudaError_t launch_fused_hh_f32_approx_gate(int shape, const FusedArgs& a, cudaStream_t s)
{
  return fused_shape<FusedHH, float, fdm_math_approx, true>(shape, a, s);
}
} // namespace fdm
