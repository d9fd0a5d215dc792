// Fused-kernel instantiations: HH, float reaction, fdm_math_approx.
#include "fdm_fused_inst.cuh"

namespace fdm {
cudaError_t launch_fused_hh_f32_approx(int shape, const FusedArgs& a, cudaStream_t s)
{
  if (a.gate)
    return launch_fused_hh_f32_approx_gate(shape, a, s);
  return fused_shape<FusedHH, float, fdm_math_approx, false>(shape, a, s);
}
} // namespace fdm
