// Fused-kernel instantiations in cluster mode: HH, float reaction, fdm_math_exact.
#include "fdm_fused_inst.cuh"

namespace fdm {
cudaError_t launch_fused_cluster_hh_f32(int shape, int csize, const FusedArgs& a, cudaStream_t s)
{
  return fused_cluster_shape<FusedHH, float, fdm_math_exact>(shape, csize, a, s);
}
} // namespace fdm
