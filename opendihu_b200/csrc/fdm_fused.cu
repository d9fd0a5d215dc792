// Fused-kernel dispatch: (model, reaction precision, math policy, CTA shape) -> instantiation.
// The instantiations live in fdm_fused_inst.cuh, compiled once per (precision, math) in the
// fdm_fused_{f64,f32}_{exact,approx}.cu translation units so that they build in parallel.
#include "fdm_fused_inst.cuh"

namespace fdm {

static const FusedShape g_shapes[] = {
#define FDM_SHAPE_ENTRY(T, M) {T, M},
  FDM_FUSED_SHAPES(FDM_SHAPE_ENTRY)
#undef FDM_SHAPE_ENTRY
};

int fused_shapes(FusedShape* out, int capacity)
{
  const int n = (int)(sizeof(g_shapes) / sizeof(g_shapes[0]));
  for (int i = 0; i < n && i < capacity; i++)
    out[i] = g_shapes[i];
  return n;
}

static const FusedShape g_cluster_shapes[] = {
#define FDM_SHAPE_ENTRY(T, M) {T, M},
  FDM_CLUSTER_SHAPES(FDM_SHAPE_ENTRY)
#undef FDM_SHAPE_ENTRY
};

int cluster_shapes(FusedShape* out, int capacity)
{
  const int n = (int)(sizeof(g_cluster_shapes) / sizeof(g_cluster_shapes[0]));
  for (int i = 0; i < n && i < capacity; i++)
    out[i] = g_cluster_shapes[i];
  return n;
}

cudaError_t launch_fused_cluster_hh_f32(int shape, int csize, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_cluster_hh_f64(int shape, int csize, const FusedArgs& a, cudaStream_t s);

cudaError_t launch_fused_cluster(int model, RealKind rk, int shape, int csize, const FusedArgs& a, cudaStream_t s)
{
  if (model != 0 || csize < 1 || csize > FDM_MAX_CLUSTER)
    return cudaErrorInvalidValue;
  return rk == REAL_F64 ? launch_fused_cluster_hh_f64(shape, csize, a, s) : launch_fused_cluster_hh_f32(shape, csize, a, s);
}

cudaError_t launch_fused(int model, RealKind rk, MathKind mk, int shape, const FusedArgs& a, cudaStream_t s)
{
  if (model != 0)
    return cudaErrorInvalidValue;
  if (rk == REAL_F64)
    return mk == MATH_EXACT ? launch_fused_hh_f64_exact(shape, a, s) : launch_fused_hh_f64_approx(shape, a, s);
  return mk == MATH_EXACT ? launch_fused_hh_f32_exact(shape, a, s) : launch_fused_hh_f32_approx(shape, a, s);
}

} // namespace fdm
