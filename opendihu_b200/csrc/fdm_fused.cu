// Fused-kernel instantiations: (model, reaction precision, math policy, CTA shape).
#include "fdm_internal.h"

#include "generated/hodgkin_huxley_1952_anone_c2_3_4.cuh"

namespace fdm {

using HH = fdm_model_hodgkin_huxley_1952_anone_c2_3_4;

// (threads per CTA, nodes per thread); capacity T*M nodes per bin
#define FDM_FUSED_SHAPES(X) \
  X(128, 8)                 \
  X(256, 4)                 \
  X(256, 6)                 \
  X(256, 8)                 \
  X(256, 10)                \
  X(512, 3)                 \
  X(512, 5)                 \
  X(1024, 3)

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

template<class Model, class RR, class Math, int T, int M>
static cudaError_t fused_one(const FusedArgs& a, cudaStream_t s)
{
  constexpr size_t smem = fused_smem_bytes<T, M>();
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(fused_kernel<Model, RR, Math, T, M>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
      return e;
    attr_set = true;
  }
  if (a.n_bins == 0)
    return cudaSuccess;
  fused_kernel<Model, RR, Math, T, M><<<a.n_bins, T, smem, s>>>(a);
  return cudaGetLastError();
}

template<class Model, class RR, class Math>
static cudaError_t fused_shape(int shape, const FusedArgs& a, cudaStream_t s)
{
  int k = 0;
#define FDM_SHAPE_CASE(T, M)                      \
  if (shape == k)                                 \
    return fused_one<Model, RR, Math, T, M>(a, s); \
  k++;
  FDM_FUSED_SHAPES(FDM_SHAPE_CASE)
#undef FDM_SHAPE_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_fused(int model, RealKind rk, MathKind mk, int shape, const FusedArgs& a, cudaStream_t s)
{
  if (model != 0)
    return cudaErrorInvalidValue;
  if (rk == REAL_F64)
    return mk == MATH_EXACT ? fused_shape<HH, double, fdm_math_exact>(shape, a, s)
                            : fused_shape<HH, double, fdm_math_approx>(shape, a, s);
  return mk == MATH_EXACT ? fused_shape<HH, float, fdm_math_exact>(shape, a, s)
                          : fused_shape<HH, float, fdm_math_approx>(shape, a, s);
}

} // namespace fdm
