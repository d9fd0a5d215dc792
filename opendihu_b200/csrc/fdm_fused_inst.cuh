// Fused-kernel instantiations for one (precision, math policy); included by fdm_fused_*.cu.
#pragma once
#include <atomic>
#include "fdm_internal.h"

#include "generated/hodgkin_huxley_1952_anone_c2_3_4.cuh"

// (threads per CTA, nodes per thread); capacity T*M nodes per bin
#define FDM_FUSED_SHAPES(X) \
  X(128, 8)                 \
  X(256, 4)                 \
  X(256, 6)                 \
  X(256, 8)                 \
  X(256, 10)                \
  X(384, 7)                 \
  X(384, 8)                 \
  X(512, 3)                 \
  X(512, 5)                 \
  X(512, 6)                 \
  X(640, 4)                 \
  X(768, 4)                 \
  X(1024, 3)

namespace fdm {

using FusedHH = fdm_model_hodgkin_huxley_1952_anone_c2_3_4;

cudaError_t launch_fused_hh_f64_exact(int shape, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_hh_f64_approx(int shape, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_hh_f32_exact(int shape, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_hh_f32_approx(int shape, const FusedArgs& a, cudaStream_t s);
// the same with onlyComputeIfHasBeenStimulated (fdm_fused_*_gate.cu)
cudaError_t launch_fused_hh_f64_exact_gate(int shape, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_hh_f64_approx_gate(int shape, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_hh_f32_exact_gate(int shape, const FusedArgs& a, cudaStream_t s);
cudaError_t launch_fused_hh_f32_approx_gate(int shape, const FusedArgs& a, cudaStream_t s);

// The dynamic shared memory limit of a kernel is set per device: once on each device (bit d of done; the
// solvers of several devices may launch from concurrent host threads).
template<class K>
static cudaError_t set_smem_once(K kernel, size_t smem, std::atomic<uint64_t>& done)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return e;
  const uint64_t bit = dev < 64 ? (uint64_t(1) << dev) : 0;
  if (bit && (done.load(std::memory_order_acquire) & bit))
    return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && bit)
    done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

template<class Model, class RR, class Math, int T, int M, bool GATE>
static cudaError_t fused_one(const FusedArgs& a, cudaStream_t s)
{
  constexpr size_t smem = fused_smem_bytes<Model, RR, Math, T, M>();
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = set_smem_once(fused_kernel<Model, RR, Math, T, M, GATE, false>, smem, attr_done);
  if (e != cudaSuccess)
    return e;
  if (a.n_bins == 0)
    return cudaSuccess;
  fused_kernel<Model, RR, Math, T, M, GATE, false><<<a.n_bins, T, smem, s>>>(a);
  return cudaGetLastError();
}

template<class Model, class RR, class Math, bool GATE>
static cudaError_t fused_shape(int shape, const FusedArgs& a, cudaStream_t s)
{
  int k = 0;
#define FDM_SHAPE_CASE(T, M)                             \
  if (shape == k)                                        \
    return fused_one<Model, RR, Math, T, M, GATE>(a, s); \
  k++;
  FDM_FUSED_SHAPES(FDM_SHAPE_CASE)
#undef FDM_SHAPE_CASE
  return cudaErrorInvalidValue;
}

// cluster mode (one fiber per thread-block cluster of csize CTAs; FDM_CLUSTER_SHAPES in fdm_internal.h)
template<class Model, class RR, class Math, int T, int M>
static cudaError_t fused_cluster_one(const FusedArgs& a, int csize, cudaStream_t s)
{
  constexpr size_t smem = fused_smem_bytes<Model, RR, Math, T, M>();
  auto kernel = fused_kernel<Model, RR, Math, T, M, false, true>;
  static std::atomic<uint64_t> attr_done{0};
  cudaError_t e = set_smem_once(kernel, smem, attr_done);
  if (e != cudaSuccess)
    return e;
  if (a.n_bins == 0)
    return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(a.n_bins * csize), 1, 1);
  cfg.blockDim = dim3(T, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, a);
}

template<class Model, class RR, class Math>
static cudaError_t fused_cluster_shape(int shape, int csize, const FusedArgs& a, cudaStream_t s)
{
  int k = 0;
#define FDM_CLUSTER_CASE(T, M)                                   \
  if (shape == k)                                                \
    return fused_cluster_one<Model, RR, Math, T, M>(a, csize, s); \
  k++;
  FDM_CLUSTER_SHAPES(FDM_CLUSTER_CASE)
#undef FDM_CLUSTER_CASE
  return cudaErrorInvalidValue;
}

} // namespace fdm
