// fdm_diffusion_solve_noalloc: the diffusion solve of fdm_diffusion_solve without any device allocation.
//
// Some callers cannot allocate device memory while they run.  Examples: an application that hands the
// whole GPU to its own memory pool at start-up (a PyTorch caching allocator, a coupled multi-physics code
// that reserves nearly all of HBM for its 3D mesh), where an extra cudaMalloc fails or fragments the pool;
// and time-critical stepping loops, where cudaMalloc/cudaFree may synchronize the device and stall other
// work.  For them this entry point takes its scratch from one array compiled into the library instead of
// calling cudaMalloc: FDM_NOALLOC_MAX_NODES nodes x 7 doubles (14.7 MB), which every GPU that loads this
// library holds until the process exits.
//
// The array is shared by all calls and keeps the previous call's contents.  Nothing in it has to start at
// zero: the factorization kernel writes every coefficient the solve reads, and the forward sweep writes
// every intermediate value before the backward sweep reads it.  Calls whose work overlaps on the GPU
// (from several host threads, or on several streams without ordering between them) use the same memory and
// race; order them on one stream or serialize them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/fdm_b200.h"
#include "fdm_internal.h"

// scratch of the allocation-free solve: 6 factorization doubles + 1 forward-sweep double per node
static __device__ __align__(256) double fdm_noalloc_scratch[7 * (size_t)FDM_NOALLOC_MAX_NODES];

// Device code that names the array, so that it stays in this file's device image (never launched).
__global__ void fdm_noalloc_keep_kernel(int write)
{
  if (write)
    fdm_noalloc_scratch[threadIdx.x] = 0.0;
}

namespace {
std::mutex g_mu;
double* g_addr[64] = {};
} // namespace

extern "C" int fdm_diffusion_solve_noalloc(int n_fibers, int64_t n_nodes, const int64_t* d_fiber_offsets,
                                           const double* d_element_lengths, const double* d_prefactor, double dt,
                                           int diffusion_scheme, double* d_vm, void* stream)
{
  using fdm::fdm_report_error;
  if (n_fibers < 0 || n_nodes < 0 ||
      (n_fibers > 0 && (!d_fiber_offsets || !d_element_lengths || !d_prefactor || !d_vm)))
    return fdm_report_error(FDM_ERR_ARG, "fdm_diffusion_solve_noalloc: bad argument");
  if (n_nodes > FDM_NOALLOC_MAX_NODES)
    return fdm_report_error(FDM_ERR_ARG, "fdm_diffusion_solve_noalloc: " + std::to_string(n_nodes) +
                                             " nodes exceed the compiled-in maximum FDM_NOALLOC_MAX_NODES = " +
                                             std::to_string((long long)FDM_NOALLOC_MAX_NODES) +
                                             "; use fdm_diffusion_solve (it allocates its scratch)");
  if (!(dt > 0) || (diffusion_scheme != FDM_IMPLICIT_EULER && diffusion_scheme != FDM_CRANK_NICOLSON))
    return fdm_report_error(FDM_ERR_ARG, "fdm_diffusion_solve_noalloc: dt must be positive and the scheme IE or CN");
  if (n_fibers == 0)
    return FDM_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fdm_report_error(FDM_ERR_CUDA, std::string("fdm_diffusion_solve_noalloc: cudaGetDevice: ") +
                                              cudaGetErrorString(e));
  if (dev < 0 || dev >= 64)
    return fdm_report_error(FDM_ERR_ARG, "fdm_diffusion_solve_noalloc: device ordinal beyond 63");
  double* scratch = nullptr;
  {
    // Set-up, once per device, with that device current: in host code the array's name only stands for
    // the symbol, so its device address is looked up here.  The first call on a device does this (and may
    // load this file's device code); make that first call before any stream capture.
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, fdm_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fdm_report_error(FDM_ERR_CUDA, std::string("fdm_diffusion_solve_noalloc: cudaGetSymbolAddress: ") +
                                                  cudaGetErrorString(e));
      g_addr[dev] = (double*)p;
    }
    scratch = g_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  // The kernels find each fiber's nodes through the device offsets and write the scratch at those nodes, so
  // the offsets must stay inside [0, n_nodes]: their two ends are read back and checked (two 8-byte copies
  // into host stack variables, no allocation); that they do not decrease in between is the caller's part.
  int64_t ends[2] = {0, 0};
  e = cudaMemcpyAsync(&ends[0], d_fiber_offsets, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&ends[1], d_fiber_offsets + n_fibers, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return fdm_report_error(FDM_ERR_CUDA, std::string("fdm_diffusion_solve_noalloc: reading the fiber offsets: ") +
                                              cudaGetErrorString(e));
  if (ends[0] < 0 || ends[1] < ends[0] || ends[1] > n_nodes)
    return fdm_report_error(FDM_ERR_ARG, "fdm_diffusion_solve_noalloc: fiber offsets [" + std::to_string(ends[0]) +
                                             ", " + std::to_string(ends[1]) + "] outside [0, n_nodes = " +
                                             std::to_string(n_nodes) + "]");
  double* coef = scratch;
  double* fwd = scratch + 6 * (size_t)n_nodes;
  e = fdm::launch_coefficients(n_fibers, d_fiber_offsets, d_element_lengths, d_prefactor, dt,
                               diffusion_scheme == FDM_IMPLICIT_EULER, coef, n_nodes, st);
  if (e == cudaSuccess)
    e = fdm::launch_diffusion(n_fibers, d_fiber_offsets, coef, n_nodes, d_vm, fwd, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return fdm_report_error(FDM_ERR_CUDA, std::string("fdm_diffusion_solve_noalloc: ") + cudaGetErrorString(e));
  return FDM_OK;
}
