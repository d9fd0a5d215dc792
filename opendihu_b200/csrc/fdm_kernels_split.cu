// Split-path kernels (reaction, diffusion, stimulation schedule) and the model table.
#define FDM_COMMON_KERNELS_TU
#include <algorithm>
#include <atomic>
#include <mutex>

#include "fdm_internal.h"
#include "fdm_equilibrium.cuh"
#include "fdm_model_launch.cuh"

#include "generated/hodgkin_huxley_1952_anone_c2_3_4.cuh"
#include "generated/shorten_ocallaghan_davidson_soboleva_2007_a32_c65.cuh"

namespace fdm {

using HH = fdm_model_hodgkin_huxley_1952_anone_c2_3_4;
using SH = fdm_model_shorten_ocallaghan_davidson_soboleva_2007_a32_c65;

static const ModelDesc g_models[] = {
  {HH::name, HH::nStates, HH::nAlgebraics, HH::nParameters, HH::statesInitialValues, HH::parameterDefaults, true},
  {SH::name, SH::nStates, SH::nAlgebraics, SH::nParameters, SH::statesInitialValues, SH::parameterDefaults, false},
};

constexpr int kBuiltinModels = (int)(sizeof(g_models) / sizeof(g_models[0]));
constexpr int kMaxModules = 64;

// run-time model modules, appended by register_model_module and never removed (their libraries stay loaded)
static ModelModule g_modules[kMaxModules];
static std::atomic<int> g_n_modules{0};
static std::mutex g_modules_mu;

int n_models() { return kBuiltinModels + g_n_modules.load(std::memory_order_acquire); }

static const ModelModule* module_of(int model)
{
  const int k = model - kBuiltinModels;
  return (k >= 0 && k < g_n_modules.load(std::memory_order_acquire)) ? &g_modules[k] : nullptr;
}

const ModelDesc* model_desc(int model)
{
  if (model >= 0 && model < kBuiltinModels)
    return &g_models[model];
  const ModelModule* m = module_of(model);
  return m ? &m->desc : nullptr;
}

int register_model_module(const ModelModule& m)
{
  std::lock_guard<std::mutex> lock(g_modules_mu);
  const int k = g_n_modules.load(std::memory_order_relaxed);
  if (k >= kMaxModules || m.abi != FDM_MODEL_MODULE_ABI)
    return -1;
  g_modules[k] = m;
  g_modules[k].desc.fused_supported = false;   // modules carry the split-path, equilibrium and adjoint kernels
  g_n_modules.store(k + 1, std::memory_order_release);
  return kBuiltinModels + k;
}

cudaError_t launch_reaction(int model, RealKind rk, MathKind mk, const ReactionArgs& a, cudaStream_t s)
{
  switch (model) {
  case 0: return reaction_model<HH>(rk, mk, a, s);
  case 1: return reaction_model<SH>(rk, mk, a, s);
  default: {
    const ModelModule* m = module_of(model);
    return m ? m->reaction(rk, mk, a, s) : cudaErrorInvalidValue;
  }
  }
}

cudaError_t launch_cellml_rhs(int model, MathKind mk, int64_t n, double t, const double* states, const double* params,
                              double* rates, double* algebraics, cudaStream_t s)
{
  if (n == 0)
    return cudaSuccess;
  switch (model) {
  case 0: return cellml_rhs_model<HH>(mk, n, t, states, params, rates, algebraics, s);
  case 1: return cellml_rhs_model<SH>(mk, n, t, states, params, rates, algebraics, s);
  default: {
    const ModelModule* m = module_of(model);
    return m ? m->cellml_rhs(mk, n, t, states, params, rates, algebraics, s) : cudaErrorInvalidValue;
  }
  }
}

cudaError_t launch_equilibrium_search(int model, MathKind mk, double* u, const double* u0, const double* params,
                               EquilibriumSearch* es, int64_t max_iterations, cudaStream_t s)
{
  switch (model) {
  case 0: return equilibrium_search_model<HH>(mk, u, u0, params, es, max_iterations, s);
  case 1: return equilibrium_search_model<SH>(mk, u, u0, params, es, max_iterations, s);
  default: {
    const ModelModule* m = module_of(model);
    return m ? m->equilibrium_search(mk, u, u0, params, es, max_iterations, s) : cudaErrorInvalidValue;
  }
  }
}

cudaError_t launch_schedule(const StimArgs& a, const SplitStep* steps, int n_steps, cudaStream_t s)
{
  if (a.n_fibers == 0)
    return cudaSuccess;
  const int T = 128;
  stimulation_schedule_kernel<<<(a.n_fibers + T - 1) / T, T, 0, s>>>(a, steps, n_steps);
  return cudaGetLastError();
}

cudaError_t launch_coefficients(int n_fibers, const int64_t* fiber_offsets, const double* element_lengths,
                                const double* prefactor, double dt, int implicit_euler, double* coef, int64_t stride,
                                cudaStream_t s)
{
  if (n_fibers == 0)
    return cudaSuccess;
  const int T = 64;
  diffusion_coefficients_kernel<<<(n_fibers + T - 1) / T, T, 0, s>>>(n_fibers, fiber_offsets, element_lengths,
                                                                     prefactor, dt, implicit_euler, coef, stride);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(256) states_to_pairs_kernel(const double* __restrict__ x, float* __restrict__ hi,
                                                              float* __restrict__ lo, int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    const float h = __double2float_rn(v);
    hi[i] = h;
    lo[i] = __double2float_rn(__dsub_rn(v, (double)h));
  }
}

__global__ void __launch_bounds__(256) pairs_to_states_kernel(const float* __restrict__ hi,
                                                              const float* __restrict__ lo, double* __restrict__ x,
                                                              int64_t n)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = __dadd_rn((double)hi[i], (double)lo[i]);
}

static unsigned elementwise_blocks(int64_t n)
{
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
}

cudaError_t launch_states_to_pairs(const double* x, float* hi, float* lo, int64_t n, cudaStream_t s)
{
  if (n <= 0)
    return cudaSuccess;
  states_to_pairs_kernel<<<elementwise_blocks(n), 256, 0, s>>>(x, hi, lo, n);
  return cudaGetLastError();
}

cudaError_t launch_pairs_to_states(const float* hi, const float* lo, double* x, int64_t n, cudaStream_t s)
{
  if (n <= 0)
    return cudaSuccess;
  pairs_to_states_kernel<<<elementwise_blocks(n), 256, 0, s>>>(hi, lo, x, n);
  return cudaGetLastError();
}

// below this many fibers the diffusion solves take a CTA per fiber (4 warps' worth of CTAs per SM would be
// needed before a warp per fiber fills the GPU)
constexpr int DIFFUSION_BLOCK_MAX_FIBERS = 4 * 148;

cudaError_t launch_diffusion(int n_fibers, const int64_t* fiber_offsets, const double* coef, int64_t stride,
                                  double* vm, double* scratch, cudaStream_t s, const int* eq_counter,
                                  const int* eq_nbuf, int n_ranks)
{
  if (n_fibers == 0)
    return cudaSuccess;
  if (n_fibers < DIFFUSION_BLOCK_MAX_FIBERS) {
    // few fibers: a CTA per fiber fills more of the GPU than a warp per fiber
    diffusion_block_kernel<256><<<(unsigned)n_fibers, 256, 0, s>>>(fiber_offsets, coef, stride, vm, scratch,
                                                                   eq_counter, eq_nbuf, n_ranks > 0 ? n_ranks : 1);
    return cudaGetLastError();
  }
  const int T = 128;
  const int64_t threads = (int64_t)n_fibers * 32;
  diffusion_warp_kernel<<<(unsigned)((threads + T - 1) / T), T, 0, s>>>(n_fibers, fiber_offsets, coef, stride, vm,
                                                                        scratch, eq_counter, eq_nbuf,
                                                                        n_ranks > 0 ? n_ranks : 1);
  return cudaGetLastError();
}

// ---- equilibrium skip ----
cudaError_t launch_equilibrium_half(int model, RealKind rk, MathKind mk, const ReactionArgs& a, const EqLayout& L,
                                    const EqSpec& e, uint8_t* info, uint8_t* prefix, uint8_t* block_agg, int n_states,
                                    bool trace, cudaStream_t s)
{
  cudaError_t ce = cudaSuccess;
  switch (model) {
  case 0: ce = reaction_eq_model<HH>(rk, mk, a, L, e, s); break;
  case 1: ce = reaction_eq_model<SH>(rk, mk, a, L, e, s); break;
  default: {
    const ModelModule* m = module_of(model);
    if (!m)
      return cudaErrorInvalidValue;
    ce = m->reaction_eq(rk, mk, a, L, e, s);
  }
  }
  if (ce != cudaSuccess || L.n_buffers == 0)
    return ce;
  const int T = 128;
  const unsigned bb = (unsigned)((L.n_buffers + T - 1) / T);
  if (rk == REAL_F64)
    eq_changed_kernel<double><<<bb, T, 0, s>>>(a, L, e, n_states, info);
  else
    eq_changed_kernel<float><<<bb, T, 0, s>>>(a, L, e, n_states, info);
  const int64_t nblk = (L.n_buffers + EQ_SCAN_T - 1) / EQ_SCAN_T;
  eq_scan_block_kernel<<<(unsigned)nblk, EQ_SCAN_T, 0, s>>>(L, info, prefix, block_agg);
  eq_scan_top_kernel<<<1, 1, 0, s>>>(block_agg, nblk);
  if (rk == REAL_F64)
    eq_commit_kernel<double><<<bb, T, 0, s>>>(a, L, e, info, prefix, block_agg, n_states);
  else
    eq_commit_kernel<float><<<bb, T, 0, s>>>(a, L, e, info, prefix, block_agg, n_states);
  if (trace && a.trace_slot)
    eq_trace_kernel<<<(unsigned)((a.n_nodes + T - 1) / T), T, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_half(int model, MathKind mk, const AdjointArgs& a, cudaStream_t s)
{
  switch (model) {
  case 0: return adjoint_model<HH>(mk, a, s);
  case 1: return adjoint_model<SH>(mk, a, s);
  default: {
    const ModelModule* m = module_of(model);
    return m ? m->adjoint_half(mk, a, s) : cudaErrorInvalidValue;
  }
  }
}

template<int T, int M>
static cudaError_t adjoint_diffusion_block(int n_fibers, const int64_t* fiber_offsets, const double* element_lengths,
                                           const double* coef, int64_t stride, double* lam, const double* u,
                                           const double* x, int implicit_euler, double* grad_prefactor,
                                           cudaStream_t s)
{
  adjoint_diffusion_block_kernel<T, M><<<(unsigned)n_fibers, T, 0, s>>>(fiber_offsets, element_lengths, coef, stride,
                                                                       lam, u, x, implicit_euler, grad_prefactor);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_diffusion(int n_fibers, const int64_t* fiber_offsets, const double* element_lengths,
                                     const double* coef, int64_t stride, double* lam, const double* u, const double* x,
                                     int implicit_euler, double* grad_prefactor, double* scratch, double* mu,
                                     int64_t max_fiber_len, cudaStream_t s)
{
  if (n_fibers == 0)
    return cudaSuccess;
  // few fibers: one CTA per fiber (block-wide scans); many fibers: one warp per fiber fills the GPU
  if (n_fibers < DIFFUSION_BLOCK_MAX_FIBERS) {
    if (max_fiber_len <= 512)
      return adjoint_diffusion_block<128, 4>(n_fibers, fiber_offsets, element_lengths, coef, stride, lam, u, x,
                                             implicit_euler, grad_prefactor, s);
    if (max_fiber_len <= 1024)
      return adjoint_diffusion_block<256, 4>(n_fibers, fiber_offsets, element_lengths, coef, stride, lam, u, x,
                                             implicit_euler, grad_prefactor, s);
    if (max_fiber_len <= 2048)
      return adjoint_diffusion_block<256, 8>(n_fibers, fiber_offsets, element_lengths, coef, stride, lam, u, x,
                                             implicit_euler, grad_prefactor, s);
    if (max_fiber_len <= 4096)
      return adjoint_diffusion_block<512, 8>(n_fibers, fiber_offsets, element_lengths, coef, stride, lam, u, x,
                                             implicit_euler, grad_prefactor, s);
  }
  const int T = 128;
  const int64_t threads = (int64_t)n_fibers * 32;
  adjoint_diffusion_warp_kernel<<<(unsigned)((threads + T - 1) / T), T, 0, s>>>(
      n_fibers, fiber_offsets, element_lengths, coef, stride, lam, u, x, implicit_euler, grad_prefactor, scratch, mu);
  return cudaGetLastError();
}

__global__ void count_nonfinite_kernel(const double* __restrict__ x, int64_t n, int* count)
{
  int local = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    local += isfinite(x[i]) ? 0 : 1;
  local = __reduce_add_sync(0xffffffffu, local);
  if ((threadIdx.x & 31) == 0 && local)
    atomicAdd(count, local);
}

cudaError_t launch_count_nonfinite(const double* x, int64_t n, int* count, cudaStream_t s)
{
  if (n == 0)
    return cudaSuccess;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 8)
    blocks = 148 * 8;
  count_nonfinite_kernel<<<blocks, 256, 0, s>>>(x, n, count);
  return cudaGetLastError();
}

} // namespace fdm
