// disableComputationWhenStatesAreCloseToEquilibrium on the split path (compute.tpp:130-254, 630-797).
//
// The reference walks the point buffers of a rank (W consecutive nodes of the rank's concatenated fibers)
// in order.  Every buffer carries a status: inactive (its substeps are skipped), neighbor_is_active or active;
// the first and the last buffer are set active at the start of every compute0D call.  A buffer that runs
// substeps is at equilibrium if no state of any of its W lanes changed by more than 1e-6 (relative; absolute
// when the smallest lane value is below 1e-11 in magnitude).  Its status, the statuses it lends its
// neighbours and a per-rank count of inactive buffers follow the rules of equilibriumAccelerationUpdate and
// isEquilibriumAccelerationCurrentPointDisabled; a rank whose count equals its number of buffers skips the
// 1D solve (compute.tpp:261-265).
//
// The walk is sequential only through one bit: whether buffer b-1 "touched" buffer b (was stimulated, or
// ended active), which turns an inactive b into neighbor_is_active before b runs.  Everything else a buffer
// does is decided by its own data.  So on the GPU:
//   1. every node computes its half step speculatively twice — variant A: all substeps (as an active buffer
//      does), variant B: from the substep at which its buffer's junction machine first stimulates (as an
//      inactive junction buffer does) — into separate arrays (reaction_eq_kernel);
//   2. every buffer evaluates the equilibrium test of both variants (eq_changed_kernel);
//   3. the touch bit is scanned over the buffers of each rank: each buffer is a map {0,1} -> {0,1}, and maps
//      compose (eq_scan_block_kernel, eq_scan_top_kernel);
//   4. every buffer then knows how it ran: commits variant A, B or nothing, writes its final status, and adds
//      its share of the count changes (eq_commit_kernel).
// The padding lanes of a rank's last buffer (past its last node) run like nodes, as in the reference, from
// their own small arrays; they enter only the equilibrium test.
#pragma once
#include "fdm_kernels.cuh"

namespace fdm {

enum : uint8_t { EQ_INACTIVE = 0, EQ_NEIGHBOR_ACTIVE = 1, EQ_ACTIVE = 2 };
constexpr int EQ_SCAN_T = 256; // buffers per block of the touch-bit scan

struct EqLayout {
  int W;
  int n_ranks;
  int64_t n_nodes;            // real nodes
  int n_pad;                  // padding lanes of all ranks
  int64_t n_buffers;          // buffers of all ranks, rank after rank
  const int* buf_of;          // [n_nodes + n_pad] buffer of a node / of a padding lane
  const int* lane_node;       // [buffer * W + lane] node, or n_nodes + padding lane
  const int* jfiber;          // [buffer] fiber whose stimulation machine runs in the buffer, or -1
  const int* buf_rank;        // [buffer]
  const int* rank_first;      // [n_ranks + 1] first buffer of each rank
  int* counter;               // [n_ranks] count of buffers set inactive (in/out)
  const uint8_t* st_in;       // [buffer] statuses before the half step
  uint8_t* st_out;            // [buffer] statuses after it
};

// speculative results, index space [0, n_nodes) real nodes, [n_nodes, n_nodes + n_pad) padding lanes
struct EqSpec {
  int64_t nt;                 // n_nodes + n_pad (stride of the arrays below)
  double* vm_pad;             // padding lanes: Vm, states (RR), residuals (RR), parameters (RR), stride n_pad
  void* states_pad;
  void* states_lo_pad;
  const void* params_pad;
  const int* pad_clamp;       // fiber whose machine clamps the padding lane, or -1
  const int* pad_gate;        // onlyComputeIfHasBeenStimulated code of the padding lane (its buffer's)
  double* vm_a;               // variant A / B results, stride nt
  void* st_a;
  void* stl_a;
  double* alg_a;              // [k * nt + i] algebraics for transfer of the last substep
  double* vm_b;
  void* st_b;
  void* stl_b;
  double* alg_b;
  uint8_t* ran_b;             // [i] 1 if variant B ran (its buffer's junction machine stimulated)
};

template<class Model, class RR, class Math>
__global__ void __launch_bounds__(128) reaction_eq_kernel(ReactionArgs a, EqLayout L, EqSpec e)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= e.nt)
    return;
  constexpr int NS = Model::nStates;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  constexpr int NSM = NS > 1 ? NS - 1 : 1;
  const bool pad = i >= a.n_nodes;
  const int64_t pi = i - a.n_nodes;
  const int64_t stride = pad ? L.n_pad : a.stride;
  const int64_t j = pad ? pi : i;
  const RR* st = (const RR*)(pad ? e.states_pad : a.states);
  const RR* stl = (const RR*)(pad ? e.states_lo_pad : a.states_lo);
  const RR* pr = (const RR*)(pad ? e.params_pad : a.params);
  const double V0 = pad ? e.vm_pad[pi] : a.vm[i];
  RR S0[NSM], L0[NSM], P[NP];
#pragma unroll
  for (int s = 1; s < NS; s++) {
    S0[s - 1] = st[(s - 1) * stride + j];
    L0[s - 1] = Compensated<RR>::value ? stl[(s - 1) * stride + j] : (RR)0;
  }
#pragma unroll
  for (int q = 0; q < Model::nParameters; q++)
    P[q] = pr[q * stride + j];
  const int cf = pad ? e.pad_clamp[pi] : a.clamp_fiber[i];
  const SplitStep s = a.steps[a.step];
  const double t0 = a.half ? s.mid : s.t;
  const int base = (a.step * 2 + a.half) * a.nsub_stride;
  const int first =
      a.gate ? gate_first(a.gate_start, a.gate_stride, pad ? e.pad_gate[pi] : a.gate[i], a.step * 2 + a.half) : 0;
  // the substep at which the machine of the buffer's junction fiber first stimulates (variant B), or -1
  const int jf = L.jfiber[L.buf_of[i]];
  int kstar = -1;
  if (jf >= 0)
    for (int k = 0; k < s.n0 && kstar < 0; k++)
      if (stim_bit(a.flags, a.words_per_fiber, jf, base + k))
        kstar = k;
  RR* sta = (RR*)e.st_a;
  RR* stla = (RR*)e.stl_a;
  RR* stb = (RR*)e.st_b;
  RR* stlb = (RR*)e.stl_b;
  for (int variant = 0; variant < (kstar >= 0 ? 2 : 1); variant++) {
    double V = V0;
    RR S[NSM], Lo[NSM];
#pragma unroll
    for (int q = 0; q < NSM; q++) {
      S[q] = S0[q];
      Lo[q] = L0[q];
    }
    const int k0 = variant == 0 ? first : max(first, kstar);
    double* alg_out = variant == 0 ? e.alg_a : e.alg_b;
    for (int k = k0; k < s.n0; k++) {
      const double t = xadd(t0, xmul((double)k, s.dt0));
      const bool stim = cf >= 0 && stim_bit(a.flags, a.words_per_fiber, cf, base + k);
      RR Pk[NP];
#pragma unroll
      for (int q = 0; q < NP; q++)
        Pk[q] = (stim && a.stimulus_mode == 1 && q == a.stimulus_parameter) ? (RR)a.stimulus_value : P[q];
      const bool vclamp = stim && a.stimulus_mode == 0;
      if (a.store_alg && k == s.n0 - 1) {
        RR alg[Model::nAlgebraics];
        heun_step<Model, RR, Math, true>(V, S, Lo, Pk, t, s.dt0, vclamp, a.vstim, alg);
        store_algebraics<Model>(alg, a.n_alg_out, a.alg_indices, alg_out, e.nt, i);
      } else {
        heun_step<Model, RR, Math, false>(V, S, Lo, Pk, t, s.dt0, vclamp, a.vstim, nullptr);
      }
    }
    double* vmo = variant == 0 ? e.vm_a : e.vm_b;
    RR* sto = variant == 0 ? sta : stb;
    RR* stlo = variant == 0 ? stla : stlb;
    vmo[i] = V;
#pragma unroll
    for (int s2 = 1; s2 < NS; s2++) {
      sto[(s2 - 1) * e.nt + i] = S[s2 - 1];
      if (Compensated<RR>::value)
        stlo[(s2 - 1) * e.nt + i] = Lo[s2 - 1];
    }
  }
  e.ran_b[i] = kstar >= 0 ? 1 : 0;
}

// equilibrium test of one buffer for the results (vm, st, stl): 1 if some state of some lane changed by more
// than 1e-6 (compute.tpp:650-690; the lane values of a state are its FP64 value, residual included)
template<class RR>
__device__ __forceinline__ bool eq_changed(const EqLayout& L, const ReactionArgs& a, const EqSpec& e, int64_t b,
                                           int n_states, const double* vm_new, const RR* st_new, const RR* stl_new)
{
  auto old_value = [&](int s, int64_t node) -> double {
    const bool pad = node >= a.n_nodes;
    if (s == 0)
      return pad ? e.vm_pad[node - a.n_nodes] : a.vm[node];
    const RR* st = (const RR*)(pad ? e.states_pad : a.states);
    const RR* stl = (const RR*)(pad ? e.states_lo_pad : a.states_lo);
    const int64_t stride = pad ? L.n_pad : a.stride;
    const int64_t j = pad ? node - a.n_nodes : node;
    return (double)st[(s - 1) * stride + j] + (Compensated<RR>::value ? (double)stl[(s - 1) * stride + j] : 0.0);
  };
  auto new_value = [&](int s, int64_t node) -> double {
    if (s == 0)
      return vm_new[node];
    return (double)st_new[(s - 1) * e.nt + node] +
           (Compensated<RR>::value ? (double)stl_new[(s - 1) * e.nt + node] : 0.0);
  };
  for (int s = 0; s < n_states; s++) {
    double vmin = INFINITY;
    for (int lane = 0; lane < L.W; lane++)
      vmin = fmin(vmin, new_value(s, L.lane_node[b * L.W + lane]));
    const bool absolute = fabs(vmin) < 1e-11;
    double change = 0.0;
    for (int lane = 0; lane < L.W; lane++) {
      const int64_t node = L.lane_node[b * L.W + lane];
      const double nv = new_value(s, node), ov = old_value(s, node);
      const double c = absolute ? fabs(nv - ov) : fabs((nv - ov) / nv);
      if (!(c <= change))
        change = c == c ? c : INFINITY;
    }
    if (change > 1e-6)
      return true;
  }
  return false;
}

#ifdef FDM_COMMON_KERNELS_TU
// per buffer: bit 0 = variant A changed, bit 1 = variant B changed, bit 2 = stimulated (variant B ran)
template<class RR>
__global__ void eq_changed_kernel(ReactionArgs a, EqLayout L, EqSpec e, int n_states, uint8_t* info)
{
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= L.n_buffers)
    return;
  uint8_t v = eq_changed<RR>(L, a, e, b, n_states, e.vm_a, (const RR*)e.st_a, (const RR*)e.stl_a) ? 1 : 0;
  const int64_t n0 = L.lane_node[b * L.W];
  if (e.ran_b[n0]) {
    v |= 4;
    if (eq_changed<RR>(L, a, e, b, n_states, e.vm_b, (const RR*)e.st_b, (const RR*)e.stl_b))
      v |= 2;
  }
  info[b] = v;
}

// status of buffer b at the start of the call (the first and the last buffer of a rank are set active)
__device__ __forceinline__ uint8_t eq_start_status(const EqLayout& L, int64_t b)
{
  const int r = L.buf_rank[b];
  if (b == L.rank_first[r] || b == L.rank_first[r + 1] - 1)
    return EQ_ACTIVE;
  return L.st_in[b];
}

// how buffer b runs given whether its left neighbour touched it: variant (0 none, 1 A, 2 B), own final status,
// and whether it touches its neighbours
struct EqRun {
  int variant;
  uint8_t final_own;
  bool touches;
};
__device__ __forceinline__ EqRun eq_run(const EqLayout& L, const uint8_t* info, int64_t b, bool touched)
{
  const uint8_t v = info[b];
  const bool stim = v & 4;
  uint8_t st = eq_start_status(L, b);
  if (st == EQ_INACTIVE && touched)
    st = EQ_NEIGHBOR_ACTIVE;
  EqRun r;
  if (st != EQ_INACTIVE) {
    r.variant = 1; // runs every substep (a stimulation only confirms "active")
    const bool changed = v & 1;
    r.final_own = changed ? EQ_ACTIVE : EQ_INACTIVE;
  } else if (stim) {
    r.variant = 2; // turned active by its stimulation: runs from the stimulating substep on
    const bool changed = v & 2;
    r.final_own = changed ? EQ_ACTIVE : EQ_INACTIVE;
  } else {
    r.variant = 0;
    r.final_own = EQ_INACTIVE;
  }
  r.touches = stim || r.final_own == EQ_ACTIVE;
  return r;
}

// scan of the touch bit: map of buffer b as 2 bits (value for input 0, value for input 1); a rank's first
// buffer has no left neighbour (constant map of input 0)
__device__ __forceinline__ uint8_t eq_map(const EqLayout& L, const uint8_t* info, int64_t b)
{
  const bool head = b == L.rank_first[L.buf_rank[b]];
  const uint8_t m0 = eq_run(L, info, b, false).touches ? 1 : 0;
  const uint8_t m1 = head ? m0 : (eq_run(L, info, b, true).touches ? 1 : 0);
  return (uint8_t)(m0 | (m1 << 1));
}
// second o first
__device__ __forceinline__ uint8_t eq_compose(uint8_t first, uint8_t second)
{
  const uint8_t f0 = first & 1, f1 = (first >> 1) & 1;
  const uint8_t r0 = (second >> f0) & 1, r1 = (second >> f1) & 1;
  return (uint8_t)(r0 | (r1 << 1));
}

// per block: exclusive prefix maps within the block (prefix[b] = composition of the maps before b in the block)
// and the block's aggregate
__global__ void __launch_bounds__(EQ_SCAN_T) eq_scan_block_kernel(EqLayout L, const uint8_t* info, uint8_t* prefix,
                                                                  uint8_t* block_agg)
{
  __shared__ uint8_t sm[EQ_SCAN_T];
  const int64_t b = (int64_t)blockIdx.x * EQ_SCAN_T + threadIdx.x;
  const uint8_t identity = 0b10;
  uint8_t m = b < L.n_buffers ? eq_map(L, info, b) : identity;
  sm[threadIdx.x] = m;
  __syncthreads();
  // Hillis-Steele inclusive scan of maps
  for (int off = 1; off < EQ_SCAN_T; off <<= 1) {
    uint8_t x = sm[threadIdx.x];
    if ((int)threadIdx.x >= off)
      x = eq_compose(sm[threadIdx.x - off], x);
    __syncthreads();
    sm[threadIdx.x] = x;
    __syncthreads();
  }
  if (b < L.n_buffers)
    prefix[b] = threadIdx.x > 0 ? sm[threadIdx.x - 1] : identity;
  if (threadIdx.x == EQ_SCAN_T - 1)
    block_agg[blockIdx.x] = sm[EQ_SCAN_T - 1];
}

// exclusive scan of the block aggregates (one thread; a few thousand blocks at most per million buffers)
__global__ void eq_scan_top_kernel(uint8_t* block_agg, int64_t n_blocks)
{
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  uint8_t acc = 0b10;
  for (int64_t k = 0; k < n_blocks; k++) {
    const uint8_t m = block_agg[k];
    block_agg[k] = acc;
    acc = eq_compose(acc, m);
  }
}

// touch bit entering buffer b
__device__ __forceinline__ bool eq_touched(const EqLayout& L, const uint8_t* prefix, const uint8_t* block_agg,
                                           int64_t b)
{
  const uint8_t m = eq_compose(block_agg[b / EQ_SCAN_T], prefix[b]);
  return m & 1; // applied to 0 (nothing left of the rank's first buffer; its map is constant)
}

// one thread per buffer: commit the variant, final status, count changes
template<class RR>
__global__ void eq_commit_kernel(ReactionArgs a, EqLayout L, EqSpec e, const uint8_t* info, const uint8_t* prefix,
                                 const uint8_t* block_agg, int n_states)
{
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= L.n_buffers)
    return;
  const int r = L.buf_rank[b];
  const int64_t first = L.rank_first[r], last = L.rank_first[r + 1] - 1;
  const EqRun run = eq_run(L, info, b, b > first && eq_touched(L, prefix, block_agg, b));
  // final status: an inactive buffer is set neighbor_is_active by a right neighbour that touches it
  uint8_t fin = run.final_own;
  if (b < last && fin == EQ_INACTIVE) {
    const EqRun right = eq_run(L, info, b + 1, run.touches);
    if (right.touches)
      fin = EQ_NEIGHBOR_ACTIVE;
  }
  L.st_out[b] = fin;
  // count: +1 when the buffer ran and ends inactive; -1 for each neighbour it finds inactive when it touches it
  int delta = (run.variant != 0 && run.final_own == EQ_INACTIVE) ? 1 : 0;
  if (run.touches) {
    if (b > first) {
      const EqRun left = eq_run(L, info, b - 1, b - 1 > first && eq_touched(L, prefix, block_agg, b - 1));
      if (left.final_own == EQ_INACTIVE)
        delta--;
    }
    if (b < last && eq_start_status(L, b + 1) == EQ_INACTIVE)
      delta--;
  }
  if (delta)
    atomicAdd(&L.counter[r], delta);
  // commit the lanes
  RR* st = (RR*)a.states;
  RR* stl = (RR*)a.states_lo;
  RR* stp = (RR*)e.states_pad;
  RR* stlp = (RR*)e.states_lo_pad;
  const RR* sa = (const RR*)(run.variant == 2 ? e.st_b : e.st_a);
  const RR* sla = (const RR*)(run.variant == 2 ? e.stl_b : e.stl_a);
  const double* va = run.variant == 2 ? e.vm_b : e.vm_a;
  const double* alg = run.variant == 2 ? e.alg_b : e.alg_a;
  if (run.variant == 0)
    return;
  for (int lane = 0; lane < L.W; lane++) {
    const int64_t node = L.lane_node[b * L.W + lane];
    const bool pad = node >= a.n_nodes;
    const int64_t j = pad ? node - a.n_nodes : node;
    const int64_t stride = pad ? L.n_pad : a.stride;
    (pad ? e.vm_pad : a.vm)[j] = va[node];
    for (int s = 1; s < n_states; s++) {
      (pad ? stp : st)[(s - 1) * stride + j] = sa[(s - 1) * e.nt + node];
      if (Compensated<RR>::value)
        (pad ? stlp : stl)[(s - 1) * stride + j] = sla[(s - 1) * e.nt + node];
    }
    if (!pad && a.store_alg)
      for (int k = 0; k < a.n_alg_out; k++)
        a.alg_out[k * a.n_nodes + node] = alg[k * e.nt + node];
  }
}

// Vm of the traced nodes after a half step 1 (the speculative kernel does not write the trace)
__global__ void eq_trace_kernel(ReactionArgs a)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_nodes || !a.trace_slot)
    return;
  const SplitStep s = a.steps[a.step];
  const int slot = a.trace_slot[i];
  if (slot >= 0)
    record_trace(a.trace, a.n_trace, a.trace_capacity, a.act, slot, s.global_no, a.vm[i]);
}
#endif // FDM_COMMON_KERNELS_TU

} // namespace fdm
