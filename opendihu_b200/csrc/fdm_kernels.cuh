// Device kernels of the fiber monodomain hot path (sm_100a).
//
// One Strang step of the reference (fast_monodomain_solver_compute.tpp:111-126) is
//   n0D Heun substeps of the CellML model on every node   (compute0D, :131-254)
//   one tridiagonal solve per fiber for the diffusion      (compute1D, :256-507)
//   n0D Heun substeps starting at the mid time             (compute0D)
// The kernels here implement it in two shapes:
//   split:  reaction_kernel (one thread per node, states in HBM) + diffusion_warp_kernel (one warp per
//           fiber, a partitioned Thomas sweep whose forward results go to a scratch array in HBM);
//   fused:  fused_kernel (one CTA per bin of whole fibers; every thread keeps M nodes' states in
//           registers across all split steps of a launch; the tridiagonal solve is a block-wide
//           scan of affine maps in FP64; coefficients live in shared memory).
// A stimulation_schedule_kernel advances each fiber's motor-unit stimulation machine
// (compute.tpp:509-627) over all substeps of a launch window and writes one bit per substep.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include <cooperative_groups.h>

#include "fdm_math.cuh"

namespace fdm {

namespace cg = cooperative_groups;

// --------------------------------------------------------------------------------------------
// exact (never contracted) FP64 arithmetic for time values, so that the discrete stimulation
// decisions are evaluated exactly as the C expressions are written
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// one Strang step of a launch window (host computes these with the reference's time rules)
struct SplitStep {
  double t;      // currentTime of the split step
  double mid;    // midTime = currentTime + 0.5*dtSplit
  double dt0;    // Heun substep width
  int n0;        // number of Heun substeps per half step
  int global_no; // split step number since the trace was set (trace row)
};

// Activation recording on the traced nodes: after every Strang step, a node whose Vm rose above the threshold
// (Vm after the previous step <= threshold < Vm now) records the step's trace row; the first `capacity` rows
// per node are kept, `count` counts them all.  `prev` starts as NaN, so the first step after the recording
// starts never records.  Each traced node is written by one thread per step: no atomics.
struct ActivationRec {
  double threshold;
  double* prev;                   // [slot] Vm after the previous step (null: recording off)
  int* count;                     // [slot]
  int* steps;                     // [slot * capacity + k]
  int capacity;
};

// the trace value of a traced node after a Strang step, and its activation record
__device__ __forceinline__ void record_trace(double* trace, int n_trace, int64_t capacity, const ActivationRec& act,
                                             int slot, int row, double V)
{
  if (row < capacity)
    trace[(int64_t)row * n_trace + slot] = V;
  if (act.prev) {
    const double p = act.prev[slot];
    if (p <= act.threshold && V > act.threshold) {
      const int c = act.count[slot];
      if (c < act.capacity)
        act.steps[(int64_t)slot * act.capacity + c] = row;
      act.count[slot] = c + 1;
    }
    act.prev[slot] = V;
  }
}

struct StimArgs {
  const uint8_t* firing_events;   // [row][col]
  int rows, cols;
  const int* motor_unit_no;       // per fiber (device order)
  const double* call_frequency;
  const double* repeat_after_first_call;
  const double* call_enable_begin;
  const double* jitter;           // per fiber n_jitter values
  int n_jitter;
  const uint8_t* evaluated;       // per fiber: 1 if the stimulation machine is advanced
  double* last_check_time;        // machine state, persistent across launches
  double* current_jitter;
  int* jitter_index;
  uint8_t* has_been_stimulated;
  uint32_t* flags;                // [fiber][words_per_fiber] one bit per substep of the window
  int words_per_fiber;
  int nsub_stride;                // bit index = (step*2 + half)*nsub_stride + substep
  int n_fibers;
  uint8_t* gate_start;            // onlyComputeIfHasBeenStimulated (or null): per fiber and half step of the
  int gate_stride;                // window, 0 if the fiber's flag was set before the half step, 1 + the
                                  // substep that sets it, 255 if it stays unset:
                                  // [fiber * gate_stride + step*2 + half]
  uint8_t* currently;             // stimulation log (or null): per fiber, did its last decision stimulate
  double* log_time;               // (time, fiber) of every stimulation begin, log_capacity entries;
  int* log_fiber;                 // log_count counts all of them (null: no entries are written)
  unsigned long long* log_count;
  long long log_capacity;
};

// onlyComputeIfHasBeenStimulated: the first substep of half step hs that a node with gate code `code`
// (attributed fiber * 4 + class, class 0/1/2 = buffer before / at / after the junction buffer) computes;
// 255 = none (compute.tpp:201-205 in the reference's buffer order: a buffer before the junction buffer
// still sees the flag unset, the junction buffer computes from the stimulating substep on, a buffer after
// it sees the flag set)
__device__ __forceinline__ int gate_first(const uint8_t* __restrict__ gate_start, int gate_stride, int code, int hs)
{
  const int st = gate_start[(int64_t)(code >> 2) * gate_stride + hs];
  const int cls = code & 3;
  if (st == 0 || st == 255)
    return st;
  return cls == 1 ? st - 1 : (cls == 0 ? 255 : 0);
}

// isCurrentPointStimulated (compute.tpp:509-627), one fiber, one substep
__device__ __forceinline__ bool stimulation_machine(const StimArgs& a, int f, double t, double& last, double& jit,
                                                    int& jidx)
{
  const double freq = a.call_frequency[f];
  const double repeat = a.repeat_after_first_call[f];
  const double begin = a.call_enable_begin[f];
  bool check = false;
  if (t >= xadd(last, xdiv(1.0, xadd(freq, jit))) && t >= xsub(begin, 1e-13)) {
    check = true;
    if (repeat != 0 && xsub(t, xadd(last, xdiv(1.0, xadd(freq, jit)))) > repeat) {
      last = xadd(last, xdiv(1.0, xadd(freq, jit)));
      double jf = 0.0;
      if (a.n_jitter > 0)
        jf = a.jitter[(int64_t)f * a.n_jitter + jidx % a.n_jitter];
      jit = xmul(jf, freq);
      jidx++;
      check = false;
    }
  }
  const int index = (int)round(xmul(t, freq));
  int row = index % a.rows;
  if (row < 0)
    row += a.rows;
  const int col = a.motor_unit_no[f] % a.cols;
  return check && a.firing_events[(int64_t)row * a.cols + col] != 0;
}

#ifdef FDM_COMMON_KERNELS_TU
__global__ void stimulation_schedule_kernel(StimArgs a, const SplitStep* __restrict__ steps, int n_steps)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.n_fibers)
    return;
  uint32_t* fl = a.flags + (int64_t)f * a.words_per_fiber;
  for (int w = 0; w < a.words_per_fiber; w++)
    fl[w] = 0u;
  if (!a.evaluated[f]) {
    if (a.gate_start) {
      const uint8_t g = a.has_been_stimulated[f] ? 0 : 255;
      for (int hs = 0; hs < 2 * n_steps; hs++)
        a.gate_start[(int64_t)f * a.gate_stride + hs] = g;
    }
    return;
  }
  double last = a.last_check_time[f], jit = a.current_jitter[f];
  int jidx = a.jitter_index[f];
  uint8_t hbs = a.has_been_stimulated[f];
  uint8_t cur = a.currently ? a.currently[f] : 0;
  for (int j = 0; j < n_steps; j++) {
    const SplitStep s = steps[j];
    for (int h = 0; h < 2; h++) {
      const double t0 = h ? s.mid : s.t;
      uint32_t word = 0u;
      int word_no = -1;
      int first = hbs ? 0 : 255;
      for (int k = 0; k < s.n0; k++) {
        const double t = xadd(t0, xmul((double)k, s.dt0));
        const bool st = stimulation_machine(a, f, t, last, jit, jidx);
        // StimulationLogging::logStimulationBegin at the first stimulating decision (compute.tpp:603-607)
        if (st && !cur && a.log_count) {
          const unsigned long long idx = atomicAdd(a.log_count, 1ull);
          if (idx < (unsigned long long)a.log_capacity) {
            a.log_time[idx] = t;
            a.log_fiber[idx] = f;
          }
        }
        cur = st ? 1 : 0;
        if (st) {
          if (first == 255)
            first = k + 1;
          hbs = 1;
          const int bit = (j * 2 + h) * a.nsub_stride + k;
          if (bit / 32 != word_no) {
            if (word_no >= 0)
              fl[word_no] |= word;
            word_no = bit / 32;
            word = 0u;
          }
          word |= 1u << (bit % 32);
        }
      }
      if (word_no >= 0)
        fl[word_no] |= word;
      if (a.gate_start)
        a.gate_start[(int64_t)f * a.gate_stride + j * 2 + h] = (uint8_t)first;
    }
  }
  a.last_check_time[f] = last;
  a.current_jitter[f] = jit;
  a.jitter_index[f] = jidx;
  a.has_been_stimulated[f] = hbs;
  if (a.currently)
    a.currently[f] = cur;
}

#endif // FDM_COMMON_KERNELS_TU

__device__ __forceinline__ bool stim_bit(const uint32_t* __restrict__ flags, int words_per_fiber, int fiber, int bit)
{
  return (__ldg(flags + (int64_t)fiber * words_per_fiber + (bit >> 5)) >> (bit & 31)) & 1u;
}

// --------------------------------------------------------------------------------------------
// one Heun step (03_generator_vc.cpp:1017-1130):
//   y* = y + dt f(y); [Vm* := vStim]; y += dt/2 (f(y) + f(y*)); [Vm := vStim]
// Vm is carried in FP64; the other states and the rates in RR (double or float).
// In FP32 every state other than Vm is a pair (S, L) whose sum is the value: the update
// S + dt/2 (f + f*) is accumulated with Fast2Sum (error of the addition kept in L).  Without it,
// increments below half an FP32 ulp of the gate are lost at every step and the slowly relaxing
// gates stagnate (a single HH cell at rest drifts 6e-3 mV from FP64 within 10 ms; with the
// compensation 1e-6 mV).
// --------------------------------------------------------------------------------------------
template<class RR>
struct Compensated {
  static constexpr bool value = false;
};
template<>
struct Compensated<float> {
  static constexpr bool value = true;
};

template<class RR>
__device__ __forceinline__ void accumulate(RR& s, RR& l, RR inc)
{
  if (Compensated<RR>::value) {
    inc += l;
    const RR t = s + inc;
    l = inc - (t - s);
    s = t;
  } else {
    s += inc;
  }
}

// right-hand side: the FP32 exact-exp mode uses the model's shared-exponential form (fewer SFU
// operations); FP64 and the approximate-exp policy (whose exp is not multiplicative) use the plain form
template<class Model, class RR, class Math>
__device__ __forceinline__ void model_rates(const RR t, const RR* y, const RR* P, RR* r, RR* alg)
{
  if constexpr (std::is_same<RR, float>::value && std::is_same<Math, fdm_math_exact>::value)
    Model::template rates_fast<RR, Math>(t, y, P, r, alg);
  else
    Model::template rates<RR, Math>(t, y, P, r, alg);
}

template<class Model, class RR, class Math, bool STORE>
__device__ __forceinline__ void heun_step(double& V, RR* __restrict__ S, RR* __restrict__ L,
                                          const RR* __restrict__ P, double t, double dt, bool clamp, double vstim,
                                          RR* __restrict__ alg_store)
{
  constexpr int NS = Model::nStates;
  RR y[NS], r[NS], ys[NS], r2[NS];
  RR alg[Model::nAlgebraics], alg2[Model::nAlgebraics];
  y[0] = (RR)V;
#pragma unroll
  for (int s = 1; s < NS; s++)
    y[s] = S[s - 1];
  const RR tr = (RR)t;
  model_rates<Model, RR, Math>(tr, y, P, r, alg);
  const RR dtr = (RR)dt;
  if (Compensated<RR>::value) {
    // FP32 reaction: y* only feeds the FP32 right-hand side, so Vm* is formed in FP32; the increment of Vm
    // is formed in FP32 and accumulated into the FP64 Vm (one conversion each way per substep)
    ys[0] = y[0] + dtr * r[0];
  } else {
    ys[0] = (RR)(V + dt * (double)r[0]);
  }
#pragma unroll
  for (int s = 1; s < NS; s++)
    ys[s] = y[s] + dtr * r[s];
  if (clamp)
    ys[0] = (RR)vstim;
  model_rates<Model, RR, Math>(tr, ys, P, r2, alg2);
  if (Compensated<RR>::value)
    V += (double)((RR)0.5 * dtr * (r[0] + r2[0]));
  else
    V += 0.5 * dt * ((double)r[0] + (double)r2[0]);
#pragma unroll
  for (int s = 1; s < NS; s++)
    accumulate<RR>(S[s - 1], L[s - 1], (RR)0.5 * dtr * (r[s] + r2[s]));
  if (clamp)
    V = vstim;
  if (STORE) {
#pragma unroll
    for (int k = 0; k < Model::nAlgebraics; k++)
      alg_store[k] = alg2[k];
  }
}

// The FP32 Heun step of two nodes at once, over fdm_f2 pairs (packed FP32 instructions).  Every state
// other than Vm is a pair (S, L) whose sum is its value: within a half step the increments dt/2 (f + f*) are
// summed into L and the right-hand side sees S + L; normalize_pair folds L back into S (Fast2Sum) at the end
// of the half step.  L stays of the size of a few increments, so no increment is lost against S (the
// stagnation the compensation exists for) at four packed operations per state and substep instead of the
// seven of a Fast2Sum per substep.  Vm is carried the same way: Vf is the node pair's Vm rounded to FP32 at
// the start of the half step and LV the sum of its increments since then; the right-hand side sees Vf + LV,
// and the caller adds LV to the FP64 Vm once, at the end of the half step, so no FP64 <-> FP32 conversion
// and no FP64 addition is left in the substep loop.  A clamped lane restarts from the stimulation value: its
// FP64 Vm is set, Vf holds the value, LV restarts at 0.  dtr / hdt are the step width and its half per node
// (a node that skips the substep has 0: y* = y, and the states stay as they are).  Used with the FP32
// exact-exponential policy only.
template<class Model>
__device__ __forceinline__ void heun_step2(fdm_f2& Vf, fdm_f2& LV, double& V0, double& V1,
                                               const fdm_f2* __restrict__ S, fdm_f2* __restrict__ L,
                                               const fdm_f2* __restrict__ P, const fdm_f2 tr, fdm_f2 dtr, fdm_f2 hdt,
                                               bool clamp0, bool clamp1, double vstim)
{
  constexpr int NS = Model::nStates;
  const float vs = (float)vstim;
  fdm_f2 y[NS], r[NS], ys[NS], r2[NS];
  fdm_f2 alg[Model::nAlgebraics];
  y[0] = Vf + LV;
#pragma unroll
  for (int s = 1; s < NS; s++)
    y[s] = S[s - 1] + L[s - 1];
  Model::template rates_fast2<fdm_math_exact>(tr, y, P, r, alg);
#pragma unroll
  for (int s = 0; s < NS; s++)
    ys[s] = dtr * r[s] + y[s];
  if (clamp0)
    ys[0].v.x = vs;
  if (clamp1)
    ys[0].v.y = vs;
  Model::template rates_fast2<fdm_math_exact>(tr, ys, P, r2, alg);
#pragma unroll
  for (int s = 1; s < NS; s++)
    L[s - 1] = hdt * (r[s] + r2[s]) + L[s - 1];
  LV = hdt * (r[0] + r2[0]) + LV;
  if (clamp0) {
    V0 = vstim;
    Vf.v.x = vs;
    LV.v.x = 0.f;
  }
  if (clamp1) {
    V1 = vstim;
    Vf.v.y = vs;
    LV.v.y = 0.f;
  }
}

// heun_step2 over the MP node pairs of one thread, without branches: every pair computes (the caller zeroes
// the Vm of nodes beyond its bin), clamps are selects (bit 2p / 2p + 1 of `clamp`: node 2p / 2p + 1 clamped;
// a constant 0 removes them).  Arithmetic per pair identical to heun_step2.  (Issuing the pairs' first
// right-hand sides before their second ones measured 0.7 % slower than pair after pair.)
template<class Model, int MP, int NSM, int NP>
__device__ __forceinline__ void heun_step2_pairs(fdm_f2 (&Vf)[MP], fdm_f2 (&LV)[MP], double* V,
                                                 fdm_f2 (&S)[MP][NSM], fdm_f2 (&L)[MP][NSM],
                                                 const fdm_f2 (&P)[MP][NP], const fdm_f2 tr, const fdm_f2 dtr,
                                                 const fdm_f2 hdt, const unsigned clamp, double vstim)
{
  constexpr int NS = Model::nStates;
  const float vs = (float)vstim;
  fdm_f2 alg[Model::nAlgebraics];
#pragma unroll
  for (int p = 0; p < MP; p++) {
    fdm_f2 r[NS], ys[NS], y[NS], r2[NS];
    y[0] = Vf[p] + LV[p];
#pragma unroll
    for (int s = 1; s < NS; s++)
      y[s] = S[p][s - 1] + L[p][s - 1];
    Model::template rates_fast2<fdm_math_exact>(tr, y, P[p], r, alg);
#pragma unroll
    for (int s = 0; s < NS; s++)
      ys[s] = dtr * r[s] + y[s];
    ys[0].v.x = ((clamp >> (2 * p)) & 1u) ? vs : ys[0].v.x;
    ys[0].v.y = ((clamp >> (2 * p + 1)) & 1u) ? vs : ys[0].v.y;
    Model::template rates_fast2<fdm_math_exact>(tr, ys, P[p], r2, alg);
#pragma unroll
    for (int s = 1; s < NS; s++)
      L[p][s - 1] = hdt * (r[s] + r2[s]) + L[p][s - 1];
    LV[p] = hdt * (r[0] + r2[0]) + LV[p];
    const bool c0 = (clamp >> (2 * p)) & 1u, c1 = (clamp >> (2 * p + 1)) & 1u;
    V[2 * p] = c0 ? vstim : V[2 * p];
    V[2 * p + 1] = c1 ? vstim : V[2 * p + 1];
    Vf[p].v.x = c0 ? vs : Vf[p].v.x;
    Vf[p].v.y = c1 ? vs : Vf[p].v.y;
    LV[p].v.x = c0 ? 0.f : LV[p].v.x;
    LV[p].v.y = c1 ? 0.f : LV[p].v.y;
  }
}

// (S, L) -> (S + L rounded, the rounding error): the Fast2Sum normalization of a compensated pair
__device__ __forceinline__ void normalize_pair(fdm_f2& S, fdm_f2& L)
{
  const fdm_f2 t = S + L;
  L = L - (t - S);
  S = t;
}

// the CellmlAdapter's generic right-hand side: one thread per instance, SoA var[index * n + i]
template<class Model, class Math>
__global__ void __launch_bounds__(128) cellml_rhs_kernel(int64_t n, double t, const double* __restrict__ states,
                                                        const double* __restrict__ params, double* __restrict__ rates,
                                                        double* __restrict__ algebraics)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  constexpr int NS = Model::nStates;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  double y[NS], r[NS], P[NP], alg[Model::nAlgebraics];
#pragma unroll
  for (int k = 0; k < Model::nAlgebraics; k++)
    alg[k] = 0.0; // algebraics replaced by parameters are not assigned
#pragma unroll
  for (int s = 0; s < NS; s++)
    y[s] = states[s * n + i];
#pragma unroll
  for (int q = 0; q < Model::nParameters; q++)
    P[q] = params[q * n + i];
  Model::template rates<double, Math>(t, y, P, r, alg);
#pragma unroll
  for (int s = 0; s < NS; s++)
    rates[s * n + i] = r[s];
  if (algebraics) {
#pragma unroll
    for (int k = 0; k < Model::nAlgebraics; k++)
      algebraics[k * n + i] = alg[k];
  }
}

// "initializeStatesToEquilibrium" (CellmlAdapter::initializeToEquilibriumValues, 03_cellml_adapter.tpp:445-515):
// classical RK4 steps of one instance (the time stays at 0: t, t + dt/2, t + dt) until the largest state
// increment (k1 + 2 k2 + 2 k3 + k4)/6 falls below 1e-5; an increment above 1e4 restarts from the initial values
// with dt/2.  One thread; a launch does at most max_iterations steps, the host repeats it up to the total limit.
struct EquilibriumSearch {
  double dt;
  double max_increment;
  int64_t iterations;
  int max_rate_no;
  int done;
};

template<class Model, class Math>
__global__ void equilibrium_search_kernel(double* __restrict__ u, const double* __restrict__ u0,
                                   const double* __restrict__ P, EquilibriumSearch* __restrict__ es,
                                   int64_t max_iterations)
{
  if (blockIdx.x != 0 || threadIdx.x != 0 || es->done)
    return;
  constexpr int NS = Model::nStates;
  double y[NS], k1[NS], k2[NS], k3[NS], k4[NS], w[NS], alg[Model::nAlgebraics];
#pragma unroll
  for (int s = 0; s < NS; s++)
    y[s] = u[s];
  double dt = es->dt, inc_max = es->max_increment;
  int rate_no = es->max_rate_no;
  for (int64_t it = 0; it < max_iterations; it++) {
    Model::template rates<double, Math>(0.0, y, P, k1, alg);
#pragma unroll
    for (int s = 0; s < NS; s++)
      w[s] = y[s] + dt / 2. * k1[s];
    Model::template rates<double, Math>(dt / 2., w, P, k2, alg);
#pragma unroll
    for (int s = 0; s < NS; s++)
      w[s] = y[s] + dt / 2. * k2[s];
    Model::template rates<double, Math>(dt / 2., w, P, k3, alg);
#pragma unroll
    for (int s = 0; s < NS; s++)
      w[s] = y[s] + dt * k3[s];
    Model::template rates<double, Math>(dt, w, P, k4, alg);
    inc_max = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
      const double inc = (k1[s] + 2 * k2[s] + 2 * k3[s] + k4[s]) / 6.;
      if (fabs(inc) > inc_max) {
        inc_max = fabs(inc);
        rate_no = s;
      }
      y[s] += dt * inc;
    }
    es->iterations++;
    if (inc_max > 1e4) {
      dt /= 2.0;
#pragma unroll
      for (int s = 0; s < NS; s++)
        y[s] = u0[s];
    }
    if (inc_max < 1e-5) {
      es->done = 1;
      break;
    }
  }
#pragma unroll
  for (int s = 0; s < NS; s++)
    u[s] = y[s];
  es->dt = dt;
  es->max_increment = inc_max;
  es->max_rate_no = rate_no;
}

// algebraicsForTransfer: copy the requested entries (selected at run time) without dynamic
// register indexing
template<class Model, class RR>
__device__ __forceinline__ void store_algebraics(const RR* alg, int n_out, const int* __restrict__ idx,
                                                 double* __restrict__ out, int64_t n_nodes, int64_t node)
{
  for (int q = 0; q < n_out; q++) {
    const int want = idx[q];
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < Model::nAlgebraics; k++)
      v = (k == want) ? (double)alg[k] : v;
    out[q * n_nodes + node] = v;
  }
}

// --------------------------------------------------------------------------------------------
// split path: reaction kernel
// --------------------------------------------------------------------------------------------
struct ReactionArgs {
  int64_t n_nodes;
  int64_t stride;                 // SoA stride of states / parameters
  double* vm;                     // [node]
  void* states;                   // RR [(s-1)*stride + node], s = 1..nStates-1
  void* states_lo;                // FP32 only: compensation terms, same layout
  const void* params;             // RR [p*stride + node]
  const int* clamp_fiber;         // per node: fiber whose machine controls the clamp, or -1
  const uint32_t* flags;
  int words_per_fiber;
  int nsub_stride;
  double vstim;
  int stimulus_mode;              // 0 clamp, 1 current (set parameter)
  int stimulus_parameter;
  double stimulus_value;
  const SplitStep* steps;
  int step;                       // index in window
  int half;                       // 0: first half step, 1: second
  int store_alg;                  // store the requested algebraics after the last substep
  int n_alg_out;
  const int* alg_indices;         // device
  double* alg_out;                // [k][node]
  const int* trace_slot;          // per node slot or -1 (may be null)
  double* trace;                  // [global split no][slot]
  int n_trace;
  int64_t trace_capacity;
  ActivationRec act;
  double* store_states;           // adjoint replay (FP64 only): input state of substep k at
                                  // store_states[(k*nStates + s)*stride + node], or null
  double* store_vm_out;           // adjoint replay: Vm after the half step also written here, or null
  int per_node;                   // 1: one thread per node whatever the size (the adjoint's checkpointed
                                  // forward, which its replay reproduces bit for bit)
  const int* gate;                // onlyComputeIfHasBeenStimulated: per node gate code, or null
  const uint8_t* gate_start;
  int gate_stride;
};

template<class Model, class RR, class Math>
__global__ void __launch_bounds__(128) reaction_kernel(ReactionArgs a)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_nodes)
    return;
  constexpr int NS = Model::nStates;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  RR* st = (RR*)a.states;
  const RR* pr = (const RR*)a.params;
  double V = a.vm[i];
  RR* stl = (RR*)a.states_lo;
  RR S[NS > 1 ? NS - 1 : 1], L[NS > 1 ? NS - 1 : 1];
#pragma unroll
  for (int s = 1; s < NS; s++) {
    S[s - 1] = st[(s - 1) * a.stride + i];
    L[s - 1] = Compensated<RR>::value ? stl[(s - 1) * a.stride + i] : (RR)0;
  }
  RR P[NP], Pstim[NP];
#pragma unroll
  for (int q = 0; q < Model::nParameters; q++) {
    P[q] = pr[q * a.stride + i];
    Pstim[q] = (a.stimulus_mode == 1 && q == a.stimulus_parameter) ? (RR)a.stimulus_value : P[q];
  }
  const int cf = a.clamp_fiber[i];
  const SplitStep s = a.steps[a.step];
  const double t0 = a.half ? s.mid : s.t;
  const int base = (a.step * 2 + a.half) * a.nsub_stride;
  const int first = a.gate ? gate_first(a.gate_start, a.gate_stride, a.gate[i], a.step * 2 + a.half) : 0;
  for (int k = 0; k < s.n0; k++) {
    const double t = xadd(t0, xmul((double)k, s.dt0));
    const bool stim = cf >= 0 && stim_bit(a.flags, a.words_per_fiber, cf, base + k);
    const bool vclamp = stim && a.stimulus_mode == 0;
    if (a.store_states) {
      a.store_states[(int64_t)(k * NS) * a.stride + i] = V;
#pragma unroll
      for (int s2 = 1; s2 < NS; s2++)
        a.store_states[(int64_t)(k * NS + s2) * a.stride + i] = (double)S[s2 - 1];
    }
    if (k < first)
      continue; // not computed before the attributed fiber was stimulated
    RR Pk[NP];
#pragma unroll
    for (int q = 0; q < NP; q++)
      Pk[q] = (stim && a.stimulus_mode == 1) ? Pstim[q] : P[q];
    if (a.store_alg && k == s.n0 - 1) {
      RR alg[Model::nAlgebraics];
      heun_step<Model, RR, Math, true>(V, S, L, Pk, t, s.dt0, vclamp, a.vstim, alg);
      store_algebraics<Model>(alg, a.n_alg_out, a.alg_indices, a.alg_out, a.n_nodes, i);
    } else {
      heun_step<Model, RR, Math, false>(V, S, L, Pk, t, s.dt0, vclamp, a.vstim, nullptr);
    }
  }
  a.vm[i] = V;
  if (a.store_vm_out)
    a.store_vm_out[i] = V;
#pragma unroll
  for (int s2 = 1; s2 < NS; s2++) {
    st[(s2 - 1) * a.stride + i] = S[s2 - 1];
    if (Compensated<RR>::value)
      stl[(s2 - 1) * a.stride + i] = L[s2 - 1];
  }
  if (a.half == 1 && a.trace_slot) {
    const int slot = a.trace_slot[i];
    if (slot >= 0)
      record_trace(a.trace, a.n_trace, a.trace_capacity, a.act, slot, s.global_no, V);
  }
}

// Split-path reaction for few nodes, FP64: the warps of a CTA share 32 nodes, warp g advancing state g of
// each (Model::rates_group evaluates one state's rate from the lines it needs).  With one thread per node a
// problem of a few ten thousand nodes leaves each SM a handful of warps whose Heun chains stall on FP64
// latency; here every node gives nStates independent chains.  The states of the 32 nodes live in shared
// memory; per substep each warp forms its y*, the CTA synchronizes, each warp forms its new state from both
// rates, the CTA synchronizes.  Same expressions and operation order as heun_step (FP64), so the same values.
template<class Model, class Math, int G>
__device__ __forceinline__ double group_rate(int g, double t, const double* y, const double* P)
{
  if constexpr (G < Model::nGroups) {
    if (g == G)
      return Model::template rates_group<double, Math, G>(t, y, P);
    return group_rate<Model, Math, G + 1>(g, t, y, P);
  } else {
    return 0.0;
  }
}

template<class Model, class Math>
__global__ void __launch_bounds__(32 * (Model::nGroups > 0 ? Model::nGroups : 1)) reaction_group_kernel(ReactionArgs a)
{
  constexpr int NS = Model::nStates;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  __shared__ double sy[NS][32], sys[NS][32];
  const int lane = threadIdx.x, g = threadIdx.y;
  const int64_t i = (int64_t)blockIdx.x * 32 + lane;
  const bool ok = i < a.n_nodes;
  const double* st = (const double*)a.states;
  const double* pr = (const double*)a.params;
  double own = 0.0;
  if (ok)
    own = g == 0 ? a.vm[i] : st[(g - 1) * a.stride + i];
  sy[g][lane] = own;
  double P[NP], Pstim[NP];
#pragma unroll
  for (int q = 0; q < Model::nParameters; q++) {
    P[q] = ok ? pr[q * a.stride + i] : 0.0;
    Pstim[q] = (a.stimulus_mode == 1 && q == a.stimulus_parameter) ? a.stimulus_value : P[q];
  }
  const int cf = ok ? a.clamp_fiber[i] : -1;
  const SplitStep s = a.steps[a.step];
  const double t0 = a.half ? s.mid : s.t;
  const int base = (a.step * 2 + a.half) * a.nsub_stride;
  __syncthreads();
  for (int k = 0; k < s.n0; k++) {
    const double t = xadd(t0, xmul((double)k, s.dt0));
    const bool stim = cf >= 0 && stim_bit(a.flags, a.words_per_fiber, cf, base + k);
    const bool vclamp = stim && a.stimulus_mode == 0;
    double Pk[NP];
#pragma unroll
    for (int q = 0; q < NP; q++)
      Pk[q] = (stim && a.stimulus_mode == 1) ? Pstim[q] : P[q];
    double y[NS];
#pragma unroll
    for (int q = 0; q < NS; q++)
      y[q] = sy[q][lane];
    const double r = group_rate<Model, Math, 0>(g, t, y, Pk);
    double ys = own + s.dt0 * r;
    if (g == 0 && vclamp)
      ys = a.vstim;
    sys[g][lane] = ys;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NS; q++)
      y[q] = sys[q][lane];
    const double r2 = group_rate<Model, Math, 0>(g, t, y, Pk);
    own += 0.5 * s.dt0 * (r + r2);
    if (g == 0 && vclamp)
      own = a.vstim;
    sy[g][lane] = own;
    __syncthreads();
  }
  if (!ok)
    return;
  if (g == 0) {
    a.vm[i] = own;
    if (a.half == 1 && a.trace_slot) {
      const int slot = a.trace_slot[i];
      if (slot >= 0)
        record_trace(a.trace, a.n_trace, a.trace_capacity, a.act, slot, s.global_no, own);
    }
  } else {
    ((double*)a.states)[(g - 1) * a.stride + i] = own;
  }
}

// --------------------------------------------------------------------------------------------
// diffusion: coefficients of the per-fiber tridiagonal system, computed once per (dt1D, prefactor)
//   IE: (K - M/dt) u+ = -M/dt u            CN: (K/2 - M/dt) u+ = (-K/2 - M/dt) u
// following the element loops of compute.tpp:336-449, and its LU factors for
//   d'_i = mulF_i d'_{i-1} + inv_i d_i,     x_i = d'_i - cp_i x_{i+1}
// Per node the six doubles are stored as coef[k*stride + node], k = 0..5 = mulF, inv, cp, l, m, r
// with d_i = l_i u_{i-1} + m_i u_i + r_i u_{i+1}.
// --------------------------------------------------------------------------------------------
#ifdef FDM_COMMON_KERNELS_TU
__global__ void diffusion_coefficients_kernel(int n_fibers, const int64_t* __restrict__ fiber_offsets,
                                              const double* __restrict__ element_lengths,
                                              const double* __restrict__ prefactor, double dt, int implicit_euler,
                                              double* __restrict__ coef, int64_t stride)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_fibers)
    return;
  const int64_t o = fiber_offsets[f];
  const int64_t n = fiber_offsets[f + 1] - o;
  const double* h = element_lengths + (o - f); // fiber f's elements follow the previous fibers' n-1 each
  const double pf = prefactor[f];
  double cp_prev = 0.0;
  for (int64_t v = 0; v < n; v++) {
    double a = 0, b = 0, c = 0, l = 0, m = 0, r = 0;
    if (v > 0) {
      const double h_left = h[v - 1];
      const double k_left = 1. / h_left * (1) * pf;
      const double m_left = h_left * 1. / 6;
      const double k_right = 1. / h_left * (-1) * pf;
      const double m_right = h_left * 1. / 3;
      if (implicit_euler) {
        a = (k_left - 1 / dt * m_left);
        b += (k_right - 1 / dt * m_right);
        l = (-1 / dt * m_left);
        m += (-1 / dt * m_right);
      } else {
        a = (k_left / 2. - 1 / dt * m_left);
        b += (k_right / 2. - 1 / dt * m_right);
        l = (-k_left / 2. - 1 / dt * m_left);
        m += (-k_right / 2. - 1 / dt * m_right);
      }
    }
    if (v < n - 1) {
      const double h_right = h[v];
      const double k_right = 1. / h_right * (1) * pf;
      const double m_right = h_right * 1. / 6;
      const double k_left = 1. / h_right * (-1) * pf;
      const double m_left = h_right * 1. / 3;
      if (implicit_euler) {
        c = (k_right - 1 / dt * m_right);
        b += (k_left - 1 / dt * m_left);
        m += (-1 / dt * m_left);
        r = (-1 / dt * m_right);
      } else {
        c = (k_right / 2. - 1 / dt * m_right);
        b += (k_left / 2. - 1 / dt * m_left);
        m += (-k_left / 2. - 1 / dt * m_left);
        r = (-k_right / 2. - 1 / dt * m_right);
      }
    }
    double inv, mulF, cp;
    if (v == 0) {
      inv = 1.0 / b;
      mulF = 0.0;
      cp = c / b;
    } else {
      const double den = b - cp_prev * a;
      inv = 1.0 / den;
      mulF = -a * inv;
      cp = (v != n - 1) ? c / den : 0.0;
    }
    cp_prev = cp;
    const int64_t i = o + v;
    coef[0 * stride + i] = mulF;
    coef[1 * stride + i] = inv;
    coef[2 * stride + i] = cp;
    coef[3 * stride + i] = l;
    coef[4 * stride + i] = m;
    coef[5 * stride + i] = r;
  }
}

#endif // FDM_COMMON_KERNELS_TU

// affine map x -> F x + G; compose(first, second) = second o first
struct Affine {
  double F, G;
};
__device__ __forceinline__ Affine compose(const Affine& first, const Affine& second)
{
  return Affine{second.F * first.F, fma(second.F, first.G, second.G)};
}

#ifdef FDM_COMMON_KERNELS_TU
// split path: one warp per fiber; each lane owns a contiguous chunk of the fiber.
// Forward sweep results d' go to `scratch` (one double per node) for the backward sweep.
// eq_counter / eq_nbuf (or null): the equilibrium skip's per-rank count of inactive buffers and number of
// buffers; a fiber of a rank whose buffers are all counted inactive is not solved (compute.tpp:261-265)
__global__ void __launch_bounds__(128) diffusion_warp_kernel(int n_fibers, const int64_t* __restrict__ fiber_offsets,
                                                             const double* __restrict__ coef, int64_t stride,
                                                             double* __restrict__ vm, double* __restrict__ scratch,
                                                             const int* __restrict__ eq_counter,
                                                             const int* __restrict__ eq_nbuf, int n_ranks)
{
  const int lane = threadIdx.x & 31;
  const int f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (f >= n_fibers)
    return;
  if (eq_counter && eq_counter[f % n_ranks] == eq_nbuf[f % n_ranks])
    return;
  const int64_t o = fiber_offsets[f];
  const int64_t n = fiber_offsets[f + 1] - o;
  const int64_t L = (n + 31) / 32;
  const int64_t lo = o + min((int64_t)lane * L, n);
  const int64_t hi = o + min((int64_t)(lane + 1) * L, n);
  const double* mulF = coef;
  const double* inv = coef + stride;
  const double* cp = coef + 2 * stride;
  const double* cl = coef + 3 * stride;
  const double* cm = coef + 4 * stride;
  const double* cr = coef + 5 * stride;
  auto rhs = [&](int64_t i) {
    const double up = i > o ? vm[i - 1] : 0.0;
    const double un = i < o + n - 1 ? vm[i + 1] : 0.0;
    return cl[i] * up + cm[i] * vm[i] + cr[i] * un;
  };
  // forward: compose the chunk
  Affine acc{1.0, 0.0};
  for (int64_t i = lo; i < hi; i++)
    acc = compose(acc, Affine{mulF[i], inv[i] * rhs(i)});
  // inclusive warp scan, then shift to exclusive
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double F = __shfl_up_sync(0xffffffffu, acc.F, off);
    const double G = __shfl_up_sync(0xffffffffu, acc.G, off);
    if (lane >= off)
      acc = compose(Affine{F, G}, acc);
  }
  double dp = __shfl_up_sync(0xffffffffu, acc.G, 1);
  if (lane == 0)
    dp = 0.0;
  for (int64_t i = lo; i < hi; i++) {
    dp = mulF[i] * dp + inv[i] * rhs(i);
    scratch[i] = dp;
  }
  __syncwarp();
  // backward: x_i = -cp_i x_{i+1} + d'_i, composed from the chunk's end
  Affine bacc{1.0, 0.0};
  for (int64_t i = hi - 1; i >= lo; i--)
    bacc = compose(bacc, Affine{-cp[i], scratch[i]});
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double F = __shfl_down_sync(0xffffffffu, bacc.F, off);
    const double G = __shfl_down_sync(0xffffffffu, bacc.G, off);
    if (lane + off < 32)
      bacc = compose(Affine{F, G}, bacc);
  }
  double x = __shfl_down_sync(0xffffffffu, bacc.G, 1);
  if (lane == 31)
    x = 0.0;
  __syncwarp();
  for (int64_t i = hi - 1; i >= lo; i--) {
    x = -cp[i] * x + scratch[i];
    vm[i] = x;
  }
}

// Adjoint of one diffusion solve A x = B u (A, B symmetric tridiagonal): given lam (the adjoint of x) per
// fiber, mu = A^{-1} lam with the same LU factors, lam_u = B mu written back to lam, and the prefactor
// gradient  d/dpf = mu^T (dB/dpf u - dA/dpf x)  with K1 v = sum over the node's elements (v_nb - v)/h:
//   implicit Euler: A = pf K1 - M/dt, B = -M/dt          -> -mu^T K1 x
//   Crank-Nicolson: A = pf/2 K1 - M/dt, B = -pf/2 K1 - M/dt -> -mu^T K1 (u + x)/2
__global__ void __launch_bounds__(128) adjoint_diffusion_warp_kernel(
    int n_fibers, const int64_t* __restrict__ fiber_offsets, const double* __restrict__ element_lengths,
    const double* __restrict__ coef, int64_t stride, double* __restrict__ lam, const double* __restrict__ u,
    const double* __restrict__ x, int implicit_euler, double* __restrict__ grad_prefactor,
    double* __restrict__ scratch, double* __restrict__ mu)
{
  const int lane = threadIdx.x & 31;
  const int f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (f >= n_fibers)
    return;
  const int64_t o = fiber_offsets[f];
  const int64_t n = fiber_offsets[f + 1] - o;
  const int64_t L = (n + 31) / 32;
  const int64_t lo = o + min((int64_t)lane * L, n);
  const int64_t hi = o + min((int64_t)(lane + 1) * L, n);
  const double* h = element_lengths + (o - f);
  const double* mulF = coef;
  const double* inv = coef + stride;
  const double* cp = coef + 2 * stride;
  const double* cl = coef + 3 * stride;
  const double* cm = coef + 4 * stride;
  const double* cr = coef + 5 * stride;
  Affine acc{1.0, 0.0};
  for (int64_t i = lo; i < hi; i++)
    acc = compose(acc, Affine{mulF[i], inv[i] * lam[i]});
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double F = __shfl_up_sync(0xffffffffu, acc.F, off);
    const double G = __shfl_up_sync(0xffffffffu, acc.G, off);
    if (lane >= off)
      acc = compose(Affine{F, G}, acc);
  }
  double dp = __shfl_up_sync(0xffffffffu, acc.G, 1);
  if (lane == 0)
    dp = 0.0;
  for (int64_t i = lo; i < hi; i++) {
    dp = mulF[i] * dp + inv[i] * lam[i];
    scratch[i] = dp;
  }
  __syncwarp();
  Affine bacc{1.0, 0.0};
  for (int64_t i = hi - 1; i >= lo; i--)
    bacc = compose(bacc, Affine{-cp[i], scratch[i]});
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double F = __shfl_down_sync(0xffffffffu, bacc.F, off);
    const double G = __shfl_down_sync(0xffffffffu, bacc.G, off);
    if (lane + off < 32)
      bacc = compose(Affine{F, G}, bacc);
  }
  double xx = __shfl_down_sync(0xffffffffu, bacc.G, 1);
  if (lane == 31)
    xx = 0.0;
  for (int64_t i = hi - 1; i >= lo; i--) {
    xx = -cp[i] * xx + scratch[i];
    mu[i] = xx;
  }
  __syncwarp();
  // lam_u = B mu, and the prefactor gradient
  double g = 0.0;
  for (int64_t i = lo; i < hi; i++) {
    const int64_t v = i - o;
    const double mp = v > 0 ? mu[i - 1] : 0.0;
    const double mn = v < n - 1 ? mu[i + 1] : 0.0;
    const double newlam = cl[i] * mp + cm[i] * mu[i] + cr[i] * mn;
    double k1 = 0.0;
    const double w = implicit_euler ? x[i] : 0.5 * (x[i] + u[i]);
    if (v > 0)
      k1 += ((implicit_euler ? x[i - 1] : 0.5 * (x[i - 1] + u[i - 1])) - w) / h[v - 1];
    if (v < n - 1)
      k1 += ((implicit_euler ? x[i + 1] : 0.5 * (x[i + 1] + u[i + 1])) - w) / h[v];
    g -= mu[i] * k1;
    scratch[i] = newlam;
  }
  __syncwarp();
  for (int64_t i = lo; i < hi; i++)
    lam[i] = scratch[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    g += __shfl_down_sync(0xffffffffu, g, off);
  if (lane == 0)
    grad_prefactor[f] += g;
}

#endif // FDM_COMMON_KERNELS_TU

// --------------------------------------------------------------------------------------------
// adjoint (discrete reverse mode of the FP64 split path)
// --------------------------------------------------------------------------------------------
struct AdjointArgs {
  int64_t n_nodes;
  const double* states;           // stored substep input states of this half step: [(k*nS + s)*N + node]
  const double* params;           // [p][node]
  double* lam;                    // adjoint of the state [s][node], in/out
  double* grad_params;            // [p][node], accumulated
  const int* clamp_fiber;
  const uint32_t* flags;
  int words_per_fiber;
  int nsub_stride;
  double vstim;
  int stimulus_mode;
  int stimulus_parameter;
  double stimulus_value;
  SplitStep step;
  int step_in_window;             // index of the split step in the flags window
  int half;
  const int* trace_slot;          // sensors: adjoint of the recorded Vm is added before half 1 is reversed
  const double* trace_grad;       // [step][slot]
  int n_trace;
  int64_t trace_row;              // row of trace_grad for this split step (or -1)
  int use_tape;                   // 1: f(y) evaluated once, its temporaries kept for the backward sweep
  const int* gate;                // onlyComputeIfHasBeenStimulated: skipped substeps are the identity
  const uint8_t* gate_start;
  int gate_stride;
};

// The right-hand side forms the adjoint uses: with exact exponentials the generated fast form
// (shared exponentials, one reciprocal per division; values equal to the plain form's to a few
// ulps, which moves the linearization point by that much), else the plain form.
template<class Model, class Math, bool FAST = std::is_same<Math, fdm_math_exact>::value>
struct AdjointForms {
  static constexpr int nTape = Model::nTape;
  __device__ __forceinline__ static void tape(double t, const double* y, const double* P, double* r, double* tp)
  {
    Model::template rates_tape<double, Math>(t, y, P, r, tp);
  }
  __device__ __forceinline__ static void vjp(double t, const double* y, const double* P, const double* lr, double* ly,
                                             double* lp)
  {
    Model::template rates_vjp<double, Math>(t, y, P, lr, ly, lp);
  }
  __device__ __forceinline__ static void vjp_tape(double t, const double* y, const double* P, const double* tp,
                                                  const double* lr, double* ly, double* lp)
  {
    Model::template rates_vjp_tape<double, Math>(t, y, P, tp, lr, ly, lp);
  }
};
template<class Model, class Math>
struct AdjointForms<Model, Math, true> {
  static constexpr int nTape = Model::nTapeFast;
  __device__ __forceinline__ static void tape(double t, const double* y, const double* P, double* r, double* tp)
  {
    Model::template rates_tape_fast<double, Math>(t, y, P, r, tp);
  }
  __device__ __forceinline__ static void vjp(double t, const double* y, const double* P, const double* lr, double* ly,
                                             double* lp)
  {
    Model::template rates_vjp_fast<double, Math>(t, y, P, lr, ly, lp);
  }
  __device__ __forceinline__ static void vjp_tape(double t, const double* y, const double* P, const double* tp,
                                                  const double* lr, double* ly, double* lp)
  {
    Model::template rates_vjp_tape_fast<double, Math>(t, y, P, tp, lr, ly, lp);
  }
};

// reverse of one half step (n0 Heun substeps) for one node:
//   forward  r = f(y); y* = y + dt r [y*_0 := vStim]; y' = y + dt/2 (r + f(y*)) [y'_0 := vStim]
//   reverse  (clamp: lam'_0 := 0); lam_* = J(y*)^T dt/2 lam' (clamp: lam_*_0 := 0);
//            lam_y = lam' + lam_* + J(y)^T (dt/2 lam' + dt lam_*)
// The stored input state of the next substep in reverse order is loaded while the current one is
// differentiated (models with at most 8 states).
template<class Model, class Math>
__global__ void __launch_bounds__(128, 3) adjoint_half_kernel(AdjointArgs a)
{
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_nodes)
    return;
  using F = AdjointForms<Model, Math>;
  constexpr int NS = Model::nStates;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  constexpr bool PREFETCH = NS <= 8;
  const int64_t N = a.n_nodes;
  double lam[NS], P[NP], gP[NP];
#pragma unroll
  for (int s = 0; s < NS; s++)
    lam[s] = a.lam[s * N + i];
#pragma unroll
  for (int q = 0; q < Model::nParameters; q++) {
    P[q] = a.params[q * N + i];
    gP[q] = 0.0;
  }
  if (a.half == 1 && a.trace_slot && a.trace_row >= 0) {
    const int slot = a.trace_slot[i];
    if (slot >= 0)
      lam[0] += a.trace_grad[a.trace_row * a.n_trace + slot];
  }
  const int cf = a.clamp_fiber[i];
  const SplitStep st = a.step;
  const double t0 = a.half ? st.mid : st.t;
  const int base = (a.step_in_window * 2 + a.half) * a.nsub_stride;
  const double dt = st.dt0;
  const int first = a.gate ? gate_first(a.gate_start, a.gate_stride, a.gate[i], a.step_in_window * 2 + a.half) : 0;
  double ynext[PREFETCH ? NS : 1];
  if (PREFETCH && st.n0 > 0) {
#pragma unroll
    for (int s = 0; s < NS; s++)
      ynext[s] = a.states[(int64_t)((st.n0 - 1) * NS + s) * N + i];
  }
  for (int k = st.n0 - 1; k >= 0; k--) {
    const double t = xadd(t0, xmul((double)k, dt));
    const bool stim = cf >= 0 && stim_bit(a.flags, a.words_per_fiber, cf, base + k);
    const bool clamp = stim && a.stimulus_mode == 0;
    double Pk[NP];
#pragma unroll
    for (int q = 0; q < NP; q++)
      Pk[q] = (stim && a.stimulus_mode == 1 && q == a.stimulus_parameter) ? a.stimulus_value : P[q];
    double y[NS], r[NS], ys[NS];
    if (PREFETCH) {
#pragma unroll
      for (int s = 0; s < NS; s++)
        y[s] = ynext[s];
      if (k > 0) {
#pragma unroll
        for (int s = 0; s < NS; s++)
          ynext[s] = a.states[(int64_t)((k - 1) * NS + s) * N + i];
      }
    } else {
#pragma unroll
      for (int s = 0; s < NS; s++)
        y[s] = a.states[(int64_t)(k * NS + s) * N + i];
    }
    if (k < first)
      continue; // the forward substep was skipped: its reverse is the identity
    constexpr bool TAPE_OK = F::nTape <= 256;
    double tape[TAPE_OK ? F::nTape : 1];
    if (TAPE_OK && a.use_tape) {
      F::tape(t, y, Pk, r, tape);
    } else {
      double alg[Model::nAlgebraics];
      Model::template rates<double, Math>(t, y, Pk, r, alg);
    }
#pragma unroll
    for (int s = 0; s < NS; s++)
      ys[s] = y[s] + dt * r[s];
    if (clamp) {
      ys[0] = a.vstim;
      lam[0] = 0.0;
    }
    double lr2[NS], lys[NS], lr[NS], gPk[NP];
#pragma unroll
    for (int s = 0; s < NS; s++) {
      lr2[s] = 0.5 * dt * lam[s];
      lys[s] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < NP; q++)
      gPk[q] = 0.0;
    F::vjp(t, ys, Pk, lr2, lys, gPk);
    if (clamp)
      lys[0] = 0.0;
#pragma unroll
    for (int s = 0; s < NS; s++) {
      lr[s] = 0.5 * dt * lam[s] + dt * lys[s];
      lam[s] = lam[s] + lys[s];
    }
    if (TAPE_OK && a.use_tape)
      F::vjp_tape(t, y, Pk, tape, lr, lam, gPk);
    else
      F::vjp(t, y, Pk, lr, lam, gPk);
#pragma unroll
    for (int q = 0; q < Model::nParameters; q++)
      if (!(stim && a.stimulus_mode == 1 && q == a.stimulus_parameter))
        gP[q] += gPk[q];
  }
#pragma unroll
  for (int s = 0; s < NS; s++)
    a.lam[s * N + i] = lam[s];
#pragma unroll
  for (int q = 0; q < Model::nParameters; q++)
    a.grad_params[q * N + i] += gP[q];
}

// --------------------------------------------------------------------------------------------
// fused path
// --------------------------------------------------------------------------------------------
constexpr int FUSED_MAX_FIBERS_PER_BIN = 32;

struct FusedArgs {
  int n_bins;
  const int* bin_fiber_start;     // [n_bins+1] range in bin_fibers
  const int* bin_fibers;          // fiber numbers, bin after bin (at most FUSED_MAX_FIBERS_PER_BIN per bin)
  const int64_t* fiber_offsets;   // node offsets of the fibers
  int64_t stride;
  double* vm;
  void* states;                   // RR SoA
  void* states_lo;                // FP32 only: compensation terms
  const void* params;             // RR SoA
  const double* coef;             // 6 x stride
  const int* clamp_fiber;
  const uint32_t* flags;
  int words_per_fiber;
  int nsub_stride;
  double vstim;
  int stimulus_mode;
  int stimulus_parameter;
  double stimulus_value;
  const SplitStep* steps;
  int n_steps;
  int store_alg;
  int n_alg_out;
  const int* alg_indices;
  double* alg_out;
  int64_t n_nodes;
  const int* trace_slot;
  double* trace;
  int n_trace;
  int64_t trace_capacity;
  ActivationRec act;
  const int* gate;                // onlyComputeIfHasBeenStimulated: per node gate code, or null
  const uint8_t* gate_start;
  int gate_stride;
};

// Block-wide exclusive scan of affine maps in thread order (REVERSE: from the last thread down): returns the
// composition of the maps of the threads before this one in scan order, and in *total (if given) the
// composition of all threads' maps.  A Hillis-Steele scan within each warp; the warp totals go to sF/sG[0, T/32)
// and, after the one barrier, every warp scans the totals itself (rather than one warp scanning them and
// broadcasting the prefixes through a second barrier).  sF/sG hold T/32 doubles each; a caller that scans again
// without a barrier in between must give the next scan other slots (warps may still read these totals when a
// fast warp writes the next ones).
template<int T, bool REVERSE>
__device__ __forceinline__ Affine block_scan_map(Affine acc, double* sF, double* sG, Affine* total)
{
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  constexpr int NW = T / 32;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    double F, G;
    if (!REVERSE) {
      F = __shfl_up_sync(0xffffffffu, acc.F, off);
      G = __shfl_up_sync(0xffffffffu, acc.G, off);
      if (lane >= off)
        acc = compose(Affine{F, G}, acc);
    } else {
      F = __shfl_down_sync(0xffffffffu, acc.F, off);
      G = __shfl_down_sync(0xffffffffu, acc.G, off);
      if (lane + off < 32)
        acc = compose(Affine{F, G}, acc);
    }
  }
  const int last_lane = REVERSE ? 0 : 31;
  if (lane == last_lane) {
    sF[warp] = acc.F;
    sG[warp] = acc.G;
  }
  double exF = REVERSE ? __shfl_down_sync(0xffffffffu, acc.F, 1) : __shfl_up_sync(0xffffffffu, acc.F, 1);
  double exG = REVERSE ? __shfl_down_sync(0xffffffffu, acc.G, 1) : __shfl_up_sync(0xffffffffu, acc.G, 1);
  const bool first_in_warp = REVERSE ? (lane == 31) : (lane == 0);
  if (first_in_warp) {
    exF = 1.0;
    exG = 0.0;
  }
  __syncthreads();
  // lane k holds the total of the k-th warp in scan order; inclusive scan over the lanes
  const int w = REVERSE ? (NW - 1 - lane) : lane;
  Affine v = lane < NW ? Affine{sF[w], sG[w]} : Affine{1.0, 0.0};
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double F = __shfl_up_sync(0xffffffffu, v.F, off);
    const double G = __shfl_up_sync(0xffffffffu, v.G, off);
    if (lane >= off)
      v = compose(Affine{F, G}, v);
  }
  // this warp's position in scan order; its exclusive prefix is the inclusive scan of the position before
  const int pos = REVERSE ? (NW - 1 - warp) : warp;
  const double pF = __shfl_sync(0xffffffffu, v.F, pos > 0 ? pos - 1 : 0);
  const double pG = __shfl_sync(0xffffffffu, v.G, pos > 0 ? pos - 1 : 0);
  const Affine wp = pos > 0 ? Affine{pF, pG} : Affine{1.0, 0.0};
  if (total) {
    total->F = __shfl_sync(0xffffffffu, v.F, NW - 1);
    total->G = __shfl_sync(0xffffffffu, v.G, NW - 1);
  }
  return compose(wp, Affine{exF, exG});
}

// the value entering this thread's first node: the exclusive prefix map applied to the zero entering the
// first node of the scan
template<int T, bool REVERSE>
__device__ __forceinline__ double block_scan_incoming(Affine acc, double* sF, double* sG)
{
  return block_scan_map<T, REVERSE>(acc, sF, sG, nullptr).G;
}

// Split path, few fibers: one diffusion solve per fiber with one CTA per fiber (a warp per fiber would leave
// most of the GPU idle).  Thread tid owns a contiguous chunk of the fiber; the forward sweep and the back
// substitution are block-wide scans of affine maps as in the fused kernel.  Same arguments and equilibrium
// skip as diffusion_warp_kernel (forward results d' in scratch).
template<int T>
__global__ void __launch_bounds__(T) diffusion_block_kernel(const int64_t* __restrict__ fiber_offsets,
                                                            const double* __restrict__ coef, int64_t stride,
                                                            double* __restrict__ vm, double* __restrict__ scratch,
                                                            const int* __restrict__ eq_counter,
                                                            const int* __restrict__ eq_nbuf, int n_ranks)
{
  __shared__ double sF[T / 32], sG[T / 32]; // warp totals (both scans: the barrier between them orders the reuse)
  const int f = blockIdx.x;
  const int tid = threadIdx.x;
  if (eq_counter && eq_counter[f % n_ranks] == eq_nbuf[f % n_ranks])
    return; // the whole CTA: the rank's buffers are all inactive
  const int64_t o = fiber_offsets[f];
  const int64_t n = fiber_offsets[f + 1] - o;
  const int64_t L = (n + T - 1) / T;
  const int64_t lo = o + min((int64_t)tid * L, n);
  const int64_t hi = o + min((int64_t)(tid + 1) * L, n);
  const double* mulF = coef;
  const double* inv = coef + stride;
  const double* cp = coef + 2 * stride;
  const double* cl = coef + 3 * stride;
  const double* cm = coef + 4 * stride;
  const double* cr = coef + 5 * stride;
  auto rhs = [&](int64_t i) {
    const double up = i > o ? vm[i - 1] : 0.0;
    const double un = i < o + n - 1 ? vm[i + 1] : 0.0;
    return cl[i] * up + cm[i] * vm[i] + cr[i] * un;
  };
  Affine acc{1.0, 0.0};
  for (int64_t i = lo; i < hi; i++)
    acc = compose(acc, Affine{mulF[i], inv[i] * rhs(i)});
  double dp = block_scan_incoming<T, false>(acc, sF, sG);
  for (int64_t i = lo; i < hi; i++) {
    dp = mulF[i] * dp + inv[i] * rhs(i);
    scratch[i] = dp;
  }
  __syncthreads(); // every read of the old Vm done, scratch complete, sF/sG free
  Affine bacc{1.0, 0.0};
  for (int64_t i = hi - 1; i >= lo; i--)
    bacc = compose(bacc, Affine{-cp[i], scratch[i]});
  double x = block_scan_incoming<T, true>(bacc, sF, sG);
  for (int64_t i = hi - 1; i >= lo; i--) {
    x = -cp[i] * x + scratch[i];
    vm[i] = x;
  }
}

// Adjoint of one diffusion solve (see adjoint_diffusion_warp_kernel for the algebra) with one CTA per
// fiber of at most T*M nodes: thread tid owns nodes tid*M .. tid*M+M-1 in registers, the two sweeps of the
// LU solve are block-wide scans of affine maps (as in the fused kernel), neighbours across threads go
// through shared memory, and the prefactor gradient is a block reduction.  Used when the fibers are few
// (a warp per fiber would leave most of the GPU idle).
template<int T, int M>
__global__ void __launch_bounds__(T) adjoint_diffusion_block_kernel(
    const int64_t* __restrict__ fiber_offsets, const double* __restrict__ element_lengths,
    const double* __restrict__ coef, int64_t stride, double* __restrict__ lam, const double* __restrict__ u,
    const double* __restrict__ x, int implicit_euler, double* __restrict__ grad_prefactor)
{
  __shared__ double sF[2 * (T / 32)], sG[2 * (T / 32)]; // warp totals: forward, backward
  __shared__ double sfirst[T], slast[T], swfirst[T], swlast[T], sred[T / 32];
  const int f = blockIdx.x;
  const int tid = threadIdx.x;
  const int64_t o = fiber_offsets[f];
  const int n = (int)(fiber_offsets[f + 1] - o);
  const double* h = element_lengths + (o - f);
  const double* mulF = coef;
  const double* inv = coef + stride;
  const double* cp = coef + 2 * stride;
  const double* cl = coef + 3 * stride;
  const double* cm = coef + 4 * stride;
  const double* cr = coef + 5 * stride;
  double d[M], mu[M], w[M];
  // forward sweep of A^{-1} lam
  Affine acc{1.0, 0.0};
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int q = tid * M + j;
    if (q < n) {
      d[j] = inv[o + q] * lam[o + q];
      acc = compose(acc, Affine{mulF[o + q], d[j]});
    } else {
      d[j] = 0.0;
    }
  }
  // forward and backward scans with one barrier each, their warp totals in the two halves of sF/sG
  double dp = block_scan_incoming<T, false>(acc, sF, sG);
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int q = tid * M + j;
    if (q < n) {
      dp = mulF[o + q] * dp + d[j];
      d[j] = dp;
    }
  }
  // backward sweep (nodes beyond the fiber carry x = 0 into its last node)
  Affine bacc{1.0, 0.0};
#pragma unroll
  for (int j = M - 1; j >= 0; j--) {
    const int q = tid * M + j;
    bacc = compose(bacc, q < n ? Affine{-cp[o + q], d[j]} : Affine{0.0, 0.0});
  }
  double xx = block_scan_incoming<T, true>(bacc, sF + T / 32, sG + T / 32);
#pragma unroll
  for (int j = M - 1; j >= 0; j--) {
    const int q = tid * M + j;
    xx = q < n ? -cp[o + q] * xx + d[j] : 0.0;
    mu[j] = xx;
    w[j] = q < n ? (implicit_euler ? x[o + q] : 0.5 * (x[o + q] + u[o + q])) : 0.0;
  }
  // neighbours of the thread's first and last node: mu and w, exchanged together
  sfirst[tid] = mu[0];
  slast[tid] = mu[M - 1];
  swfirst[tid] = w[0];
  swlast[tid] = w[M - 1];
  __syncthreads();
  const double mu_prev = tid > 0 ? slast[tid - 1] : 0.0;
  const double mu_next = tid < T - 1 ? sfirst[tid + 1] : 0.0;
  const double w_prev = tid > 0 ? swlast[tid - 1] : 0.0;
  const double w_next = tid < T - 1 ? swfirst[tid + 1] : 0.0;
  // lam_u = B mu and the prefactor gradient -mu^T K1 w
  double g = 0.0;
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int q = tid * M + j;
    if (q >= n)
      continue;
    const double mp = q > 0 ? (j > 0 ? mu[j - 1] : mu_prev) : 0.0;
    const double mn = q < n - 1 ? (j < M - 1 ? mu[j + 1] : mu_next) : 0.0;
    lam[o + q] = cl[o + q] * mp + cm[o + q] * mu[j] + cr[o + q] * mn;
    double k1 = 0.0;
    if (q > 0)
      k1 += ((j > 0 ? w[j - 1] : w_prev) - w[j]) / h[q - 1];
    if (q < n - 1)
      k1 += ((j < M - 1 ? w[j + 1] : w_next) - w[j]) / h[q];
    g -= mu[j] * k1;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    g += __shfl_down_sync(0xffffffffu, g, off);
  if ((tid & 31) == 0)
    sred[tid >> 5] = g;
  __syncthreads();
  if (tid == 0) {
    double sum = 0.0;
    for (int k = 0; k < T / 32; k++)
      sum += sred[k];
    grad_prefactor[f] += sum;
  }
}

// GATE: onlyComputeIfHasBeenStimulated is on (a.gate is set); a separate instantiation so that the
// default path carries none of its per-substep checks.
// CLUSTER: for few fibers (the GPU would be mostly idle with one CTA per bin), one fiber per thread-block
// cluster: CTA r of the cluster holds the fiber's nodes [r * T*M, (r+1) * T*M); the CTAs exchange the Vm of
// their edge nodes and the totals of their scans through distributed shared memory, with three cluster
// barriers per Strang step (every CTA of a cluster takes every barrier: no CTA returns early).
template<class Model, class RR, class Math, int T, int M, bool GATE, bool CLUSTER>
__global__ void __launch_bounds__(T, 1) fused_kernel(FusedArgs a)
{
  constexpr int NS = Model::nStates;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  constexpr int CAP = T * M;
  extern __shared__ double smem[];
  // 5 x CAP coefficients: mulF, cp, and the right-hand side stencil l, m, r premultiplied by inv
  double* sc = smem;
  double* vfirst = sc + 5 * CAP;     // T
  double* vlast = vfirst + T;        // T
  double* sF = vlast + T;            // 2 * (T/32) + 1
  double* sG = sF + 2 * (T / 32) + 1; // 2 * (T/32) + 1
  int* s_cf = (int*)(sG + 2 * (T / 32) + 1); // CAP: clamp fiber of each node (-1: not a junction node)
  int* s_ts = s_cf + CAP;                // CAP: trace slot of each node (-1: not traced)
  int* s_gate = s_ts + CAP;              // CAP: gate code of each node (onlyComputeIfHasBeenStimulated)
  // paired FP32 path: the parameters of node pair p of thread tid, parameter k, at (p * NP + k) * T + tid
  fdm_f2* sP2 = (fdm_f2*)(s_gate + CAP);
  __shared__ int64_t fib_global[FUSED_MAX_FIBERS_PER_BIN];
  __shared__ int fib_local[FUSED_MAX_FIBERS_PER_BIN + 1];

  __shared__ double ctot[4];      // cluster mode: this CTA's forward and backward scan totals (F, G)
  __shared__ double cpre[2 * 16]; // cluster mode: the other CTAs' totals this CTA composes
  const int tid = threadIdx.x;
  int bin = blockIdx.x, crank = 0, csize = 1;
  if constexpr (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    crank = (int)cl.block_rank();
    csize = (int)cl.num_blocks();
    bin = blockIdx.x / csize;
  } else {
    if (bin >= a.n_bins)
      return;
  }
  // the bin's fibers, concatenated in bin-local node numbering (cluster mode: this CTA's part of one fiber)
  const int f0 = a.bin_fiber_start[bin];
  const int nf = CLUSTER ? 1 : a.bin_fiber_start[bin + 1] - f0;
  if (tid == 0) {
    if (CLUSTER) {
      const int fib = a.bin_fibers[f0];
      const int64_t len = a.fiber_offsets[fib + 1] - a.fiber_offsets[fib];
      const int64_t lo = (int64_t)crank * CAP;
      fib_global[0] = a.fiber_offsets[fib] + lo;
      fib_local[0] = 0;
      fib_local[1] = (int)max((int64_t)0, min((int64_t)CAP, len - lo));
    } else {
      int loc = 0;
      for (int k = 0; k < nf; k++) {
        const int fib = a.bin_fibers[f0 + k];
        fib_global[k] = a.fiber_offsets[fib];
        fib_local[k] = loc;
        loc += (int)(a.fiber_offsets[fib + 1] - a.fiber_offsets[fib]);
      }
      fib_local[nf] = loc;
    }
  }
  __syncthreads();
  // cluster mode: barrier over the cluster's CTAs (and of this CTA's threads)
  auto cluster_sync = [&]() {
    if constexpr (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
  };
  // cluster mode: the value entering this thread's first node of a sweep, from the CTA's own scan (ex, total)
  // and the totals of the CTAs before it in sweep order
  auto cluster_incoming = [&](Affine ex, Affine total, bool reverse) -> double {
    if constexpr (!CLUSTER) {
      (void)total;
      (void)reverse;
      return ex.G;
    } else {
      cg::cluster_group cl = cg::this_cluster();
      const int slot = reverse ? 2 : 0;
      if (tid == 0) {
        ctot[slot] = total.F;
        ctot[slot + 1] = total.G;
      }
      cl.sync();
      // thread k < csize fetches CTA k's total (the ranks before this one in sweep order are used)
      if (tid < csize) {
        const double* remote = cl.map_shared_rank(ctot, tid);
        cpre[2 * tid] = remote[slot];
        cpre[2 * tid + 1] = remote[slot + 1];
      }
      __syncthreads();
      Affine pre{1.0, 0.0};
      if (!reverse) {
        for (int k = 0; k < crank; k++)
          pre = compose(pre, Affine{cpre[2 * k], cpre[2 * k + 1]});
      } else {
        for (int k = csize - 1; k > crank; k--)
          pre = compose(pre, Affine{cpre[2 * k], cpre[2 * k + 1]});
      }
      return compose(pre, ex).G;
    }
  };
  const int nb = fib_local[nf];
  auto global_node = [&](int q) -> int64_t {
    int k = 0;
    while (k + 1 < nf && q >= fib_local[k + 1])
      k++;
    return fib_global[k] + (q - fib_local[k]);
  };

  // coefficients into shared memory (zero beyond the bin: those nodes carry x = 0); the forward sweep's
  // inv * d is formed as (inv l) u_{i-1} + (inv m) u_i + (inv r) u_{i+1}.  The per-node shared arrays hold
  // node j of thread t (bin node t * M + j) at slot j * T + t: a warp's accesses to one j are consecutive
  // words, free of bank conflicts
  for (int sl = tid; sl < CAP; sl += T) {
    const int q = (sl % T) * M + sl / T;
    const bool ok = q < nb;
    const int64_t g = ok ? global_node(q) : 0;
    const double inv = ok ? a.coef[1 * a.stride + g] : 0.0;
    sc[0 * CAP + sl] = ok ? a.coef[0 * a.stride + g] : 0.0;
    sc[1 * CAP + sl] = ok ? a.coef[2 * a.stride + g] : 0.0;
#pragma unroll
    for (int k = 3; k < 6; k++)
      sc[(k - 1) * CAP + sl] = ok ? inv * a.coef[k * a.stride + g] : 0.0;
  }

  const RR* pr = (const RR*)a.params;
  RR* st = (RR*)a.states;
  RR* stl = (RR*)a.states_lo;
  double V[M];
  RR S[M][NS > 1 ? NS - 1 : 1];
  RR L[M][NS > 1 ? NS - 1 : 1];
  RR P[M][NP];
  unsigned cmask = 0u; // bit j: node j is a junction node (its clamp fiber in s_cf)
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int q = tid * M + j;
    const bool ok = q < nb;
    const int64_t i = ok ? global_node(q) : 0;
    V[j] = ok ? a.vm[i] : 0.0;
#pragma unroll
    for (int s = 1; s < NS; s++) {
      S[j][s - 1] = ok ? st[(s - 1) * a.stride + i] : (RR)0;
      L[j][s - 1] = (ok && Compensated<RR>::value) ? stl[(s - 1) * a.stride + i] : (RR)0;
    }
#pragma unroll
    for (int p = 0; p < Model::nParameters; p++)
      P[j][p] = ok ? pr[p * a.stride + i] : (RR)0;
    const int cfj = ok ? a.clamp_fiber[i] : -1;
    s_cf[j * T + tid] = cfj;
    cmask |= (cfj >= 0 ? 1u : 0u) << j;
    s_ts[j * T + tid] = (ok && a.trace_slot) ? a.trace_slot[i] : -1;
    s_gate[j * T + tid] = (ok && a.gate) ? a.gate[i] : 0;
  }
  // the clamp fiber of the thread's junction nodes when they all belong to one fiber (the usual case: a
  // junction is a few consecutive nodes of one fiber): one flag read per substep instead of one per node
  int cf_first = -1;
  bool cf_one = true;
#pragma unroll
  for (int j = 0; j < M; j++) {
    if ((cmask >> j) & 1u) {
      const int c = s_cf[j * T + tid];
      cf_one = cf_one && (cf_first < 0 || c == cf_first);
      cf_first = cf_first < 0 ? c : cf_first;
    }
  }
  // stimulation bit of node j at substep bit `bit` (junction nodes only read their fiber's bit)
  auto node_stim = [&](int j, int bit) -> bool {
    return ((cmask >> j) & 1u) && stim_bit(a.flags, a.words_per_fiber, s_cf[j * T + tid], bit);
  };
  // FP32 exact-exponential reaction: nodes (2p, 2p+1) advance together in packed FP32 (heun_step2);
  // an odd last node runs alone
  constexpr bool PAIR = std::is_same<RR, float>::value && std::is_same<Math, fdm_math_exact>::value;
  constexpr int MP = PAIR ? M / 2 : 0;
  constexpr unsigned pair_mask = (1u << (2 * MP)) - 1u; // the paired nodes' bits
  constexpr int NSM = NS > 1 ? NS - 1 : 1;
  fdm_f2 S2[MP > 0 ? MP : 1][NSM], L2[MP > 0 ? MP : 1][NSM];
  if constexpr (PAIR) {
#pragma unroll
    for (int p = 0; p < MP; p++) {
#pragma unroll
      for (int s = 0; s < NSM; s++) {
        S2[p][s] = fdm_f2((float)S[2 * p][s], (float)S[2 * p + 1][s]);
        L2[p][s] = fdm_f2((float)L[2 * p][s], (float)L[2 * p + 1][s]);
      }
#pragma unroll
      for (int q = 0; q < NP; q++)
        sP2[(p * NP + q) * T + tid] = fdm_f2((float)P[2 * p][q], (float)P[2 * p + 1][q]);
    }
  }
  // the scalar state of node j (from the pair arrays where node j is paired)
  auto unpack = [&](int j, RR* Sj, RR* Lj, RR* Pj) {
#pragma unroll
    for (int s = 0; s < NSM; s++) {
      Sj[s] = S[j][s];
      Lj[s] = L[j][s];
    }
#pragma unroll
    for (int q = 0; q < NP; q++)
      Pj[q] = P[j][q];
    if constexpr (PAIR) {
      if (j < 2 * MP) {
#pragma unroll
        for (int s = 0; s < NSM; s++) {
          Sj[s] = (RR)((j & 1) ? S2[j >> 1][s].v.y : S2[j >> 1][s].v.x);
          Lj[s] = (RR)((j & 1) ? L2[j >> 1][s].v.y : L2[j >> 1][s].v.x);
        }
#pragma unroll
        for (int q = 0; q < NP; q++)
          Pj[q] = (RR)((j & 1) ? sP2[((j >> 1) * NP + q) * T + tid].v.y : sP2[((j >> 1) * NP + q) * T + tid].v.x);
      }
    }
  };
  auto repack = [&](int j, const RR* Sj, const RR* Lj) {
#pragma unroll
    for (int s = 0; s < NSM; s++) {
      S[j][s] = Sj[s];
      L[j][s] = Lj[s];
    }
    if constexpr (PAIR) {
      if (j < 2 * MP) {
#pragma unroll
        for (int s = 0; s < NSM; s++) {
          if (j & 1) {
            S2[j >> 1][s].v.y = (float)Sj[s];
            L2[j >> 1][s].v.y = (float)Lj[s];
          } else {
            S2[j >> 1][s].v.x = (float)Sj[s];
            L2[j >> 1][s].v.x = (float)Lj[s];
          }
        }
      }
    }
  };
  // one Heun substep of a node that runs alone
  auto scalar_node = [&](int j, double t, double dt0, int bit) {
    const bool stim = node_stim(j, bit);
    if (stim && a.stimulus_mode == 1) {
      // stimulus current: the junction nodes see the stimulus parameter while stimulated
      RR Pk[NP];
#pragma unroll
      for (int p = 0; p < NP; p++)
        Pk[p] = p == a.stimulus_parameter ? (RR)a.stimulus_value : P[j][p];
      heun_step<Model, RR, Math, false>(V[j], S[j], L[j], Pk, t, dt0, false, a.vstim, nullptr);
    } else {
      heun_step<Model, RR, Math, false>(V[j], S[j], L[j], P[j], t, dt0, stim, a.vstim, nullptr);
    }
  };
  __syncthreads();

  for (int step = 0; step < a.n_steps; step++) {
    const SplitStep s = a.steps[step];
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
      const double t0 = half ? s.mid : s.t;
      const int base = (step * 2 + half) * a.nsub_stride;
      // the substep after which algebraicsForTransfer are stored runs outside the hot loop
      const bool store_here = a.store_alg && half == 1 && step == a.n_steps - 1;
      const int k_end = store_here ? s.n0 - 1 : s.n0;
      // onlyComputeIfHasBeenStimulated: each node's first computed substep of this half step, 8 bits each
      constexpr bool gate_on = GATE;
      unsigned gfirst[(M + 3) / 4];
#pragma unroll
      for (int w = 0; w < (M + 3) / 4; w++)
        gfirst[w] = 0u;
      if constexpr (gate_on) {
#pragma unroll
        for (int j = 0; j < M; j++)
          gfirst[j >> 2] |= (unsigned)gate_first(a.gate_start, a.gate_stride, s_gate[j * T + tid], step * 2 + half)
                            << (8 * (j & 3));
      }
      auto node_on = [&](int j, int k) -> bool { return k >= (int)((gfirst[j >> 2] >> (8 * (j & 3))) & 0xffu); };
      // paired nodes: Vm in FP32 over the half step (value at its start + the sum of the increments since)
      fdm_f2 Vf[MP > 0 ? MP : 1], LV[MP > 0 ? MP : 1];
      if constexpr (PAIR) {
#pragma unroll
        for (int p = 0; p < MP; p++) {
          Vf[p] = fdm_f2((float)V[2 * p], (float)V[2 * p + 1]);
          LV[p] = fdm_f2(0.f, 0.f);
        }
      }
#pragma unroll 1
      for (int k = 0; k < k_end; k++) {
        const double t = xadd(t0, xmul((double)k, s.dt0));
        if constexpr (gate_on) {
          // a substep that no node of the warp computes is skipped by the whole warp
          bool any = false;
#pragma unroll
          for (int j = 0; j < M; j++)
            any = any || (tid * M + j < nb && node_on(j, k));
          if (!__any_sync(0xffffffffu, any))
            continue;
        }
        if constexpr (PAIR && !gate_on && MP > 0) {
          // all pairs in one block (nodes beyond the bin compute too; their Vm is zeroed after the half step).
          // Stimulated junction nodes are rare (a few substeps per firing): the clamp and the stimulus
          // parameter are applied in a second copy of the step that a warp takes only when one of its nodes
          // is stimulated, so the common step carries no selects and no per-node flag reads
          const float dtf = (float)s.dt0;
          unsigned clamp = 0u; // bit j: node j stimulated in this substep
          if (cmask) {
            if (cf_one) {
              clamp = stim_bit(a.flags, a.words_per_fiber, cf_first, base + k) ? cmask : 0u;
            } else {
#pragma unroll
              for (int j = 0; j < 2 * MP; j++)
                clamp |= (node_stim(j, base + k) ? 1u : 0u) << j;
            }
          }
          fdm_f2 Pk[MP > 0 ? MP : 1][NP];
#pragma unroll
          for (int p = 0; p < MP; p++)
#pragma unroll
            for (int q = 0; q < NP; q++)
              Pk[p][q] = sP2[(p * NP + q) * T + tid];
          if (__any_sync(0xffffffffu, (clamp & pair_mask) != 0u)) {
            const bool m1 = a.stimulus_mode == 1;
            const float sv = (float)a.stimulus_value;
#pragma unroll
            for (int p = 0; p < MP; p++)
#pragma unroll
              for (int q = 0; q < NP; q++) {
                const bool hit = m1 && q == a.stimulus_parameter;
                Pk[p][q] = fdm_f2((hit && ((clamp >> (2 * p)) & 1u)) ? sv : Pk[p][q].v.x,
                                  (hit && ((clamp >> (2 * p + 1)) & 1u)) ? sv : Pk[p][q].v.y);
              }
            heun_step2_pairs<Model, MP, NSM, NP>(Vf, LV, V, S2, L2, Pk, fdm_f2((float)t), fdm_f2(dtf),
                                                 fdm_f2(0.5f * dtf), m1 ? 0u : (clamp & pair_mask), a.vstim);
          } else {
            heun_step2_pairs<Model, MP, NSM, NP>(Vf, LV, V, S2, L2, Pk, fdm_f2((float)t), fdm_f2(dtf),
                                                 fdm_f2(0.5f * dtf), 0u, a.vstim);
          }
          if constexpr (M % 2 == 1) {
            if (tid * M + M - 1 < nb)
              scalar_node(M - 1, t, s.dt0, base + k);
          }
        } else if constexpr (PAIR) {
          const float dtf = (float)s.dt0;
          const fdm_f2 dt_all(dtf), hdt_all(0.5f * dtf);
#pragma unroll
          for (int p = 0; p < MP; p++) {
            const int j0 = 2 * p;
            if (tid * M + j0 >= nb)
              continue;
            // a node that does not compute this substep gets step width 0 (its state stays as it is)
            fdm_f2 dtr = dt_all, hdt = hdt_all;
            if constexpr (gate_on) {
              const bool c0 = node_on(j0, k), c1 = node_on(j0 + 1, k);
              if (!c0 && !c1)
                continue;
              dtr = fdm_f2(c0 ? dtf : 0.f, c1 ? dtf : 0.f);
              hdt = fdm_f2(c0 ? 0.5f * dtf : 0.f, c1 ? 0.5f * dtf : 0.f);
            }
            const bool stim0 = node_stim(j0, base + k);
            const bool stim1 = node_stim(j0 + 1, base + k);
            fdm_f2 Pp[NP];
#pragma unroll
            for (int q = 0; q < NP; q++)
              Pp[q] = sP2[(p * NP + q) * T + tid];
            if ((stim0 || stim1) && a.stimulus_mode == 1) {
              fdm_f2 Pk[NP];
              const float sv = (float)a.stimulus_value;
#pragma unroll
              for (int q = 0; q < NP; q++) {
                Pk[q] = Pp[q];
                if (q == a.stimulus_parameter) {
                  if (stim0)
                    Pk[q].v.x = sv;
                  if (stim1)
                    Pk[q].v.y = sv;
                }
              }
              heun_step2<Model>(Vf[p], LV[p], V[j0], V[j0 + 1], S2[p], L2[p], Pk, fdm_f2((float)t), dtr, hdt,
                                    false, false, a.vstim);
            } else {
              heun_step2<Model>(Vf[p], LV[p], V[j0], V[j0 + 1], S2[p], L2[p], Pp, fdm_f2((float)t), dtr, hdt,
                                    stim0, stim1, a.vstim);
            }
          }
          if constexpr (M % 2 == 1) {
            if (tid * M + M - 1 < nb && (!gate_on || node_on(M - 1, k)))
              scalar_node(M - 1, t, s.dt0, base + k);
          }
        } else {
#pragma unroll
          for (int j = 0; j < M; j++) {
            if (tid * M + j >= nb || (gate_on && !node_on(j, k)))
              continue;
            scalar_node(j, t, s.dt0, base + k);
          }
        }
      }
      if constexpr (PAIR) {
#pragma unroll
        for (int p = 0; p < MP; p++) {
          V[2 * p] += (double)LV[p].v.x;
          V[2 * p + 1] += (double)LV[p].v.y;
#pragma unroll
          for (int q = 0; q < NSM; q++)
            normalize_pair(S2[p][q], L2[p][q]);
        }
        if constexpr (!gate_on) {
          // nodes beyond the bin carry Vm = 0 into the diffusion (zero coefficients, finite values); only the
          // threads at the bin's end hold such nodes
          if (tid * M + 2 * MP > nb) {
#pragma unroll
            for (int j = 0; j < 2 * MP; j++)
              V[j] = tid * M + j < nb ? V[j] : 0.0;
          }
        }
      }
      if (store_here) {
        const int k = s.n0 - 1;
        const double t = xadd(t0, xmul((double)k, s.dt0));
#pragma unroll
        for (int j = 0; j < M; j++) {
          if (tid * M + j >= nb || (gate_on && !node_on(j, k)))
            continue;
          const bool stim = node_stim(j, base + k);
          RR Sj[NSM], Lj[NSM], Pj[NP];
          unpack(j, Sj, Lj, Pj);
          RR Pk[NP];
#pragma unroll
          for (int p = 0; p < NP; p++)
            Pk[p] = (stim && a.stimulus_mode == 1 && p == a.stimulus_parameter) ? (RR)a.stimulus_value : Pj[p];
          RR alg[Model::nAlgebraics];
          heun_step<Model, RR, Math, true>(V[j], Sj, Lj, Pk, t, s.dt0, stim && a.stimulus_mode == 0, a.vstim, alg);
          repack(j, Sj, Lj);
          store_algebraics<Model>(alg, a.n_alg_out, a.alg_indices, a.alg_out, a.n_nodes, global_node(tid * M + j));
        }
      }
      if (half == 1)
        break;

      // ---- diffusion: block-wide tridiagonal solve in FP64 ----
      vfirst[tid] = V[0];
      vlast[tid] = V[M - 1];
      cluster_sync();
      double vprev = tid > 0 ? vlast[tid - 1] : 0.0;
      double vnext = tid < T - 1 ? vfirst[tid + 1] : 0.0;
      if constexpr (CLUSTER) {
        cg::cluster_group cl = cg::this_cluster();
        if (tid == 0 && crank > 0)
          vprev = cl.map_shared_rank(vlast, crank - 1)[T - 1];
        if (tid == T - 1 && crank < csize - 1)
          vnext = cl.map_shared_rank(vfirst, crank + 1)[0];
      }
      double d[M];
#pragma unroll
      for (int j = 0; j < M; j++) {
        const int q = j * T + tid;
        const double um = j > 0 ? V[j - 1] : vprev;
        const double up = j < M - 1 ? V[j + 1] : vnext;
        d[j] = sc[2 * CAP + q] * um + sc[3 * CAP + q] * V[j] + sc[4 * CAP + q] * up;
      }
      Affine acc{1.0, 0.0};
#pragma unroll
      for (int j = 0; j < M; j++) {
        const int q = j * T + tid;
        acc = compose(acc, Affine{sc[0 * CAP + q], d[j]});
      }
      Affine tot_f;
      // one barrier per scan (block_scan_map), the forward and backward warp totals in separate halves of sF/sG
      const Affine ex_f = block_scan_map<T, false>(acc, sF, sG, &tot_f);
      double dp = cluster_incoming(ex_f, tot_f, false);
#pragma unroll
      for (int j = 0; j < M; j++) {
        const int q = j * T + tid;
        dp = sc[0 * CAP + q] * dp + d[j];
        d[j] = dp;
      }
      Affine bacc{1.0, 0.0};
#pragma unroll
      for (int j = M - 1; j >= 0; j--) {
        const int q = j * T + tid;
        bacc = compose(bacc, Affine{-sc[1 * CAP + q], d[j]});
      }
      // No barrier is needed before the backward scan: its warp totals go to the other half of sF/sG (the
      // forward totals may still be read).  In cluster mode the backward scan's CTA totals take other slots of
      // ctot, and cpre is rewritten only after the backward cluster barrier, which every forward read precedes.
      Affine tot_b;
      const Affine ex_b = block_scan_map<T, true>(bacc, sF + T / 32, sG + T / 32, &tot_b);
      double x = cluster_incoming(ex_b, tot_b, true);
#pragma unroll
      for (int j = M - 1; j >= 0; j--) {
        const int q = j * T + tid;
        x = -sc[1 * CAP + q] * x + d[j];
        V[j] = x;
      }
      // the next writes of vfirst/vlast, sF/sG and ctot come after the next diffusion's first (cluster)
      // barrier, or after this one's backward cluster barrier, which every read of this one precedes
    }
    if (a.trace_slot) {
#pragma unroll
      for (int j = 0; j < M; j++)
        if (s_ts[j * T + tid] >= 0)
          record_trace(a.trace, a.n_trace, a.trace_capacity, a.act, s_ts[j * T + tid], s.global_no, V[j]);
    }
  }

  // cluster mode: no CTA leaves while another may still read its shared memory
  if constexpr (CLUSTER)
    cg::this_cluster().sync();
  if constexpr (PAIR) {
#pragma unroll
    for (int j = 0; j < 2 * MP; j++) {
      RR Sj[NSM], Lj[NSM], Pj[NP];
      unpack(j, Sj, Lj, Pj);
#pragma unroll
      for (int s = 0; s < NSM; s++) {
        S[j][s] = Sj[s];
        L[j][s] = Lj[s];
      }
    }
  }
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int q = tid * M + j;
    if (q < nb) {
      const int64_t i = global_node(q);
      a.vm[i] = V[j];
#pragma unroll
      for (int s = 1; s < NS; s++) {
        st[(s - 1) * a.stride + i] = S[j][s - 1];
        if (Compensated<RR>::value)
          stl[(s - 1) * a.stride + i] = L[j][s - 1];
      }
    }
  }
}

template<class Model, class RR, class Math, int T, int M>
constexpr size_t fused_smem_bytes()
{
  constexpr bool PAIR = std::is_same<RR, float>::value && std::is_same<Math, fdm_math_exact>::value;
  constexpr int NP = Model::nParameters > 0 ? Model::nParameters : 1;
  return sizeof(double) * (5 * T * M + 2 * T + 4 * (T / 32) + 2) + sizeof(int) * 3 * T * M +
         (PAIR ? sizeof(fdm_f2) * (M / 2) * NP * T : 0);
}

} // namespace fdm
