// Host side of the fiber monodomain solver and its C ABI (include/fdm_b200.h).
//
// The solver restates the host logic of the reference's FastMonodomainSolverBase:
//   time stepping rule        core/src/time_stepping_scheme/00_time_stepping_scheme.cpp:15-68
//   RepeatedCall loop         core/src/time_stepping_scheme/repeated_call.tpp:43-80
//   Strang step timing        fast_monodomain_solver_compute.tpp:64-129
//   NMJ clamp selection       fast_monodomain_solver_compute.tpp:158-166 (vc) / fast_monodomain_solver_gpu.tpp:538-540
//   stimulation machine init  fast_monodomain_solver_initialization.tpp:342-347
// and drives the kernels of fdm_kernels.cuh over launch windows of split steps.
//
// Time values are computed here with the exact C expressions of the reference; this file is
// compiled with -ffp-contract=off so that no multiply-add is fused.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/fdm_b200.h"
#include "fdm_internal.h"

using namespace fdm;

namespace {

thread_local std::string g_create_error;

struct Tss {
  double start = 0, end = 0, dt = 0, target = 0;
  int n = 1;
  void init(double s, double e, double d)
  {
    start = s;
    end = e;
    dt = d;
    target = d;
  }
  void set_dt(double d)
  {
    target = d;
    long double nn = std::ceil((long double)(end - start) / d - 1e-1);
    n = nn < 1 ? 1 : (int)nn;
    dt = (end - start) / n;
  }
  void set_span(double s, double e)
  {
    start = s;
    end = e;
    if (target > e - s)
      dt = e - s;
    set_dt(dt);
  }
};

// Allocation-failure hook (fdm_debug_fail_allocation): the countdown-th allocation of a solver buffer from
// the moment it is set fails as if the device were out of memory; 0 = off.
std::atomic<int64_t> g_fail_countdown{0};

bool injected_allocation_failure()
{
  int64_t c = g_fail_countdown.load();
  while (c > 0) {
    if (g_fail_countdown.compare_exchange_weak(c, c - 1))
      return c == 1;
  }
  return false;
}

// device memory of the solver handles (pinned host staging: pinned_alloc); both honour the hook
cudaError_t device_alloc(void** p, size_t bytes)
{
  if (injected_allocation_failure())
    return cudaErrorMemoryAllocation;
  return cudaMalloc(p, bytes);
}

cudaError_t pinned_alloc(void** p, size_t bytes)
{
  if (injected_allocation_failure())
    return cudaErrorMemoryAllocation;
  return cudaMallocHost(p, bytes);
}

template<class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t count)
  {
    if (count <= n && p)
      return cudaSuccess;
    if (p)
      cudaFree(p);
    p = nullptr;
    n = 0;
    if (count == 0)
      count = 1;
    cudaError_t e = device_alloc((void**)&p, count * sizeof(T));
    if (e == cudaSuccess)
      n = count;
    return e;
  }
  void release()
  {
    if (p)
      cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

} // namespace

struct fdm_solver {
  fdm_config cfg{};
  const ModelDesc* model = nullptr;
  std::string err;
  cudaStream_t stream = nullptr;
  int real_bytes = 8;

  // fibers
  int n_fibers = 0;
  int64_t n_nodes = 0;
  std::vector<int64_t> off;
  std::vector<int64_t> elem_off;
  std::vector<double> prefactor;
  int64_t max_fiber_len = 0;

  // fused bins
  int shape = -1;    // index into fused_shapes, or into cluster_shapes when cluster > 1
  int cluster = 1;   // CTAs per fiber (thread-block cluster mode when > 1)
  int n_bins = 0;
  std::vector<int> bin_start, bin_fibers;

  // clamp selection
  std::vector<int64_t> clamp_first;
  std::vector<int> clamp_count;
  std::vector<uint8_t> evaluated;

  // device buffers
  DevBuf<double> vm, coef, scratch, prefactor_d, elem_d, alg_out, trace;
  DevBuf<unsigned char> states, states_lo, params;
  DevBuf<int64_t> off_d, elem_off_d;
  DevBuf<int> clamp_fiber, bin_start_d, bin_fibers_d, alg_idx, trace_slot, nonfinite;
  // onlyComputeIfHasBeenStimulated: per node code (attributed fiber * 4 + class), per fiber and half step of
  // a window the first substep a junction-class node computes (0 = all, 255 = none)
  DevBuf<int> gate;
  DevBuf<uint8_t> gate_start;
  std::vector<int> gate_h;
  bool gate_set = false;

  // disableComputationWhenStatesAreCloseToEquilibrium (fdm_equilibrium.cuh): buffer layout of the ranks,
  // statuses (double-buffered per half step), counts, padding lanes and the speculative results
  struct Equilibrium {
    bool on = false;
    int64_t n_buffers = 0;
    int n_pad = 0;
    std::vector<int> pad_src;       // per padding lane: node whose parameters it holds
    DevBuf<int> buf_of, lane_node, jfiber, buf_rank, rank_first, counter, nbuf, pad_clamp, pad_gate;
    DevBuf<uint8_t> st[2], info, prefix, block_agg, ran_b;
    DevBuf<double> vm_pad, vm_a, vm_b, alg_a, alg_b;
    DevBuf<uint8_t> states_pad, states_lo_pad, params_pad, st_a, stl_a, st_b, stl_b; // reaction precision
    DevBuf<uint8_t> ck_st, ck_states_pad, ck_states_lo_pad;
    DevBuf<int> ck_counter;
    DevBuf<double> ck_vm_pad;
    bool ck_valid = false;
  } eq;
  DevBuf<uint8_t> firing, evaluated_d, hbs;
  DevBuf<uint8_t> cur_stim;        // per fiber: did its last stimulation decision stimulate
  // stimulation log: (time, fiber) of the stimulation begins, log_cap entries, log_n counts all
  DevBuf<double> log_t;
  DevBuf<int> log_f;
  DevBuf<unsigned long long> log_n;
  int64_t log_cap = 0;
  int64_t log_dropped = 0;  // begins counted past the capacity before the log last grew (not stored)
  DevBuf<int> mu;
  DevBuf<double> freq, repeat, begin, jitter, last_check, cur_jitter;
  DevBuf<int> jitter_idx;
  DevBuf<uint32_t> flags;
  DevBuf<SplitStep> steps_d;
  SplitStep* steps_h = nullptr;   // pinned, 2 slots of step_capacity
  int step_capacity = 0;
  cudaEvent_t slot_ev[2] = {nullptr, nullptr};
  int slot = 0;
  int firing_rows = 0, firing_cols = 0, n_jitter = 0;
  bool stimulation_set = false;
  std::vector<double> stim_freq, stim_begin; // for rewinding the stimulation machine

  // checkpoint
  DevBuf<double> ck_vm, ck_last, ck_jit;
  DevBuf<unsigned char> ck_states, ck_states_lo;
  DevBuf<int> ck_jidx;
  DevBuf<uint8_t> ck_hbs, ck_cur;
  bool ck_valid = false;
  Tss ck_strang, ck_heun, ck_diff;
  bool ck_tss_init = false;
  int64_t ck_split = 0;

  // time stepping state (persists across advances, as the reference's scheme objects do)
  Tss strang, heun, diff;
  bool tss_init = false;
  double coef_dt = -1.0;
  bool coef_valid = false;
  int64_t split_no = 0;

  // outputs
  int n_alg_out = 0;
  int n_trace = 0;
  int64_t trace_capacity = 0;
  int64_t trace_base = 0;        // split step number at fdm_set_trace: trace rows count from it
  // activation recording on the traced nodes (fdm_set_activation_recording)
  DevBuf<double> act_prev;
  DevBuf<int> act_count, act_steps;
  double act_threshold = 0.0;
  int act_cap = 0;

  // adjoint (checkpointed forward, replay + reverse)
  struct Adjoint {
    bool ready = false;
    int kc = 0, n_seg = 0, n_sensors = 0, n0max = 1;
    std::vector<SplitStep> steps;
    std::vector<double> dt1s;
    DevBuf<double> ck_vm, ck_states, ck_last, ck_jit, fin_vm, fin_states, fin_last, fin_jit;
    DevBuf<int> ck_jidx, fin_jidx;
    DevBuf<uint8_t> ck_hbs, fin_hbs;
    Tss fin_strang, fin_heun, fin_diff;
    int64_t fin_split = 0;
    // two buffer sets (stored substep states H, Vm before each diffusion solve U -- Vm after it is the
    // stored input of the next half step --, stimulation bits)
    // so that the replay of one segment overlaps the reverse sweep of the next one in reverse order
    DevBuf<double> H[2], U[2], lam, gP, gpf, mu, ascratch, tgrad;
    DevBuf<double> coefs;                           // one factorization per distinct diffusion step width
    DevBuf<uint32_t> flags[2];
    DevBuf<uint8_t> gates[2];
    cudaStream_t rstream = nullptr;                 // reverse sweeps
    cudaEvent_t replayed[2] = {nullptr, nullptr};   // buffer k filled by a replay
    cudaEvent_t reversed[2] = {nullptr, nullptr};   // buffer k consumed by a reverse sweep
    void release()
    {
      for (auto* b : {&ck_vm, &ck_states, &ck_last, &ck_jit, &fin_vm, &fin_states, &fin_last, &fin_jit, &H[0], &H[1],
                      &U[0], &U[1], &lam, &gP, &gpf, &mu, &ascratch, &tgrad, &coefs})
        b->release();
      flags[0].release();
      flags[1].release();
      gates[0].release();
      gates[1].release();
      ck_jidx.release();
      fin_jidx.release();
      ck_hbs.release();
      fin_hbs.release();
      for (int k = 0; k < 2; k++) {
        if (replayed[k])
          cudaEventDestroy(replayed[k]);
        if (reversed[k])
          cudaEventDestroy(reversed[k]);
        replayed[k] = reversed[k] = nullptr;
      }
      if (rstream)
        cudaStreamDestroy(rstream);
      rstream = nullptr;
      ready = false;
    }
  } adj;

  // pinned host staging for the state transfers, and the events that mark the chunks of a device-to-host
  // transfer as landed
  void* stage = nullptr;
  size_t stage_bytes = 0;
  std::vector<cudaEvent_t> xfer_ev;
  DevBuf<double> xfer64; // direct transfers from fdm_host_alloc memory: the other states in FP64 (FP32 mode)

  // split-path window graphs: (steps, words, nsub, flags pointer) -> executable graph
  std::map<std::tuple<int, int, int, const void*>, cudaGraphExec_t> graphs;

  // timing
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  double main_ms = 0, adv_ms = 0, adj_ms = 0;
  bool finish_pending = false;   // an fdm_advance_async whose timing and NaN check fdm_wait still owes
  bool adj_forward = false;      // inside fdm_adjoint_forward: the reaction runs one thread per node
  int adjoint_tape = 1; // FDM_ADJOINT_TAPE=0 selects the re-evaluating reverse step (for measurements)
  int64_t main_launches = 0, launches = 0;
  cudaEvent_t adv_start = nullptr, adv_stop = nullptr;
};

static int fail(fdm_solver* s, int code, const std::string& msg)
{
  if (s)
    s->err = msg;
  else
    g_create_error = msg;
  return code;
}

int fdm::fdm_report_error(int code, const std::string& msg)
{
  g_create_error = msg;
  return code;
}

static int cuda_fail(fdm_solver* s, cudaError_t e, const char* what)
{
  return fail(s, FDM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// every entry point that touches the device first makes the solver's device current
#define FDM_BIND(s)                                            \
  do {                                                         \
    cudaError_t eb_ = cudaSetDevice((s)->cfg.device);          \
    if (eb_ != cudaSuccess)                                    \
      return cuda_fail((s), eb_, "cudaSetDevice");             \
  } while (0)

#define FDM_CUDA(call)                          \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess)                      \
      return cuda_fail(s, e_, #call);           \
  } while (0)

// captured window graphs hold kernel arguments by value: drop them whenever those can change
static void invalidate_graphs(fdm_solver* s)
{
  for (cudaEvent_t e : s->xfer_ev)
    cudaEventDestroy(e);
  s->xfer_ev.clear();
  s->xfer64.release();
  for (auto& kv : s->graphs)
    cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
}

extern "C" void fdm_config_default(fdm_config* c)
{
  std::memset(c, 0, sizeof(*c));
  c->model = FDM_MODEL_HODGKIN_HUXLEY_1952;
  c->diffusion_scheme = FDM_IMPLICIT_EULER;
  c->method = FDM_METHOD_SPLIT;
  c->reaction_precision = FDM_FP64;
  c->approximate_exponential_function = 0;
  c->clamp_rule = FDM_CLAMP_VC_LANES;
  c->vc_width = 4;
  c->n_ranks = 1;
  c->stimulus_mode = FDM_STIMULUS_CLAMP;
  c->stimulus_parameter = 0;
  c->stimulus_value = 0.0;
  c->value_for_stimulated_point = 20.0;
  c->dt_repeated_call = 1e-3;
  c->dt_splitting = 1e-3;
  c->dt_0d = 1e-4;
  c->dt_1d = 1e-3;
  c->steps_per_launch = 0;
  c->threads_per_block = 0;
  c->nodes_per_thread = 0;
  c->check_nan = 1;
  c->profile = 0;
  c->device = 0;
  c->use_graph = 1;
}

extern "C" const char* fdm_last_error(const fdm_solver* s)
{
  return s ? s->err.c_str() : g_create_error.c_str();
}

extern "C" int fdm_model_parameter_defaults(int model, double* defaults)
{
  const ModelDesc* m = model_desc(model);
  if (!m || !defaults)
    return fail(nullptr, FDM_ERR_ARG, "fdm_model_parameter_defaults: bad argument");
  std::memcpy(defaults, m->parameter_defaults, sizeof(double) * m->n_parameters);
  return FDM_OK;
}

extern "C" int fdm_register_model_library(const char* path, int* model_id)
{
  if (!path || !model_id)
    return fail(nullptr, FDM_ERR_ARG, "fdm_register_model_library: bad argument");
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) {
    const char* why = dlerror();
    return fail(nullptr, FDM_ERR_ARG, std::string("fdm_register_model_library: cannot load ") + path + ": " +
                                          (why ? why : "unknown error"));
  }
  auto entry = (ModelModuleEntry)dlsym(h, "fdm_model_module_v1");
  ModelModule m{};
  if (!entry || entry(&m) != 0) {
    dlclose(h);
    return fail(nullptr, FDM_ERR_ARG, std::string("fdm_register_model_library: ") + path +
                                          " is not a model module (no fdm_model_module_v1)");
  }
  if (m.abi != FDM_MODEL_MODULE_ABI) {
    dlclose(h);
    return fail(nullptr, FDM_ERR_ARG, std::string("fdm_register_model_library: ") + path +
                                          " was built against another version of this library; rebuild it");
  }
  for (int k = 0; k < n_models(); k++) { // the same model loaded again: its existing number
    const ModelDesc* d = model_desc(k);
    if (d && d->name && m.desc.name && std::strcmp(d->name, m.desc.name) == 0) {
      *model_id = k;
      return FDM_OK;   // the library stays loaded (its handle is kept by the first registration)
    }
  }
  const int id = register_model_module(m);
  if (id < 0) {
    dlclose(h);
    return fail(nullptr, FDM_ERR_ARG, "fdm_register_model_library: too many model modules");
  }
  *model_id = id;
  return FDM_OK;   // the library stays loaded for the life of the process
}

extern "C" int fdm_model_info(int model, int* n_states, int* n_algebraics, int* n_parameters, double* states_initial)
{
  const ModelDesc* m = model_desc(model);
  if (!m)
    return fail(nullptr, FDM_ERR_ARG, "unknown model");
  if (n_states)
    *n_states = m->n_states;
  if (n_algebraics)
    *n_algebraics = m->n_algebraics;
  if (n_parameters)
    *n_parameters = m->n_parameters;
  if (states_initial)
    std::memcpy(states_initial, m->states_initial, sizeof(double) * m->n_states);
  return FDM_OK;
}

extern "C" int fdm_fused_cluster_shapes(int* threads, int* nodes_per_thread, int capacity)
{
  FusedShape sh[64];
  const int n = cluster_shapes(sh, 64);
  for (int i = 0; i < n && i < capacity; i++) {
    if (threads)
      threads[i] = sh[i].threads;
    if (nodes_per_thread)
      nodes_per_thread[i] = sh[i].nodes_per_thread;
  }
  return n;
}

extern "C" int fdm_fused_layout(const fdm_solver* s, int* threads, int* nodes_per_thread, int* cluster_size,
                                int* n_blocks)
{
  if (!s || s->cfg.method != FDM_METHOD_FUSED || s->shape < 0)
    return fail(const_cast<fdm_solver*>(s), FDM_ERR_ARG, "fdm_fused_layout: no fused launch set up");
  FusedShape sh[64];
  if (s->cluster > 1)
    cluster_shapes(sh, 64);
  else
    fused_shapes(sh, 64);
  if (threads)
    *threads = sh[s->shape].threads;
  if (nodes_per_thread)
    *nodes_per_thread = sh[s->shape].nodes_per_thread;
  if (cluster_size)
    *cluster_size = s->cluster;
  if (n_blocks)
    *n_blocks = s->n_bins * s->cluster;
  return FDM_OK;
}

extern "C" int fdm_fused_shapes(int* threads, int* nodes_per_thread, int capacity)
{
  FusedShape sh[64];
  const int n = fused_shapes(sh, 64);
  for (int i = 0; i < n && i < capacity; i++) {
    if (threads)
      threads[i] = sh[i].threads;
    if (nodes_per_thread)
      nodes_per_thread[i] = sh[i].nodes_per_thread;
  }
  return n;
}

extern "C" int fdm_create(const fdm_config* cfg, fdm_solver** out)
{
  if (!cfg || !out)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: null argument");
  *out = nullptr;
  const ModelDesc* m = model_desc(cfg->model);
  if (!m)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: unknown model");
  if (cfg->diffusion_scheme != FDM_IMPLICIT_EULER && cfg->diffusion_scheme != FDM_CRANK_NICOLSON)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: diffusion scheme must be ImplicitEuler or CrankNicolson");
  if (cfg->method != FDM_METHOD_SPLIT && cfg->method != FDM_METHOD_FUSED)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: unknown method");
  if (cfg->method == FDM_METHOD_FUSED && !m->fused_supported)
    return fail(nullptr, FDM_ERR_UNSUPPORTED,
                std::string("fdm_create: the fused kernel is not built for model ") + m->name +
                    " (its states do not fit in registers); use FDM_METHOD_SPLIT");
  if (cfg->reaction_precision != FDM_FP64 && cfg->reaction_precision != FDM_FP32_REACTION)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: unknown reaction precision");
  if (cfg->clamp_rule != FDM_CLAMP_VC_LANES && cfg->clamp_rule != FDM_CLAMP_CENTER)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: unknown clamp rule");
  if (cfg->vc_width < 1 || cfg->n_ranks < 1)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: vc_width and n_ranks must be >= 1");
  if (cfg->stimulus_mode == FDM_STIMULUS_CURRENT &&
      (cfg->stimulus_parameter < 0 || cfg->stimulus_parameter >= m->n_parameters))
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: stimulus_parameter out of range");
  if (!(cfg->dt_repeated_call > 0) || !(cfg->dt_splitting > 0) || !(cfg->dt_0d > 0) || !(cfg->dt_1d > 0))
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: time step widths must be positive");
  if (cfg->cluster_size < 0 || cfg->cluster_size > FDM_MAX_CLUSTER)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: cluster_size must be in [0, 8]");
  if (cfg->cluster_size >= 2 &&
      (cfg->method != FDM_METHOD_FUSED || cfg->model != FDM_MODEL_HODGKIN_HUXLEY_1952 ||
       cfg->approximate_exponential_function || cfg->only_compute_if_stimulated))
    return fail(nullptr, FDM_ERR_UNSUPPORTED, "fdm_create: cluster mode needs FDM_METHOD_FUSED, the HH model, exact "
                                              "exponentials and only_compute_if_stimulated off");
  if (cfg->skip_close_to_equilibrium &&
      (cfg->method != FDM_METHOD_SPLIT || cfg->clamp_rule != FDM_CLAMP_VC_LANES))
    return fail(nullptr, FDM_ERR_UNSUPPORTED, "fdm_create: the equilibrium skip (point buffers of the vc path) "
                                              "needs FDM_METHOD_SPLIT and FDM_CLAMP_VC_LANES");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, FDM_ERR_NO_DEVICE, "fdm_create: no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev)
    return fail(nullptr, FDM_ERR_ARG, "fdm_create: device ordinal out of range");
  if (cudaSetDevice(cfg->device) != cudaSuccess)
    return fail(nullptr, FDM_ERR_CUDA, "fdm_create: cudaSetDevice failed");
  fdm_solver* s = new fdm_solver();
  s->cfg = *cfg;
  if (s->cfg.steps_per_launch <= 0)
    s->cfg.steps_per_launch = 100;
  s->model = m;
  s->real_bytes = cfg->reaction_precision == FDM_FP64 ? 8 : 4;
  if (const char* env = std::getenv("FDM_ADJOINT_TAPE"))
    s->adjoint_tape = std::atoi(env) != 0;
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = pinned_alloc((void**)&s->steps_h, sizeof(SplitStep) * 2 * s->cfg.steps_per_launch);
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&s->slot_ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaEventCreateWithFlags(&s->slot_ev[1], cudaEventDisableTiming);
  if (e == cudaSuccess)
    e = cudaEventCreate(&s->adv_start);
  if (e == cudaSuccess)
    e = cudaEventCreate(&s->adv_stop);
  if (e == cudaSuccess)
    e = s->steps_d.alloc(s->cfg.steps_per_launch);
  s->step_capacity = s->cfg.steps_per_launch;
  if (e == cudaSuccess)
    e = s->nonfinite.alloc(1);
  if (e != cudaSuccess) {
    fdm_destroy(s);
    return fail(nullptr, FDM_ERR_CUDA, std::string("fdm_create: ") + cudaGetErrorString(e));
  }
  *out = s;
  return FDM_OK;
}

extern "C" int fdm_destroy(fdm_solver* s)
{
  if (!s)
    return FDM_OK;
  cudaSetDevice(s->cfg.device);
  if (s->stream)
    cudaStreamSynchronize(s->stream);
  for (auto* b : {&s->vm, &s->coef, &s->scratch, &s->prefactor_d, &s->elem_d, &s->alg_out, &s->trace, &s->freq,
                  &s->repeat, &s->begin, &s->jitter, &s->last_check, &s->cur_jitter, &s->ck_vm, &s->ck_last,
                  &s->ck_jit})
    b->release();
  s->states.release();
  s->states_lo.release();
  s->params.release();
  s->ck_states.release();
  s->ck_states_lo.release();
  s->off_d.release();
  s->elem_off_d.release();
  for (auto* b : {&s->clamp_fiber, &s->bin_start_d, &s->bin_fibers_d, &s->alg_idx, &s->trace_slot, &s->nonfinite,
                  &s->mu, &s->jitter_idx, &s->ck_jidx})
    b->release();
  s->firing.release();
  s->evaluated_d.release();
  s->hbs.release();
  s->ck_hbs.release();
  s->cur_stim.release();
  s->ck_cur.release();
  s->log_t.release();
  s->log_f.release();
  s->log_n.release();
  s->log_cap = 0;
  s->log_dropped = 0;
  s->act_prev.release();
  s->act_count.release();
  s->act_steps.release();
  s->flags.release();
  s->steps_d.release();
  s->adj.release();
  for (auto& kv : s->graphs)
    cudaGraphExecDestroy(kv.second);
  s->graphs.clear();
  if (s->stage)
    cudaFreeHost(s->stage);
  if (s->steps_h)
    cudaFreeHost(s->steps_h);
  for (auto ev : s->slot_ev)
    if (ev)
      cudaEventDestroy(ev);
  for (auto ev : s->ev_pool)
    cudaEventDestroy(ev);
  if (s->adv_start)
    cudaEventDestroy(s->adv_start);
  if (s->adv_stop)
    cudaEventDestroy(s->adv_stop);
  if (s->stream)
    cudaStreamDestroy(s->stream);
  delete s;
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// fibers, bins
// ---------------------------------------------------------------------------------------------

// First-fit-decreasing packing of whole fibers into bins of `cap` nodes (at most
// FUSED_MAX_FIBERS_PER_BIN fibers per bin); bins are then ordered longest first.
static void pack_bins(const std::vector<int64_t>& off, int64_t cap, std::vector<int>& bin_start,
                      std::vector<int>& bin_fibers)
{
  const int nf = (int)off.size() - 1;
  std::vector<int> order(nf);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
  std::vector<int64_t> fill;
  std::vector<std::vector<int>> bins;
  for (int f : order) {
    const int64_t len = off[f + 1] - off[f];
    int chosen = -1;
    for (size_t b = 0; b < bins.size(); b++)
      if (fill[b] + len <= cap && (int)bins[b].size() < FUSED_MAX_FIBERS_PER_BIN) {
        chosen = (int)b;
        break;
      }
    if (chosen < 0) {
      bins.emplace_back();
      fill.push_back(0);
      chosen = (int)bins.size() - 1;
    }
    bins[chosen].push_back(f);
    fill[chosen] += len;
  }
  bin_start.assign(1, 0);
  bin_fibers.clear();
  for (auto& b : bins) {
    for (int f : b)
      bin_fibers.push_back(f);
    bin_start.push_back((int)bin_fibers.size());
  }
}

static int choose_shape(fdm_solver* s)
{
  FusedShape sh[64];
  const int n = fused_shapes(sh, 64);
  int best = -1;
  int64_t best_cap = 0;
  for (int i = 0; i < n; i++) {
    const int64_t cap = (int64_t)sh[i].threads * sh[i].nodes_per_thread;
    if (s->cfg.threads_per_block > 0 || s->cfg.nodes_per_thread > 0) {
      if (sh[i].threads == s->cfg.threads_per_block && sh[i].nodes_per_thread == s->cfg.nodes_per_thread)
        return cap >= s->max_fiber_len ? i : -2;
      continue;
    }
    // default (without the autotuner): the smallest capacity that holds the longest fiber among the
    // shapes with at least 512 threads (16 warps per SM for the HH register footprint)
    if (cap >= s->max_fiber_len && sh[i].threads >= 512 && (best < 0 || cap < best_cap)) {
      best = i;
      best_cap = cap;
    }
  }
  if (s->cfg.threads_per_block > 0 || s->cfg.nodes_per_thread > 0)
    return -2;
  if (best < 0)
    for (int i = 0; i < n; i++) {
      const int64_t cap = (int64_t)sh[i].threads * sh[i].nodes_per_thread;
      if (cap >= s->max_fiber_len && (best < 0 || cap < best_cap)) {
        best = i;
        best_cap = cap;
      }
    }
  return best;
}

// Cluster mode: a fiber spread over the CTAs of one thread-block cluster. Chosen automatically when the
// regular packing gives fewer CTAs than half the SMs (or no regular shape holds the longest fiber); returns
// the index into cluster_shapes and the CTAs per fiber, or -1 (regular packing), or -2 (a forced cluster
// size or shape that cannot hold the longest fiber).
static int choose_cluster(fdm_solver* s, int regular_bins, int* csize_out)
{
  const fdm_config& c = s->cfg;
  const bool forced = c.cluster_size >= 2;
  const bool shape_forced = c.threads_per_block > 0 || c.nodes_per_thread > 0;
  if (c.cluster_size == 1 || c.method != FDM_METHOD_FUSED || c.model != FDM_MODEL_HODGKIN_HUXLEY_1952 ||
      c.approximate_exponential_function || c.only_compute_if_stimulated)
    return -1;
  int n_sm = 148;
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, c.device);
  if (!forced && (shape_forced || (regular_bins > 0 && 2 * regular_bins > n_sm)))
    return -1;
  FusedShape sh[64];
  const int n = cluster_shapes(sh, 64);
  int best = -1, best_cs = 0;
  int64_t best_key = 0;
  for (int i = 0; i < n; i++) {
    if (shape_forced && (sh[i].threads != c.threads_per_block || sh[i].nodes_per_thread != c.nodes_per_thread))
      continue;
    const int64_t cap = (int64_t)sh[i].threads * sh[i].nodes_per_thread;
    int64_t cs = (s->max_fiber_len + cap - 1) / cap;
    if (forced) {
      if (cs > c.cluster_size)
        continue;
      cs = c.cluster_size;
    } else if (cs < 2 || cs > FDM_MAX_CLUSTER) {
      continue;
    }
    // prefer: all CTAs resident at once, fewer nodes per thread, then more CTAs
    const int64_t ctas = (int64_t)s->n_fibers * cs;
    const int64_t key = (ctas <= n_sm ? 0 : (int64_t)1 << 40) + ((int64_t)sh[i].nodes_per_thread << 20) - ctas;
    if (best < 0 || key < best_key) {
      best = i;
      best_cs = (int)cs;
      best_key = key;
    }
  }
  if (best < 0)
    return forced ? -2 : -1;
  *csize_out = best_cs;
  return best;
}

static int upload_clamp(fdm_solver* s);
static int upload_gate(fdm_solver* s);
static int eq_copy_pad_params(fdm_solver* s);
static int eq_reset(fdm_solver* s);

static int set_fibers(fdm_solver* s, int n_fibers, const int64_t* fiber_offsets, const double* element_lengths,
                      const double* prefactor)
{
  if (!s || n_fibers < 0 || (n_fibers > 0 && (!fiber_offsets || !element_lengths || !prefactor)))
    return fail(s, FDM_ERR_ARG, "fdm_set_fibers: bad argument");
  FDM_BIND(s);
  invalidate_graphs(s);
  if (n_fibers > 0 && fiber_offsets[0] != 0)
    return fail(s, FDM_ERR_ARG, "fdm_set_fibers: fiber_offsets[0] must be 0");
  int64_t maxlen = 0;
  for (int f = 0; f < n_fibers; f++) {
    const int64_t len = fiber_offsets[f + 1] - fiber_offsets[f];
    if (len < 2)
      return fail(s, FDM_ERR_ARG, "fdm_set_fibers: every fiber needs at least 2 nodes (1 element)");
    maxlen = std::max(maxlen, len);
    if (!(prefactor[f] > 0) || !std::isfinite(prefactor[f]))
      return fail(s, FDM_ERR_ARG, "fdm_set_fibers: prefactor must be positive and finite");
  }
  s->n_fibers = n_fibers;
  s->off.assign(fiber_offsets, fiber_offsets + n_fibers + 1);
  if (n_fibers == 0)
    s->off.assign(1, 0);
  s->n_nodes = s->off.back();
  s->max_fiber_len = maxlen;
  s->elem_off.resize(n_fibers + 1);
  for (int f = 0; f <= n_fibers; f++)
    s->elem_off[f] = s->off[f] - f;
  const int64_t n_elem = s->n_nodes - n_fibers;
  for (int64_t e = 0; e < n_elem; e++)
    if (!(element_lengths[e] > 0) || !std::isfinite(element_lengths[e]))
      return fail(s, FDM_ERR_ARG, "fdm_set_fibers: element lengths must be positive and finite");
  s->prefactor.assign(prefactor, prefactor + n_fibers);

  const int NS = s->model->n_states, NP = s->model->n_parameters;
  const int64_t N = std::max<int64_t>(s->n_nodes, 1);
  FDM_CUDA(s->vm.alloc(N));
  FDM_CUDA(s->states.alloc((size_t)N * std::max(NS - 1, 1) * s->real_bytes));
  if (s->real_bytes == 4)
    FDM_CUDA(s->states_lo.alloc((size_t)N * std::max(NS - 1, 1) * 4));
  FDM_CUDA(s->params.alloc((size_t)N * std::max(NP, 1) * s->real_bytes));
  FDM_CUDA(s->coef.alloc((size_t)N * 6));
  if (s->cfg.method == FDM_METHOD_SPLIT)
    FDM_CUDA(s->scratch.alloc(N));
  FDM_CUDA(s->clamp_fiber.alloc(N));
  FDM_CUDA(s->off_d.alloc(n_fibers + 1));
  FDM_CUDA(s->elem_off_d.alloc(n_fibers + 1));
  FDM_CUDA(s->elem_d.alloc(std::max<int64_t>(n_elem, 1)));
  FDM_CUDA(s->prefactor_d.alloc(std::max(n_fibers, 1)));
  FDM_CUDA(cudaMemcpyAsync(s->off_d.p, s->off.data(), sizeof(int64_t) * (n_fibers + 1), cudaMemcpyHostToDevice,
                           s->stream));
  FDM_CUDA(cudaMemcpyAsync(s->elem_off_d.p, s->elem_off.data(), sizeof(int64_t) * (n_fibers + 1),
                           cudaMemcpyHostToDevice, s->stream));
  if (n_elem > 0)
    FDM_CUDA(cudaMemcpyAsync(s->elem_d.p, element_lengths, sizeof(double) * n_elem, cudaMemcpyHostToDevice,
                             s->stream));
  if (n_fibers > 0)
    FDM_CUDA(cudaMemcpyAsync(s->prefactor_d.p, prefactor, sizeof(double) * n_fibers, cudaMemcpyHostToDevice,
                             s->stream));
  s->coef_valid = false;

  // initial states and default parameters (initializeStates on every buffer)
  std::vector<double> st((size_t)NS * s->n_nodes);
  for (int k = 0; k < NS; k++)
    std::fill(st.begin() + (size_t)k * s->n_nodes, st.begin() + (size_t)(k + 1) * s->n_nodes,
              s->model->states_initial[k]);
  int rc = fdm_set_states(s, st.data());
  if (rc)
    return rc;
  // default parameters: the model file's raw value of each constant parameter, 0 for algebraic ones
  std::vector<double> pz((size_t)std::max(NP, 1) * s->n_nodes, 0.0);
  for (int q = 0; q < NP; q++)
    std::fill(pz.begin() + (size_t)q * s->n_nodes, pz.begin() + (size_t)(q + 1) * s->n_nodes,
              s->model->parameter_defaults[q]);
  if (NP > 0) {
    rc = fdm_set_parameters(s, pz.data());
    if (rc)
      return rc;
  }

  // fused bins
  s->cluster = 1;
  if (s->cfg.method == FDM_METHOD_FUSED && n_fibers > 0) {
    const int regular = s->cfg.cluster_size >= 2 ? -1 : choose_shape(s);
    if (regular >= 0) {
      FusedShape sh[64];
      fused_shapes(sh, 64);
      pack_bins(s->off, (int64_t)sh[regular].threads * sh[regular].nodes_per_thread, s->bin_start, s->bin_fibers);
    }
    int csize = 1;
    const int cshape = choose_cluster(s, regular >= 0 ? (int)s->bin_start.size() - 1 : 0, &csize);
    if (cshape >= 0) {
      // one fiber per cluster
      s->shape = cshape;
      s->cluster = csize;
      s->bin_start.resize(n_fibers + 1);
      s->bin_fibers.resize(n_fibers);
      for (int f = 0; f <= n_fibers; f++)
        s->bin_start[f] = f;
      for (int f = 0; f < n_fibers; f++)
        s->bin_fibers[f] = f;
    } else if (regular >= 0 && cshape == -1) {
      s->shape = regular;
    } else {
      return fail(s, FDM_ERR_UNSUPPORTED, "fdm_set_fibers: no fused kernel shape holds the longest fiber (" +
                                              std::to_string(maxlen) +
                                              " nodes) with the requested threads/nodes/cluster size");
    }
    s->n_bins = (int)s->bin_start.size() - 1;
    FDM_CUDA(s->bin_start_d.alloc(s->bin_start.size()));
    FDM_CUDA(s->bin_fibers_d.alloc(std::max<size_t>(s->bin_fibers.size(), 1)));
    FDM_CUDA(cudaMemcpyAsync(s->bin_start_d.p, s->bin_start.data(), sizeof(int) * s->bin_start.size(),
                             cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->bin_fibers_d.p, s->bin_fibers.data(), sizeof(int) * s->bin_fibers.size(),
                             cudaMemcpyHostToDevice, s->stream));
  }
  s->stimulation_set = false;
  s->gate_set = false;
  s->split_no = 0;
  s->tss_init = false;
  s->ck_valid = false;
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

// A failed fdm_set_fibers (a bad argument, a failed allocation) leaves the solver without fibers: its buffers
// may be partly released, so nothing may run on them until fdm_set_fibers succeeds.
extern "C" int fdm_set_fibers(fdm_solver* s, int n_fibers, const int64_t* fiber_offsets,
                              const double* element_lengths, const double* prefactor)
{
  const int rc = set_fibers(s, n_fibers, fiber_offsets, element_lengths, prefactor);
  if (rc != FDM_OK && s) {
    s->n_fibers = 0;
    s->n_nodes = 0;
    s->max_fiber_len = 0;
    s->off.assign(1, 0);
    s->elem_off.assign(1, 0);
    s->prefactor.clear();
    s->n_bins = 0;
    s->bin_start.assign(1, 0);
    s->bin_fibers.clear();
    s->stimulation_set = false;
    s->gate_set = false;
    s->ck_valid = false;
    s->eq.on = false;
    s->n_alg_out = 0;
    s->n_trace = 0;
    s->trace_capacity = 0;
    s->coef_valid = false;
  }
  return rc;
}

extern "C" int fdm_set_prefactor(fdm_solver* s, const double* prefactor)
{
  if (!s || !prefactor)
    return fail(s, FDM_ERR_ARG, "fdm_set_prefactor: bad argument");
  FDM_BIND(s);
  for (int f = 0; f < s->n_fibers; f++)
    if (!(prefactor[f] > 0) || !std::isfinite(prefactor[f]))
      return fail(s, FDM_ERR_ARG, "fdm_set_prefactor: prefactor must be positive and finite");
  s->prefactor.assign(prefactor, prefactor + s->n_fibers);
  if (s->n_fibers > 0)
    FDM_CUDA(cudaMemcpyAsync(s->prefactor_d.p, prefactor, sizeof(double) * s->n_fibers, cudaMemcpyHostToDevice,
                             s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->coef_valid = false;
  return FDM_OK;
}

// host-side parallel loop for the conversions at the boundary
template<class F>
static void parallel_for(size_t n, F fn)
{
  unsigned nt = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (n < (1u << 16) || nt == 1) {
    fn(0, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t chunk = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; t++) {
    const size_t a = t * chunk, b = std::min(n, a + chunk);
    if (a < b)
      th.emplace_back([=] { fn(a, b); });
  }
  for (auto& t : th)
    t.join();
}

static cudaError_t ensure_stage(fdm_solver* s, size_t bytes)
{
  if (bytes <= s->stage_bytes)
    return cudaSuccess;
  if (s->stage)
    cudaFreeHost(s->stage);
  s->stage = nullptr;
  s->stage_bytes = 0;
  cudaError_t e = pinned_alloc(&s->stage, bytes);
  if (e == cudaSuccess)
    s->stage_bytes = bytes;
  return e;
}

// Page-locked host buffers handed out by fdm_host_alloc: start -> size.  A state array that lies inside one
// is transferred by DMA directly, without the staging copy.
static std::mutex g_host_mu;
static std::map<uintptr_t, size_t> g_host_bufs;

static bool host_buffer_holds(const void* p, size_t bytes)
{
  const uintptr_t a = (uintptr_t)p;
  std::lock_guard<std::mutex> lk(g_host_mu);
  auto it = g_host_bufs.upper_bound(a);
  if (it == g_host_bufs.begin())
    return false;
  --it;
  return a >= it->first && a + bytes <= it->first + it->second;
}

extern "C" int fdm_host_alloc(size_t bytes, void** ptr)
{
  if (!ptr || bytes == 0)
    return fail(nullptr, FDM_ERR_ARG, "fdm_host_alloc: bad argument");
  *ptr = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(nullptr, FDM_ERR_NO_DEVICE, "fdm_host_alloc: no CUDA device");
  }
  void* p = nullptr;
  const cudaError_t e = pinned_alloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(nullptr, FDM_ERR_CUDA, std::string("fdm_host_alloc: ") + cudaGetErrorString(e));
  }
  std::lock_guard<std::mutex> lk(g_host_mu);
  g_host_bufs[(uintptr_t)p] = bytes;
  *ptr = p;
  return FDM_OK;
}

extern "C" int fdm_host_free(void* ptr)
{
  if (!ptr)
    return FDM_OK;
  {
    std::lock_guard<std::mutex> lk(g_host_mu);
    auto it = g_host_bufs.find((uintptr_t)ptr);
    if (it == g_host_bufs.end())
      return fail(nullptr, FDM_ERR_ARG, "fdm_host_free: not a pointer from fdm_host_alloc");
    g_host_bufs.erase(it);
  }
  const cudaError_t e = cudaFreeHost(ptr);
  if (e != cudaSuccess)
    return fail(nullptr, FDM_ERR_CUDA, std::string("fdm_host_free: ") + cudaGetErrorString(e));
  return FDM_OK;
}

// State transfers between the caller's FP64 arrays and the device, through pinned staging: the work is cut
// into chunks of nodes; host threads take the chunks in order, and a chunk's DMA is queued as soon as its
// staging part is written (set) or its staging part is converted as soon as its DMA has landed (get), so the
// host copies and conversions overlap the transfers.  A chunk of the other states carries FP64 values, or
// FP32 (value, residual) pairs in FP32 mode.
namespace {
struct XferChunk {
  bool vm;        // Vm (FP64) or the other states
  size_t a, b;    // element range of Vm [0, N) or of the other states [0, M)
};
constexpr size_t kXferChunk = (size_t)1 << 20;

std::vector<XferChunk> xfer_chunks(size_t N, size_t M)
{
  std::vector<XferChunk> c;
  for (size_t a = 0; a < N; a += kXferChunk)
    c.push_back({true, a, std::min(N, a + kXferChunk)});
  for (size_t a = 0; a < M; a += kXferChunk)
    c.push_back({false, a, std::min(M, a + kXferChunk)});
  return c;
}

// runs fn(chunk index) on up to 16 host threads, chunks claimed in order; the first error wins
template<class F>
cudaError_t for_chunks(int device, size_t n, F fn)
{
  std::atomic<size_t> next{0};
  std::atomic<int> err{(int)cudaSuccess};
  auto work = [&]() {
    cudaError_t e = cudaSetDevice(device);
    while (e == cudaSuccess) {
      const size_t j = next.fetch_add(1);
      if (j >= n)
        break;
      e = fn(j);
    }
    if (e != cudaSuccess) {
      int expected = (int)cudaSuccess;
      err.compare_exchange_strong(expected, (int)e);
    }
  };
  const unsigned nt = (unsigned)std::min<size_t>(n, std::min(16u, std::max(1u, std::thread::hardware_concurrency())));
  if (nt <= 1) {
    work();
  } else {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++)
      th.emplace_back(work);
    for (auto& t : th)
      t.join();
  }
  return (cudaError_t)err.load();
}
} // namespace

// SoA host doubles -> device (Vm in FP64, other states in the reaction precision)
extern "C" int fdm_set_states(fdm_solver* s, const double* states)
{
  if (!s || (!states && s->n_nodes > 0))
    return fail(s, FDM_ERR_ARG, "fdm_set_states: bad argument");
  if (s->n_nodes == 0)
    return FDM_OK;
  FDM_BIND(s);
  const int NS = s->model->n_states;
  const size_t N = (size_t)s->n_nodes;
  const size_t M = N * (size_t)std::max(NS - 1, 0);
  if (host_buffer_holds(states, (N + M) * sizeof(double))) {
    // page-locked caller memory: DMA straight from it (FP32 mode: the other states through a device FP64
    // buffer and the conversion kernel)
    FDM_CUDA(cudaMemcpyAsync(s->vm.p, states, N * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    if (M > 0) {
      if (s->real_bytes == 8) {
        FDM_CUDA(cudaMemcpyAsync(s->states.p, states + N, M * sizeof(double), cudaMemcpyHostToDevice, s->stream));
      } else {
        if (s->xfer64.n < M)
          FDM_CUDA(s->xfer64.alloc(M));
        FDM_CUDA(cudaMemcpyAsync(s->xfer64.p, states + N, M * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        FDM_CUDA(launch_states_to_pairs(s->xfer64.p, (float*)s->states.p, (float*)s->states_lo.p, (int64_t)M,
                                        s->stream));
      }
    }
    FDM_CUDA(cudaStreamSynchronize(s->stream));
    return FDM_OK;
  }
  // staging layout: Vm (N doubles), then the other states as FP64 or as FP32 (value, residual) arrays
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  FDM_CUDA(ensure_stage(s, N * 8 + M * 8));
  double* vm = (double*)s->stage;
  double* st = vm + N;
  float* hi = (float*)(vm + N);
  float* lo = hi + M;
  const bool f64 = s->real_bytes == 8;
  const std::vector<XferChunk> chunks = xfer_chunks(N, M);
  FDM_CUDA(for_chunks(s->cfg.device, chunks.size(), [&](size_t j) -> cudaError_t {
    const XferChunk& c = chunks[j];
    const size_t n = c.b - c.a;
    if (c.vm) {
      std::memcpy(vm + c.a, states + c.a, n * sizeof(double));
      return cudaMemcpyAsync(s->vm.p + c.a, vm + c.a, n * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    }
    if (f64) {
      std::memcpy(st + c.a, states + N + c.a, n * sizeof(double));
      return cudaMemcpyAsync((double*)s->states.p + c.a, st + c.a, n * sizeof(double), cudaMemcpyHostToDevice,
                             s->stream);
    }
    for (size_t i = c.a; i < c.b; i++) {
      hi[i] = (float)states[N + i];
      lo[i] = (float)(states[N + i] - (double)hi[i]);
    }
    cudaError_t e = cudaMemcpyAsync((float*)s->states.p + c.a, hi + c.a, n * sizeof(float), cudaMemcpyHostToDevice,
                                    s->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync((float*)s->states_lo.p + c.a, lo + c.a, n * sizeof(float), cudaMemcpyHostToDevice,
                          s->stream);
    return e;
  }));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_get_states(fdm_solver* s, double* states)
{
  if (!s || (!states && s->n_nodes > 0))
    return fail(s, FDM_ERR_ARG, "fdm_get_states: bad argument");
  if (s->n_nodes == 0)
    return FDM_OK;
  FDM_BIND(s);
  const int NS = s->model->n_states;
  const size_t N = (size_t)s->n_nodes;
  const size_t M = N * (size_t)std::max(NS - 1, 0);
  if (host_buffer_holds(states, (N + M) * sizeof(double))) {
    if (M > 0) {
      if (s->real_bytes == 8) {
        FDM_CUDA(cudaMemcpyAsync(states + N, s->states.p, M * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
      } else {
        if (s->xfer64.n < M)
          FDM_CUDA(s->xfer64.alloc(M));
        FDM_CUDA(launch_pairs_to_states((const float*)s->states.p, (const float*)s->states_lo.p, s->xfer64.p,
                                        (int64_t)M, s->stream));
        FDM_CUDA(cudaMemcpyAsync(states + N, s->xfer64.p, M * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
      }
    }
    FDM_CUDA(cudaMemcpyAsync(states, s->vm.p, N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
    return FDM_OK;
  }
  FDM_CUDA(ensure_stage(s, N * 8 + M * 8));
  double* vm = (double*)s->stage;
  double* st = vm + N;
  float* hi = (float*)(vm + N);
  float* lo = hi + M;
  const bool f64 = s->real_bytes == 8;
  const std::vector<XferChunk> chunks = xfer_chunks(N, M);
  while (s->xfer_ev.size() < chunks.size()) {
    cudaEvent_t e = nullptr;
    FDM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    s->xfer_ev.push_back(e);
  }
  // every chunk's DMA queued in order, each followed by its event
  for (size_t j = 0; j < chunks.size(); j++) {
    const XferChunk& c = chunks[j];
    const size_t n = c.b - c.a;
    if (c.vm) {
      FDM_CUDA(cudaMemcpyAsync(vm + c.a, s->vm.p + c.a, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    } else if (f64) {
      FDM_CUDA(cudaMemcpyAsync(st + c.a, (const double*)s->states.p + c.a, n * sizeof(double), cudaMemcpyDeviceToHost,
                               s->stream));
    } else {
      FDM_CUDA(cudaMemcpyAsync(hi + c.a, (const float*)s->states.p + c.a, n * sizeof(float), cudaMemcpyDeviceToHost,
                               s->stream));
      FDM_CUDA(cudaMemcpyAsync(lo + c.a, (const float*)s->states_lo.p + c.a, n * sizeof(float),
                               cudaMemcpyDeviceToHost, s->stream));
    }
    FDM_CUDA(cudaEventRecord(s->xfer_ev[j], s->stream));
  }
  FDM_CUDA(for_chunks(s->cfg.device, chunks.size(), [&](size_t j) -> cudaError_t {
    const cudaError_t e = cudaEventSynchronize(s->xfer_ev[j]);
    if (e != cudaSuccess)
      return e;
    const XferChunk& c = chunks[j];
    if (c.vm)
      std::memcpy(states + c.a, vm + c.a, (c.b - c.a) * sizeof(double));
    else if (f64)
      std::memcpy(states + N + c.a, st + c.a, (c.b - c.a) * sizeof(double));
    else
      for (size_t i = c.a; i < c.b; i++)
        states[N + i] = (double)hi[i] + (double)lo[i];
    return cudaSuccess;
  }));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_get_vm(fdm_solver* s, double* vm)
{
  if (!s || (!vm && s->n_nodes > 0))
    return fail(s, FDM_ERR_ARG, "fdm_get_vm: bad argument");
  if (s->n_nodes == 0)
    return FDM_OK;
  FDM_BIND(s);
  if (s->n_nodes == 0)
    return FDM_OK;
  FDM_CUDA(cudaMemcpyAsync(vm, s->vm.p, sizeof(double) * s->n_nodes, cudaMemcpyDeviceToHost, s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_set_parameters(fdm_solver* s, const double* parameters)
{
  if (!s || (!parameters && s->n_nodes > 0))
    return fail(s, FDM_ERR_ARG, "fdm_set_parameters: bad argument");
  if (s->n_nodes == 0)
    return FDM_OK;
  FDM_BIND(s);
  const int NP = s->model->n_parameters;
  const size_t n = (size_t)NP * s->n_nodes;
  if (n == 0)
    return FDM_OK;
  if (s->real_bytes == 8) {
    FDM_CUDA(cudaMemcpyAsync(s->params.p, parameters, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
  } else {
    std::vector<float> tmp(n);
    for (size_t i = 0; i < n; i++)
      tmp[i] = (float)parameters[i];
    FDM_CUDA(cudaMemcpyAsync(s->params.p, tmp.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s->stream));
  }
  if (s->eq.on) {
    int rc = eq_copy_pad_params(s);
    if (rc)
      return rc;
  }
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_get_parameters(fdm_solver* s, double* parameters)
{
  if (!s || (!parameters && s->n_nodes > 0))
    return fail(s, FDM_ERR_ARG, "fdm_get_parameters: bad argument");
  if (s->n_nodes == 0)
    return FDM_OK;
  FDM_BIND(s);
  const size_t n = (size_t)s->model->n_parameters * s->n_nodes;
  if (n == 0)
    return FDM_OK;
  if (s->real_bytes == 8) {
    FDM_CUDA(cudaMemcpyAsync(parameters, s->params.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
  } else {
    std::vector<float> tmp(n);
    FDM_CUDA(cudaMemcpyAsync(tmp.data(), s->params.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t i = 0; i < n; i++)
      parameters[i] = tmp[i];
  }
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// stimulation
// ---------------------------------------------------------------------------------------------

// Clamp node selection.  Fibers are laid out as on n_ranks ranks (fiberNo % n_ranks), each rank with
// its fibers concatenated (valuesOffset) and cut into buffers of W lanes; a buffer b is "in the centre"
// of the fiber its first lane is attributed to by int(b * W / valuesLength[0]) when the junction index
// falls inside it, and then lanes 0..min(3,W)-1 of b are clamped (compute.tpp:158-166, 03_generator_vc.cpp:1031-1038).
static void select_clamp_vc(int W, int R, int n_fibers, const int64_t* off, const int* center, int64_t* first_out,
                            int* count_out, uint8_t* eval_out)
{
  for (int f = 0; f < n_fibers; f++) {
    first_out[f] = -1;
    count_out[f] = 0;
    eval_out[f] = 0;
  }
  for (int r = 0; r < R; r++) {
    std::vector<int> fib;
    std::vector<int64_t> vo;
    int64_t total = 0;
    for (int f = r; f < n_fibers; f += R) {
      fib.push_back(f);
      vo.push_back(total);
      total += off[f + 1] - off[f];
    }
    if (fib.empty())
      continue;
    vo.push_back(total);
    const int64_t nbuf = (total + W - 1) / W;
    const double factor = (double)W / (double)(vo[1] - vo[0]);
    const int lanes = std::min(3, W);
    for (int64_t b = 0; b < nbuf; b++) {
      int local = (int)(b * factor);
      if (local >= (int)fib.size())
        local = (int)fib.size() - 1;
      const int f = fib[local];
      const int64_t index_in_fiber = b * W - vo[local];
      if ((unsigned long)((long)center[f] - (long)index_in_fiber) < (unsigned long)W) {
        eval_out[f] = 1;
        int64_t first = -1;
        int cnt = 0;
        for (int lane = 0; lane < lanes; lane++) {
          const int64_t i = b * W + lane;
          if (i >= total)
            break;
          const size_t l2 = (size_t)(std::upper_bound(vo.begin(), vo.end(), i) - vo.begin()) - 1;
          const int64_t g = off[fib[l2]] + (i - vo[l2]);
          if (first < 0)
            first = g;
          cnt++;
        }
        first_out[f] = first;
        count_out[f] = cnt;
      }
    }
  }
}

// junction node and its two neighbours inside the fiber (fast_monodomain_solver_gpu.tpp:538-540)
static void select_clamp_center(int n_fibers, const int64_t* off, const int* center, int64_t* first_out,
                                int* count_out, uint8_t* eval_out)
{
  for (int f = 0; f < n_fibers; f++) {
    first_out[f] = -1;
    count_out[f] = 0;
    eval_out[f] = 1;
    const int64_t n = off[f + 1] - off[f];
    const int64_t lo = std::max<int64_t>(center[f] - 1, 0), hi = std::min<int64_t>(center[f] + 1, n - 1);
    if (hi < lo)
      continue;
    first_out[f] = off[f] + lo;
    count_out[f] = (int)(hi - lo + 1);
  }
}

// onlyComputeIfHasBeenStimulated (compute.tpp:158-205): the reference walks the point buffers of a rank in
// order; a buffer is skipped while the flag of the fiber it is attributed to (int(b * W / valuesLength[0]))
// is false, and that flag is set by the fiber's junction buffer when its machine first stimulates.  So a
// node computes every substep once the flag was set before the call (code class any), and within the call
// of the first stimulation: nothing if its buffer lies before the junction buffer (class 0), from the
// stimulating substep on if it is the junction buffer (class 1), everything if it lies after it (class 2).
static void select_gate_vc(int W, int R, int n_fibers, const int64_t* off, const int* center, int* codes)
{
  for (int r = 0; r < R; r++) {
    std::vector<int> fib;
    std::vector<int64_t> vo;
    int64_t total = 0;
    for (int f = r; f < n_fibers; f += R) {
      fib.push_back(f);
      vo.push_back(total);
      total += off[f + 1] - off[f];
    }
    if (fib.empty())
      continue;
    vo.push_back(total);
    const int nl = (int)fib.size();
    const int64_t nbuf = (total + W - 1) / W;
    const double factor = (double)W / (double)(vo[1] - vo[0]);
    auto attributed = [&](int64_t b) {
      int local = (int)(b * factor);
      return local >= nl ? nl - 1 : local;
    };
    std::vector<int64_t> jb(nl, -1);
    for (int64_t b = 0; b < nbuf; b++) {
      const int local = attributed(b);
      const int64_t index_in_fiber = b * W - vo[local];
      if ((unsigned long)((long)center[fib[local]] - (long)index_in_fiber) < (unsigned long)W)
        jb[local] = b;
    }
    int l2 = 0;
    for (int64_t b = 0; b < nbuf; b++) {
      const int local = attributed(b);
      const int cls = jb[local] < 0 ? 0 : (b < jb[local] ? 0 : (b == jb[local] ? 1 : 2));
      for (int lane = 0; lane < W; lane++) {
        const int64_t i = b * W + lane;
        if (i >= total)
          break;
        while (i >= vo[l2 + 1])
          l2++;
        codes[off[fib[l2]] + (i - vo[l2])] = fib[local] * 4 + cls;
      }
    }
  }
}

// the centre-1..centre+1 rule: every node of a fiber follows its own fiber's flag from the substep on
// that sets it
static void select_gate_center(int n_fibers, const int64_t* off, int* codes)
{
  for (int f = 0; f < n_fibers; f++)
    for (int64_t i = off[f]; i < off[f + 1]; i++)
      codes[i] = f * 4 + 1;
}

extern "C" int fdm_select_gate_codes(int clamp_rule, int vc_width, int n_ranks, int n_fibers,
                                     const int64_t* fiber_offsets, const int* stimulation_point_index, int* codes)
{
  if (n_fibers < 0 || vc_width < 1 || n_ranks < 1 ||
      (n_fibers > 0 && (!fiber_offsets || !stimulation_point_index || !codes)))
    return fail(nullptr, FDM_ERR_ARG, "fdm_select_gate_codes: bad argument");
  if (clamp_rule == FDM_CLAMP_VC_LANES)
    select_gate_vc(vc_width, n_ranks, n_fibers, fiber_offsets, stimulation_point_index, codes);
  else if (clamp_rule == FDM_CLAMP_CENTER)
    select_gate_center(n_fibers, fiber_offsets, codes);
  else
    return fail(nullptr, FDM_ERR_ARG, "fdm_select_gate_codes: unknown clamp rule");
  return FDM_OK;
}

extern "C" int fdm_select_clamp_nodes(int clamp_rule, int vc_width, int n_ranks, int n_fibers,
                                      const int64_t* fiber_offsets, const int* stimulation_point_index,
                                      int64_t* first_node, int* count, uint8_t* evaluated)
{
  if (n_fibers < 0 || vc_width < 1 || n_ranks < 1 ||
      (n_fibers > 0 && (!fiber_offsets || !stimulation_point_index || !first_node || !count || !evaluated)))
    return fail(nullptr, FDM_ERR_ARG, "fdm_select_clamp_nodes: bad argument");
  if (clamp_rule == FDM_CLAMP_VC_LANES)
    select_clamp_vc(vc_width, n_ranks, n_fibers, fiber_offsets, stimulation_point_index, first_node, count, evaluated);
  else if (clamp_rule == FDM_CLAMP_CENTER)
    select_clamp_center(n_fibers, fiber_offsets, stimulation_point_index, first_node, count, evaluated);
  else
    return fail(nullptr, FDM_ERR_ARG, "fdm_select_clamp_nodes: unknown clamp rule");
  return FDM_OK;
}

static int upload_gate(fdm_solver* s)
{
  s->gate_set = false;
  FDM_CUDA(s->gate.alloc((size_t)std::max<int64_t>(s->n_nodes, 1)));
  FDM_CUDA(cudaMemcpyAsync(s->gate.p, s->gate_h.data(), sizeof(int) * s->n_nodes, cudaMemcpyHostToDevice, s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->gate_set = true;
  return FDM_OK;
}

// equilibrium skip: padding lanes hold the parameters of their rank's first node (the reference fills
// every lane with the first instance's values before it copies the fibers' values in)
static int eq_copy_pad_params(fdm_solver* s)
{
  auto& E = s->eq;
  const int NP = s->model->n_parameters;
  const int rb = s->real_bytes;
  for (int p = 0; p < E.n_pad; p++)
    for (int q = 0; q < NP; q++)
      FDM_CUDA(cudaMemcpyAsync(E.params_pad.p + ((size_t)q * E.n_pad + p) * rb,
                               (const uint8_t*)s->params.p + ((size_t)q * s->n_nodes + E.pad_src[p]) * rb, rb,
                               cudaMemcpyDeviceToDevice, s->stream));
  return FDM_OK;
}

// statuses all active, counts 0, padding lanes at the model's initial values (initialization.tpp:128-134, 430-431)
static int eq_reset(fdm_solver* s)
{
  auto& E = s->eq;
  const int NS = s->model->n_states;
  const int R = s->cfg.n_ranks;
  for (int k = 0; k < 2; k++)
    FDM_CUDA(cudaMemsetAsync(E.st[k].p, EQ_ACTIVE, std::max<int64_t>(E.n_buffers, 1), s->stream));
  FDM_CUDA(cudaMemsetAsync(E.counter.p, 0, sizeof(int) * R, s->stream));
  if (E.n_pad > 0) {
    std::vector<double> vm(E.n_pad, s->model->states_initial[0]);
    std::vector<uint8_t> st((size_t)std::max(NS - 1, 1) * E.n_pad * s->real_bytes, 0);
    for (int q = 1; q < NS; q++)
      for (int p = 0; p < E.n_pad; p++) {
        const size_t at = ((size_t)(q - 1) * E.n_pad + p) * s->real_bytes;
        if (s->real_bytes == 8) {
          const double v = s->model->states_initial[q];
          std::memcpy(&st[at], &v, 8);
        } else {
          const float v = (float)s->model->states_initial[q];
          std::memcpy(&st[at], &v, 4);
        }
      }
    FDM_CUDA(cudaMemcpyAsync(E.vm_pad.p, vm.data(), sizeof(double) * E.n_pad, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.states_pad.p, st.data(), st.size(), cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemsetAsync(E.states_lo_pad.p, 0, st.size(), s->stream));
  }
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

// the point-buffer layout of the vc path: rank r holds fibers r, r+R, ... concatenated, cut into buffers of W
// lanes; the buffer's attributed fiber int(b W / len0), its junction fiber, and the padding lanes
static int eq_build(fdm_solver* s, const std::vector<int>& center)
{
  auto& E = s->eq;
  E.on = false;   // until every buffer below is in place
  const int W = s->cfg.vc_width, R = s->cfg.n_ranks, nf = s->n_fibers;
  const int64_t N = s->n_nodes;
  const int NS = s->model->n_states, NP = s->model->n_parameters;
  std::vector<int> rank_first(R + 1, 0), nbuf(R, 0), buf_rank, jfiber, lane_node, buf_of(N, 0), pad_clamp, pad_gate;
  std::vector<int> buf_code; // onlyComputeIfHasBeenStimulated code of each buffer (for its padding lanes)
  E.pad_src.clear();
  int n_pad = 0;
  for (int r = 0; r < R; r++) {
    rank_first[r] = (int)buf_rank.size();
    std::vector<int> fib;
    std::vector<int64_t> vo;
    int64_t total = 0;
    for (int f = r; f < nf; f += R) {
      fib.push_back(f);
      vo.push_back(total);
      total += s->off[f + 1] - s->off[f];
    }
    if (fib.empty())
      continue;
    vo.push_back(total);
    const int nl = (int)fib.size();
    const int64_t nb = (total + W - 1) / W;
    nbuf[r] = (int)nb;
    const double factor = (double)W / (double)(vo[1] - vo[0]);
    std::vector<int64_t> jb(nl, -1);
    std::vector<int> att(nb);
    for (int64_t b = 0; b < nb; b++) {
      int local = (int)(b * factor);
      if (local >= nl)
        local = nl - 1;
      att[b] = local;
      const int64_t index_in_fiber = b * W - vo[local];
      if ((unsigned long)((long)center[fib[local]] - (long)index_in_fiber) < (unsigned long)W)
        jb[local] = b;
    }
    int l2 = 0;
    for (int64_t b = 0; b < nb; b++) {
      const int gb = (int)buf_rank.size();
      buf_rank.push_back(r);
      const int local = att[b];
      jfiber.push_back(jb[local] == b ? fib[local] : -1);
      const int cls = jb[local] < 0 ? 0 : (b < jb[local] ? 0 : (b == jb[local] ? 1 : 2));
      buf_code.push_back(fib[local] * 4 + cls);
      for (int lane = 0; lane < W; lane++) {
        const int64_t i = b * W + lane;
        if (i < total) {
          while (i >= vo[l2 + 1])
            l2++;
          const int64_t g = s->off[fib[l2]] + (i - vo[l2]);
          lane_node.push_back((int)g);
          buf_of[g] = gb;
        } else {
          lane_node.push_back((int)(N + n_pad));
          buf_of.push_back(gb);
          pad_clamp.push_back((jb[local] == b && lane < std::min(3, W)) ? fib[local] : -1);
          pad_gate.push_back(fib[local] * 4 + cls);
          E.pad_src.push_back((int)s->off[fib[0]]);
          n_pad++;
        }
      }
    }
  }
  rank_first[R] = (int)buf_rank.size();
  E.n_buffers = (int64_t)buf_rank.size();
  E.n_pad = n_pad;
  const int64_t nt = N + n_pad;
  const size_t nsm = (size_t)std::max(NS - 1, 1), rb = (size_t)s->real_bytes;
  auto up = [&](DevBuf<int>& d, const std::vector<int>& h) -> cudaError_t {
    cudaError_t e = d.alloc(std::max<size_t>(h.size(), 1));
    if (e == cudaSuccess && !h.empty())
      e = cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, s->stream);
    return e;
  };
  FDM_CUDA(up(E.buf_of, buf_of));
  FDM_CUDA(up(E.lane_node, lane_node));
  FDM_CUDA(up(E.jfiber, jfiber));
  FDM_CUDA(up(E.buf_rank, buf_rank));
  FDM_CUDA(up(E.rank_first, rank_first));
  FDM_CUDA(up(E.nbuf, nbuf));
  FDM_CUDA(up(E.pad_clamp, pad_clamp));
  FDM_CUDA(up(E.pad_gate, pad_gate));
  FDM_CUDA(E.counter.alloc(R));
  for (int k = 0; k < 2; k++)
    FDM_CUDA(E.st[k].alloc(std::max<int64_t>(E.n_buffers, 1)));
  FDM_CUDA(E.info.alloc(std::max<int64_t>(E.n_buffers, 1)));
  FDM_CUDA(E.prefix.alloc(std::max<int64_t>(E.n_buffers, 1)));
  FDM_CUDA(E.block_agg.alloc(std::max<int64_t>((E.n_buffers + EQ_SCAN_T - 1) / EQ_SCAN_T, 1)));
  FDM_CUDA(E.ran_b.alloc(std::max<int64_t>(nt, 1)));
  FDM_CUDA(E.vm_pad.alloc(std::max(n_pad, 1)));
  FDM_CUDA(E.states_pad.alloc(nsm * std::max(n_pad, 1) * rb));
  FDM_CUDA(E.states_lo_pad.alloc(nsm * std::max(n_pad, 1) * rb));
  FDM_CUDA(E.params_pad.alloc((size_t)std::max(NP, 1) * std::max(n_pad, 1) * rb));
  FDM_CUDA(E.vm_a.alloc(std::max<int64_t>(nt, 1)));
  FDM_CUDA(E.vm_b.alloc(std::max<int64_t>(nt, 1)));
  FDM_CUDA(E.st_a.alloc(nsm * std::max<int64_t>(nt, 1) * rb));
  FDM_CUDA(E.stl_a.alloc(nsm * std::max<int64_t>(nt, 1) * rb));
  FDM_CUDA(E.st_b.alloc(nsm * std::max<int64_t>(nt, 1) * rb));
  FDM_CUDA(E.stl_b.alloc(nsm * std::max<int64_t>(nt, 1) * rb));
  FDM_CUDA(E.alg_a.alloc((size_t)std::max(s->n_alg_out, 1) * std::max<int64_t>(nt, 1)));
  FDM_CUDA(E.alg_b.alloc((size_t)std::max(s->n_alg_out, 1) * std::max<int64_t>(nt, 1)));
  int rc = eq_copy_pad_params(s);
  if (rc)
    return rc;
  rc = eq_reset(s);
  if (rc)
    return rc;
  E.on = true;
  E.ck_valid = false;
  (void)buf_code;
  return FDM_OK;
}

static int upload_clamp(fdm_solver* s)
{
  std::vector<int> cf((size_t)std::max<int64_t>(s->n_nodes, 1), -1);
  for (int f = 0; f < s->n_fibers; f++)
    for (int k = 0; k < s->clamp_count[f]; k++)
      cf[s->clamp_first[f] + k] = f;
  FDM_CUDA(cudaMemcpyAsync(s->clamp_fiber.p, cf.data(), sizeof(int) * s->n_nodes, cudaMemcpyHostToDevice,
                           s->stream));
  FDM_CUDA(cudaMemcpyAsync(s->evaluated_d.p, s->evaluated.data(), s->n_fibers, cudaMemcpyHostToDevice, s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_set_stimulation(fdm_solver* s, const uint8_t* firing_events, int rows, int cols,
                                   const int* motor_unit_no, const int* stimulation_point_index,
                                   const double* call_frequency, const double* repeat_after_first_call,
                                   const double* call_enable_begin, const double* jitter, int n_jitter)
{
  if (!s || rows < 1 || cols < 1 || !firing_events || n_jitter < 0 || (n_jitter > 0 && !jitter))
    return fail(s, FDM_ERR_ARG, "fdm_set_stimulation: bad argument (firing events need at least one row and column)");
  FDM_BIND(s);
  invalidate_graphs(s);
  const int nf = s->n_fibers;
  if (nf > 0 && (!motor_unit_no || !stimulation_point_index || !call_frequency || !repeat_after_first_call ||
                 !call_enable_begin))
    return fail(s, FDM_ERR_ARG, "fdm_set_stimulation: null per-fiber array");
  std::vector<int> center(nf);
  for (int f = 0; f < nf; f++) {
    if (motor_unit_no[f] < 0)
      return fail(s, FDM_ERR_ARG, "fdm_set_stimulation: motor unit numbers must be >= 0");
    center[f] = stimulation_point_index[f];
    if (call_frequency[f] != 0 && repeat_after_first_call[f] == 0)
      return fail(s, FDM_ERR_ARG,
                  "fdm_set_stimulation: setSpecificStatesCallFrequency is set but setSpecificStatesRepeatAfterFirstCall "
                  "is not (03_cellml_adapter.tpp:177-181)");
  }
  s->stimulation_set = false;   // until every buffer below is in place
  s->eq.on = false;
  s->gate_set = false;
  s->firing_rows = rows;
  s->firing_cols = cols;
  s->n_jitter = n_jitter;
  FDM_CUDA(s->firing.alloc((size_t)rows * cols));
  FDM_CUDA(s->mu.alloc(std::max(nf, 1)));
  FDM_CUDA(s->freq.alloc(std::max(nf, 1)));
  FDM_CUDA(s->repeat.alloc(std::max(nf, 1)));
  FDM_CUDA(s->begin.alloc(std::max(nf, 1)));
  FDM_CUDA(s->jitter.alloc(std::max<size_t>((size_t)nf * n_jitter, 1)));
  FDM_CUDA(s->last_check.alloc(std::max(nf, 1)));
  FDM_CUDA(s->cur_jitter.alloc(std::max(nf, 1)));
  FDM_CUDA(s->jitter_idx.alloc(std::max(nf, 1)));
  FDM_CUDA(s->hbs.alloc(std::max(nf, 1)));
  FDM_CUDA(s->cur_stim.alloc(std::max(nf, 1)));
  FDM_CUDA(s->evaluated_d.alloc(std::max(nf, 1)));
  FDM_CUDA(cudaMemcpyAsync(s->firing.p, firing_events, (size_t)rows * cols, cudaMemcpyHostToDevice, s->stream));
  if (nf > 0) {
    FDM_CUDA(cudaMemcpyAsync(s->mu.p, motor_unit_no, sizeof(int) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->freq.p, call_frequency, sizeof(double) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->repeat.p, repeat_after_first_call, sizeof(double) * nf, cudaMemcpyHostToDevice,
                             s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->begin.p, call_enable_begin, sizeof(double) * nf, cudaMemcpyHostToDevice,
                             s->stream));
    if (n_jitter > 0)
      FDM_CUDA(cudaMemcpyAsync(s->jitter.p, jitter, sizeof(double) * nf * n_jitter, cudaMemcpyHostToDevice,
                               s->stream));
    s->stim_freq.assign(call_frequency, call_frequency + nf);
    s->stim_begin.assign(call_enable_begin, call_enable_begin + nf);
    // initial machine state (initialization.tpp:342-344)
    std::vector<double> last(nf), cj(nf, 0.0);
    std::vector<int> ji(nf, 0);
    std::vector<uint8_t> h0(nf, 0);
    for (int f = 0; f < nf; f++)
      last[f] = call_enable_begin[f] - 1e-13 - 1. / (call_frequency[f] + cj[f]);
    FDM_CUDA(cudaMemcpyAsync(s->last_check.p, last.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->cur_jitter.p, cj.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->jitter_idx.p, ji.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->hbs.p, h0.data(), nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->cur_stim.p, h0.data(), nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
  }
  s->clamp_first.assign(nf, -1);
  s->clamp_count.assign(nf, 0);
  s->evaluated.assign(nf, 0);
  if (s->cfg.clamp_rule == FDM_CLAMP_VC_LANES)
    select_clamp_vc(s->cfg.vc_width, s->cfg.n_ranks, nf, s->off.data(), center.data(), s->clamp_first.data(),
                    s->clamp_count.data(), s->evaluated.data());
  else
    select_clamp_center(nf, s->off.data(), center.data(), s->clamp_first.data(), s->clamp_count.data(),
                        s->evaluated.data());
  int rc = upload_clamp(s);
  if (rc)
    return rc;
  if (s->cfg.skip_close_to_equilibrium) {
    rc = eq_build(s, center);
    if (rc)
      return rc;
  }
  if (s->cfg.only_compute_if_stimulated) {
    s->gate_h.assign((size_t)std::max<int64_t>(s->n_nodes, 1), 0);
    if (s->cfg.clamp_rule == FDM_CLAMP_VC_LANES)
      select_gate_vc(s->cfg.vc_width, s->cfg.n_ranks, nf, s->off.data(), center.data(), s->gate_h.data());
    else
      select_gate_center(nf, s->off.data(), s->gate_h.data());
    rc = upload_gate(s);
    if (rc)
      return rc;
  }
  s->stimulation_set = true;
  return FDM_OK;
}

extern "C" int fdm_get_equilibrium_state(fdm_solver* s, int64_t* n_buffers, uint8_t* status, int* counter)
{
  if (!s || !s->eq.on)
    return fail(s, FDM_ERR_ARG, "fdm_get_equilibrium_state: the equilibrium skip is not on (or fdm_set_stimulation "
                                "was not called)");
  FDM_BIND(s);
  if (n_buffers)
    *n_buffers = s->eq.n_buffers;
  if (status && s->eq.n_buffers > 0)
    FDM_CUDA(cudaMemcpyAsync(status, s->eq.st[0].p, s->eq.n_buffers, cudaMemcpyDeviceToHost, s->stream));
  if (counter)
    FDM_CUDA(cudaMemcpyAsync(counter, s->eq.counter.p, sizeof(int) * s->cfg.n_ranks, cudaMemcpyDeviceToHost,
                             s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

namespace fdm {
int solver_vm_device(fdm_solver* s, const double** vm, int64_t* n_nodes, cudaStream_t* stream, int* device)
{
  if (!s || !s->vm.p)
    return FDM_ERR_ARG;
  *vm = s->vm.p;
  *n_nodes = s->n_nodes;
  *stream = s->stream;
  *device = s->cfg.device;
  return FDM_OK;
}
} // namespace fdm

extern "C" int fdm_get_compute_state_information(fdm_solver* s, double* out)
{
  if (!s || (!out && s->n_nodes > 0) || !s->stimulation_set)
    return fail(s, FDM_ERR_ARG, "fdm_get_compute_state_information: call fdm_set_stimulation first; no null array");
  FDM_BIND(s);
  const int64_t N = s->n_nodes;
  if (N == 0)
    return FDM_OK;
  // the status of the node's point buffer (2 = active for every buffer while the equilibrium skip is off)
  if (s->eq.on) {
    std::vector<int> buf_of(N);
    std::vector<uint8_t> st(s->eq.n_buffers);
    FDM_CUDA(cudaMemcpyAsync(buf_of.data(), s->eq.buf_of.p, sizeof(int) * N, cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaMemcpyAsync(st.data(), s->eq.st[0].p, s->eq.n_buffers, cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
    for (int64_t i = 0; i < N; i++)
      out[i] = (double)st[buf_of[i]];
  } else {
    std::fill(out, out + N, 2.0);
  }
  // -1 on every node of a fiber that has not been stimulated yet (own fiber, onlyComputeIfHasBeenStimulated)
  if (s->cfg.only_compute_if_stimulated) {
    std::vector<uint8_t> hbs(s->n_fibers);
    FDM_CUDA(cudaMemcpyAsync(hbs.data(), s->hbs.p, s->n_fibers, cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
    for (int f = 0; f < s->n_fibers; f++)
      if (!hbs[f])
        std::fill(out + s->off[f], out + s->off[f + 1], -1.0);
  }
  return FDM_OK;
}

extern "C" int fdm_set_gate_codes(fdm_solver* s, const int* codes)
{
  if (!s || !s->stimulation_set || !codes || !s->cfg.only_compute_if_stimulated)
    return fail(s, FDM_ERR_ARG, "fdm_set_gate_codes: needs only_compute_if_stimulated and fdm_set_stimulation first");
  FDM_BIND(s);
  for (int64_t i = 0; i < s->n_nodes; i++)
    if (codes[i] < 0 || codes[i] / 4 >= s->n_fibers || codes[i] % 4 > 2)
      return fail(s, FDM_ERR_ARG, "fdm_set_gate_codes: code out of range");
  s->gate_h.assign(codes, codes + s->n_nodes);
  invalidate_graphs(s);
  return upload_gate(s);
}

extern "C" int fdm_set_clamp_nodes(fdm_solver* s, const int64_t* first_node, const int* count,
                                   const uint8_t* evaluated)
{
  if (!s || !s->stimulation_set || !first_node || !count || !evaluated)
    return fail(s, FDM_ERR_ARG, "fdm_set_clamp_nodes: call fdm_set_stimulation first; no null arrays");
  FDM_BIND(s);
  for (int f = 0; f < s->n_fibers; f++)
    if (count[f] < 0 || (count[f] > 0 && (first_node[f] < 0 || first_node[f] + count[f] > s->n_nodes)))
      return fail(s, FDM_ERR_ARG, "fdm_set_clamp_nodes: clamp nodes out of range");
  s->clamp_first.assign(first_node, first_node + s->n_fibers);
  s->clamp_count.assign(count, count + s->n_fibers);
  s->evaluated.assign(evaluated, evaluated + s->n_fibers);
  invalidate_graphs(s);
  return upload_clamp(s);
}

extern "C" int fdm_get_clamp_nodes(fdm_solver* s, int64_t* first_node, int* count, uint8_t* evaluated)
{
  if (!s || !s->stimulation_set)
    return fail(s, FDM_ERR_ARG, "fdm_get_clamp_nodes: call fdm_set_stimulation first");
  for (int f = 0; f < s->n_fibers; f++) {
    if (first_node)
      first_node[f] = s->clamp_first[f];
    if (count)
      count[f] = s->clamp_count[f];
    if (evaluated)
      evaluated[f] = s->evaluated[f];
  }
  return FDM_OK;
}

extern "C" int fdm_set_algebraics_for_transfer(fdm_solver* s, int n, const int* idx)
{
  if (!s || n < 0 || (n > 0 && !idx))
    return fail(s, FDM_ERR_ARG, "fdm_set_algebraics_for_transfer: bad argument");
  FDM_BIND(s);
  invalidate_graphs(s);
  for (int k = 0; k < n; k++)
    if (idx[k] < 0 || idx[k] >= s->model->n_algebraics)
      return fail(s, FDM_ERR_ARG, "fdm_set_algebraics_for_transfer: algebraic index out of range");
  s->n_alg_out = 0;   // set once the buffers are in place
  FDM_CUDA(s->alg_idx.alloc(std::max(n, 1)));
  FDM_CUDA(s->alg_out.alloc(std::max<size_t>((size_t)n * s->n_nodes, 1)));
  if (n > 0) {
    FDM_CUDA(cudaMemcpyAsync(s->alg_idx.p, idx, sizeof(int) * n, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemsetAsync(s->alg_out.p, 0, sizeof(double) * n * s->n_nodes, s->stream));
  }
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->n_alg_out = n;
  return FDM_OK;
}

extern "C" int fdm_get_algebraics(fdm_solver* s, double* out)
{
  if (!s || !out)
    return fail(s, FDM_ERR_ARG, "fdm_get_algebraics: bad argument");
  FDM_BIND(s);
  if (s->n_alg_out == 0 || s->n_nodes == 0)
    return FDM_OK;
  FDM_CUDA(cudaMemcpyAsync(out, s->alg_out.p, sizeof(double) * s->n_alg_out * s->n_nodes, cudaMemcpyDeviceToHost,
                           s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_set_trace(fdm_solver* s, int n, const int64_t* nodes, int64_t capacity)
{
  if (!s || n < 0 || (n > 0 && !nodes) || capacity < 0)
    return fail(s, FDM_ERR_ARG, "fdm_set_trace: bad argument");
  FDM_BIND(s);
  invalidate_graphs(s);
  std::vector<int> slot((size_t)std::max<int64_t>(s->n_nodes, 1), -1);
  for (int k = 0; k < n; k++) {
    if (nodes[k] < 0 || nodes[k] >= s->n_nodes)
      return fail(s, FDM_ERR_ARG, "fdm_set_trace: node index out of range");
    if (slot[nodes[k]] >= 0)
      return fail(s, FDM_ERR_ARG, "fdm_set_trace: duplicate node");
    slot[nodes[k]] = k;
  }
  s->n_trace = 0;   // set once the buffers are in place
  s->trace_capacity = 0;
  s->act_cap = 0;   // the slots change: activation recording stops (fdm_set_activation_recording restarts it)
  s->trace_base = s->split_no;
  if (n > 0) {
    FDM_CUDA(s->trace_slot.alloc(s->n_nodes));
    FDM_CUDA(s->trace.alloc(std::max<size_t>((size_t)n * capacity, 1)));
    FDM_CUDA(cudaMemcpyAsync(s->trace_slot.p, slot.data(), sizeof(int) * s->n_nodes, cudaMemcpyHostToDevice,
                             s->stream));
    FDM_CUDA(cudaMemsetAsync(s->trace.p, 0, sizeof(double) * std::max<size_t>((size_t)n * capacity, 1), s->stream));
  }
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->n_trace = n;
  s->trace_capacity = n > 0 ? capacity : 0;
  return FDM_OK;
}

extern "C" int fdm_get_trace(fdm_solver* s, double* out, int64_t* n_steps)
{
  if (!s)
    return fail(s, FDM_ERR_ARG, "fdm_get_trace: bad argument");
  FDM_BIND(s);
  const int64_t rec = std::min(std::max<int64_t>(s->split_no - s->trace_base, 0), s->trace_capacity);
  if (n_steps)
    *n_steps = rec;
  if (out && rec > 0 && s->n_trace > 0) {
    FDM_CUDA(cudaMemcpyAsync(out, s->trace.p, sizeof(double) * rec * s->n_trace, cudaMemcpyDeviceToHost, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
  }
  return FDM_OK;
}

extern "C" int fdm_set_activation_recording(fdm_solver* s, double threshold, int capacity_per_node)
{
  if (!s || capacity_per_node < 0 || !std::isfinite(threshold))
    return fail(s, FDM_ERR_ARG, "fdm_set_activation_recording: bad argument");
  if (capacity_per_node > 0 && s->n_trace == 0)
    return fail(s, FDM_ERR_ARG, "fdm_set_activation_recording: set the traced nodes first (fdm_set_trace)");
  FDM_BIND(s);
  {
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  invalidate_graphs(s);
  s->act_cap = 0;   // set once the buffers are in place
  if (capacity_per_node == 0)
    return FDM_OK;
  const size_t n = (size_t)s->n_trace;
  FDM_CUDA(s->act_prev.alloc(n));
  FDM_CUDA(s->act_count.alloc(n));
  FDM_CUDA(s->act_steps.alloc(n * (size_t)capacity_per_node));
  std::vector<double> nan(n, std::numeric_limits<double>::quiet_NaN());
  FDM_CUDA(cudaMemcpyAsync(s->act_prev.p, nan.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
  FDM_CUDA(cudaMemsetAsync(s->act_count.p, 0, sizeof(int) * n, s->stream));
  FDM_CUDA(cudaMemsetAsync(s->act_steps.p, 0xff, sizeof(int) * n * (size_t)capacity_per_node, s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->act_threshold = threshold;
  s->act_cap = capacity_per_node;
  return FDM_OK;
}

extern "C" int fdm_get_activation_steps(fdm_solver* s, int* counts, int* steps)
{
  if (!s)
    return fail(s, FDM_ERR_ARG, "fdm_get_activation_steps: bad argument");
  if (s->act_cap == 0)
    return fail(s, FDM_ERR_ARG, "fdm_get_activation_steps: activation recording is off");
  FDM_BIND(s);
  {
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  const size_t n = (size_t)s->n_trace;
  if (counts)
    FDM_CUDA(cudaMemcpyAsync(counts, s->act_count.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s->stream));
  if (steps)
    FDM_CUDA(cudaMemcpyAsync(steps, s->act_steps.p, sizeof(int) * n * (size_t)s->act_cap, cudaMemcpyDeviceToHost,
                             s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// advance
// ---------------------------------------------------------------------------------------------

static cudaEvent_t next_event(fdm_solver* s)
{
  if (s->ev_used == s->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess)
      return nullptr;
    s->ev_pool.push_back(e);
  }
  return s->ev_pool[s->ev_used++];
}

static int ensure_coefficients(fdm_solver* s, double dt1)
{
  // The reference recomputes dt1D = ((t+dtSplit)-t)/n1D at every call, which varies in the last bits;
  // the factorization is reused while dt1D stays within a relative 1e-12 of the factorized value.
  if (s->coef_valid && std::fabs(dt1 - s->coef_dt) <= 1e-12 * std::fabs(s->coef_dt))
    return FDM_OK;
  FDM_CUDA(launch_coefficients(s->n_fibers, s->off_d.p, s->elem_d.p, s->prefactor_d.p, dt1,
                               s->cfg.diffusion_scheme == FDM_IMPLICIT_EULER, s->coef.p, s->n_nodes, s->stream));
  s->launches++;
  s->coef_dt = dt1;
  s->coef_valid = true;
  return FDM_OK;
}

struct WindowInfo {
  int words = 0, nsub = 1;
  const uint8_t* gate_start = nullptr; // onlyComputeIfHasBeenStimulated: first substeps of the window
  int gate_stride = 0;
};

static ActivationRec activation_rec(const fdm_solver* s)
{
  ActivationRec r{};
  if (s->act_cap > 0 && s->n_trace > 0) {
    r.threshold = s->act_threshold;
    r.prev = s->act_prev.p;
    r.count = s->act_count.p;
    r.steps = s->act_steps.p;
    r.capacity = s->act_cap;
  }
  return r;
}

static int ensure_step_capacity(fdm_solver* s, int n)
{
  if (n <= s->step_capacity)
    return FDM_OK;
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  if (s->steps_h)
    FDM_CUDA(cudaFreeHost(s->steps_h));
  s->steps_h = nullptr;
  s->step_capacity = 0;   // until both buffers are in place
  FDM_CUDA(pinned_alloc((void**)&s->steps_h, sizeof(SplitStep) * 2 * (size_t)n));
  FDM_CUDA(s->steps_d.alloc(n));
  s->step_capacity = n;
  return FDM_OK;
}

// uploads a window of split steps (through a pinned slot) and runs the stimulation schedule for it
static int prepare_window(fdm_solver* s, const SplitStep* host_steps, int n_steps, WindowInfo* wi,
                          uint32_t* flags_buf = nullptr, uint8_t* gate_buf = nullptr)
{
  int rc = ensure_step_capacity(s, n_steps);
  if (rc)
    return rc;
  const int slot = s->slot;
  s->slot ^= 1;
  FDM_CUDA(cudaEventSynchronize(s->slot_ev[slot]));
  SplitStep* hs = s->steps_h + (size_t)slot * s->step_capacity;
  std::memcpy(hs, host_steps, sizeof(SplitStep) * n_steps);
  int nsub = 1;
  for (int j = 0; j < n_steps; j++)
    nsub = std::max(nsub, hs[j].n0);
  const int bits = n_steps * 2 * nsub;
  const int words = (bits + 31) / 32;
  if (!flags_buf)
    FDM_CUDA(s->flags.alloc((size_t)words * std::max(s->n_fibers, 1)));
  FDM_CUDA(cudaMemcpyAsync(s->steps_d.p, hs, sizeof(SplitStep) * n_steps, cudaMemcpyHostToDevice, s->stream));
  FDM_CUDA(cudaEventRecord(s->slot_ev[slot], s->stream));
  wi->words = words;
  wi->nsub = nsub;
  StimArgs sa{};
  sa.firing_events = s->firing.p;
  sa.rows = s->firing_rows;
  sa.cols = s->firing_cols;
  sa.motor_unit_no = s->mu.p;
  sa.call_frequency = s->freq.p;
  sa.repeat_after_first_call = s->repeat.p;
  sa.call_enable_begin = s->begin.p;
  sa.jitter = s->jitter.p;
  sa.n_jitter = s->n_jitter;
  sa.evaluated = s->evaluated_d.p;
  sa.last_check_time = s->last_check.p;
  sa.current_jitter = s->cur_jitter.p;
  sa.jitter_index = s->jitter_idx.p;
  sa.has_been_stimulated = s->hbs.p;
  sa.flags = flags_buf ? flags_buf : s->flags.p;
  if (!flags_buf) { // an advance (the adjoint's replay windows bring their own flags and log nothing)
    sa.currently = s->cur_stim.p;
    if (s->log_cap > 0) {
      sa.log_time = s->log_t.p;
      sa.log_fiber = s->log_f.p;
      sa.log_count = s->log_n.p;
      sa.log_capacity = s->log_cap;
    }
  }
  sa.words_per_fiber = words;
  sa.nsub_stride = nsub;
  sa.n_fibers = s->n_fibers;
  if (s->gate_set) {
    if (nsub > 253)
      return fail(s, FDM_ERR_UNSUPPORTED, "onlyComputeIfHasBeenStimulated supports at most 253 Heun substeps per half step");
    if (!gate_buf) {
      const size_t need = (size_t)std::max(s->n_fibers, 1) * 2 * s->step_capacity;
      if (s->gate_start.n < need) {
        FDM_CUDA(cudaStreamSynchronize(s->stream));
        FDM_CUDA(s->gate_start.alloc(need));
        invalidate_graphs(s);
      }
      gate_buf = s->gate_start.p;
    }
    sa.gate_start = gate_buf;
    sa.gate_stride = 2 * s->step_capacity;
  }
  wi->gate_start = sa.gate_start;
  wi->gate_stride = sa.gate_stride;
  FDM_CUDA(launch_schedule(sa, s->steps_d.p, n_steps, s->stream));
  s->launches++;
  return FDM_OK;
}

static int run_window(fdm_solver* s, const SplitStep* host_steps, int n_steps, double dt1, bool store_alg)
{
  if (n_steps == 0 || s->n_fibers == 0)
    return FDM_OK;
  int rc = ensure_coefficients(s, dt1);
  if (rc)
    return rc;
  WindowInfo wi;
  rc = prepare_window(s, host_steps, n_steps, &wi);
  if (rc)
    return rc;
  const int words = wi.words, nsub = wi.nsub;

  const RealKind rk = s->real_bytes == 8 ? REAL_F64 : REAL_F32;
  const MathKind mk = s->cfg.approximate_exponential_function ? MATH_APPROX : MATH_EXACT;
  const bool prof = s->cfg.profile != 0;

  if (s->cfg.method == FDM_METHOD_FUSED) {
    FusedArgs fa{};
    fa.n_bins = s->n_bins;
    fa.bin_fiber_start = s->bin_start_d.p;
    fa.bin_fibers = s->bin_fibers_d.p;
    fa.fiber_offsets = s->off_d.p;
    fa.stride = s->n_nodes;
    fa.vm = s->vm.p;
    fa.states = s->states.p;
    fa.states_lo = s->states_lo.p;
    fa.params = s->params.p;
    fa.coef = s->coef.p;
    fa.clamp_fiber = s->clamp_fiber.p;
    fa.flags = s->flags.p;
    fa.words_per_fiber = words;
    fa.gate = s->gate_set ? s->gate.p : nullptr;
    fa.gate_start = wi.gate_start;
    fa.gate_stride = wi.gate_stride;
    fa.nsub_stride = nsub;
    fa.vstim = s->cfg.value_for_stimulated_point;
    fa.stimulus_mode = s->cfg.stimulus_mode;
    fa.stimulus_parameter = s->cfg.stimulus_parameter;
    fa.stimulus_value = s->cfg.stimulus_value;
    fa.steps = s->steps_d.p;
    fa.n_steps = n_steps;
    fa.store_alg = store_alg && s->n_alg_out > 0;
    fa.n_alg_out = s->n_alg_out;
    fa.alg_indices = s->alg_idx.p;
    fa.alg_out = s->alg_out.p;
    fa.n_nodes = s->n_nodes;
    fa.trace_slot = s->n_trace > 0 ? s->trace_slot.p : nullptr;
    fa.trace = s->trace.p;
    fa.n_trace = s->n_trace;
    fa.trace_capacity = s->trace_capacity;
    fa.act = activation_rec(s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof) {
      e0 = next_event(s);
      e1 = next_event(s);
      FDM_CUDA(cudaEventRecord(e0, s->stream));
    }
    if (s->cluster > 1)
      FDM_CUDA(launch_fused_cluster(s->cfg.model, rk, s->shape, s->cluster, fa, s->stream));
    else
      FDM_CUDA(launch_fused(s->cfg.model, rk, mk, s->shape, fa, s->stream));
    s->launches++;
    if (prof)
      FDM_CUDA(cudaEventRecord(e1, s->stream));
    return FDM_OK;
  }

  ReactionArgs ra{};
  ra.n_nodes = s->n_nodes;
  ra.stride = s->n_nodes;
  ra.vm = s->vm.p;
  ra.states = s->states.p;
  ra.states_lo = s->states_lo.p;
  ra.params = s->params.p;
  ra.clamp_fiber = s->clamp_fiber.p;
  ra.flags = s->flags.p;
  ra.words_per_fiber = words;
  ra.gate = s->gate_set ? s->gate.p : nullptr;
  ra.gate_start = wi.gate_start;
  ra.gate_stride = wi.gate_stride;
  ra.nsub_stride = nsub;
  ra.vstim = s->cfg.value_for_stimulated_point;
  ra.stimulus_mode = s->cfg.stimulus_mode;
  ra.stimulus_parameter = s->cfg.stimulus_parameter;
  ra.stimulus_value = s->cfg.stimulus_value;
  ra.steps = s->steps_d.p;
  ra.n_alg_out = s->n_alg_out;
  ra.alg_indices = s->alg_idx.p;
  ra.alg_out = s->alg_out.p;
  ra.trace_slot = s->n_trace > 0 ? s->trace_slot.p : nullptr;
  ra.trace = s->trace.p;
  ra.n_trace = s->n_trace;
  ra.trace_capacity = s->trace_capacity;
  ra.act = activation_rec(s);
  ra.per_node = s->adj_forward ? 1 : 0;
  if (s->eq.on) {
    // equilibrium skip: every half step is a speculative reaction, the buffer scan and a commit; the statuses
    // alternate between the two status arrays, and a window has an even number of half steps
    auto& E = s->eq;
    const int64_t nt = s->n_nodes + E.n_pad;
    FDM_CUDA(E.alg_a.alloc((size_t)std::max(s->n_alg_out, 1) * std::max<int64_t>(nt, 1)));
    FDM_CUDA(E.alg_b.alloc((size_t)std::max(s->n_alg_out, 1) * std::max<int64_t>(nt, 1)));
    EqLayout L{};
    L.W = s->cfg.vc_width;
    L.n_ranks = s->cfg.n_ranks;
    L.n_nodes = s->n_nodes;
    L.n_pad = E.n_pad;
    L.n_buffers = E.n_buffers;
    L.buf_of = E.buf_of.p;
    L.lane_node = E.lane_node.p;
    L.jfiber = E.jfiber.p;
    L.buf_rank = E.buf_rank.p;
    L.rank_first = E.rank_first.p;
    L.counter = E.counter.p;
    EqSpec e{};
    e.nt = nt;
    e.vm_pad = E.vm_pad.p;
    e.states_pad = E.states_pad.p;
    e.states_lo_pad = E.states_lo_pad.p;
    e.params_pad = E.params_pad.p;
    e.pad_clamp = E.pad_clamp.p;
    e.pad_gate = E.pad_gate.p;
    e.vm_a = E.vm_a.p;
    e.st_a = E.st_a.p;
    e.stl_a = E.stl_a.p;
    e.alg_a = E.alg_a.p;
    e.vm_b = E.vm_b.p;
    e.st_b = E.st_b.p;
    e.stl_b = E.stl_b.p;
    e.alg_b = E.alg_b.p;
    e.ran_b = E.ran_b.p;
    int cur = 0;
    for (int j = 0; j < n_steps; j++) {
      ra.step = j;
      for (int half = 0; half < 2; half++) {
        ra.half = half;
        ra.store_alg = (store_alg && s->n_alg_out > 0 && half == 1 && j == n_steps - 1) ? 1 : 0;
        L.st_in = E.st[cur].p;
        L.st_out = E.st[cur ^ 1].p;
        FDM_CUDA(launch_equilibrium_half(s->cfg.model, rk, mk, ra, L, e, E.info.p, E.prefix.p, E.block_agg.p,
                                         s->model->n_states, half == 1, s->stream));
        s->launches += 6;
        cur ^= 1;
        if (half == 0) {
          FDM_CUDA(launch_diffusion(s->n_fibers, s->off_d.p, s->coef.p, s->n_nodes, s->vm.p, s->scratch.p,
                                         s->stream, E.counter.p, E.nbuf.p, s->cfg.n_ranks));
          s->launches++;
        }
      }
    }
    return FDM_OK;
  }
  // without profiling, a window that stores no algebraics replays a captured CUDA graph of its launches
  const bool graph_ok = s->cfg.use_graph && !prof && !(store_alg && s->n_alg_out > 0);
  if (graph_ok) {
    const auto key = std::make_tuple(n_steps, words, nsub, (const void*)s->flags.p);
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {
      cudaGraph_t g = nullptr;
      FDM_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t ce = cudaSuccess;
      for (int j = 0; j < n_steps && ce == cudaSuccess; j++) {
        ra.step = j;
        for (int half = 0; half < 2 && ce == cudaSuccess; half++) {
          ra.half = half;
          ra.store_alg = 0;
          ce = launch_reaction(s->cfg.model, rk, mk, ra, s->stream);
          if (ce == cudaSuccess && half == 0)
            ce = launch_diffusion(s->n_fibers, s->off_d.p, s->coef.p, s->n_nodes, s->vm.p, s->scratch.p,
                                       s->stream);
        }
      }
      cudaError_t ee = cudaStreamEndCapture(s->stream, &g);
      if (ce != cudaSuccess)
        return cuda_fail(s, ce, "capture of the window launches");
      FDM_CUDA(ee);
      cudaGraphExec_t ex = nullptr;
      cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      FDM_CUDA(ie);
      it = s->graphs.emplace(key, ex).first;
    }
    FDM_CUDA(cudaGraphLaunch(it->second, s->stream));
    s->launches += 3 * (int64_t)n_steps;
    return FDM_OK;
  }
  for (int j = 0; j < n_steps; j++) {
    ra.step = j;
    for (int half = 0; half < 2; half++) {
      ra.half = half;
      ra.store_alg = (store_alg && s->n_alg_out > 0 && half == 1 && j == n_steps - 1) ? 1 : 0;
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (prof) {
        e0 = next_event(s);
        e1 = next_event(s);
        FDM_CUDA(cudaEventRecord(e0, s->stream));
      }
      FDM_CUDA(launch_reaction(s->cfg.model, rk, mk, ra, s->stream));
      s->launches++;
      if (prof)
        FDM_CUDA(cudaEventRecord(e1, s->stream));
      if (half == 0) {
        FDM_CUDA(launch_diffusion(s->n_fibers, s->off_d.p, s->coef.p, s->n_nodes, s->vm.p, s->scratch.p,
                                       s->stream));
        s->launches++;
      }
    }
  }
  return FDM_OK;
}

// The split steps of RepeatedCall<FastMonodomainSolver>::advanceTimeSpan over [t_start, t_end]
// (repeated_call.tpp:43-75, fast_monodomain_solver_compute.tpp:64-129), with the time-step objects'
// state carried from call to call as the reference's scheme objects carry it.
// the RepeatedCall pieces k_begin <= k < k_end (k_end < 0: to the last) of the span [t_start, t_end] as split
// steps (repeated_call.tpp:43-80: piece k starts at start + k/n*span); an advance split into consecutive piece
// ranges gives the same step times as one over the whole span.  piece_steps, when given, receives the number of
// split steps of each planned piece.
static void plan_advance(fdm_solver* s, double t_start, double t_end, std::vector<SplitStep>& steps,
                         std::vector<double>& dt1s, int64_t k_begin = 0, int64_t k_end = -1,
                         int* piece_steps = nullptr)
{
  Tss rc;
  rc.init(t_start, t_end, s->cfg.dt_repeated_call);
  rc.set_dt(s->cfg.dt_repeated_call);
  const double span = rc.end - rc.start;
  if (!s->tss_init) {
    s->strang.init(t_start, t_start + s->cfg.dt_splitting, s->cfg.dt_splitting);
    s->heun.init(t_start, t_start + s->cfg.dt_0d, s->cfg.dt_0d);
    s->diff.init(t_start, t_start + s->cfg.dt_1d, s->cfg.dt_1d);
    s->tss_init = true;
  }
  if (k_end < 0 || k_end > rc.n)
    k_end = rc.n;
  for (int64_t k = k_begin; k < k_end; k++) {
    const double t = k == 0 ? rc.start : rc.start + (double)k / rc.n * span;
    s->strang.set_span(t, t + rc.dt);
    const double start = s->strang.start;
    const double dts = s->strang.dt;
    const int ns = s->strang.n;
    s->heun.set_span(start, start + 0.5 * dts);
    s->diff.set_span(start, start + dts);
    for (int j = 0; j < ns; j++) {
      SplitStep st;
      const double tc = start + j * dts;
      st.t = tc;
      st.mid = tc + 0.5 * dts;
      st.dt0 = s->heun.dt;
      st.n0 = s->heun.n;
      st.global_no = (int)std::min<int64_t>(std::max<int64_t>(s->split_no - s->trace_base, 0), 2147483647);
      s->split_no++;
      steps.push_back(st);
      dt1s.push_back(s->diff.dt);
    }
    if (piece_steps)
      piece_steps[k - k_begin] = ns;
  }
}

static int64_t repeated_call_pieces(const fdm_solver* s, double t_start, double t_end)
{
  Tss rc;
  rc.init(t_start, t_end, s->cfg.dt_repeated_call);
  rc.set_dt(s->cfg.dt_repeated_call);
  return rc.n;
}

// runs planned steps in windows of at most steps_per_launch steps that share the diffusion step width
static int run_planned(fdm_solver* s, const std::vector<SplitStep>& steps, const std::vector<double>& dt1s,
                       size_t begin, size_t end, bool store_at_end)
{
  const int K = s->cfg.steps_per_launch;
  size_t w0 = begin;
  while (w0 < end) {
    size_t w1 = w0 + 1;
    while (w1 < end && (int)(w1 - w0) < K && std::fabs(dt1s[w1] - dt1s[w0]) <= 1e-12 * std::fabs(dt1s[w0]))
      w1++;
    int r = run_window(s, steps.data() + w0, (int)(w1 - w0), dt1s[w0], store_at_end && w1 == end);
    if (r)
      return r;
    w0 = w1;
  }
  return FDM_OK;
}

// the end of an advance's device work: its stop event and the count of non-finite Vm values, enqueued behind it
static int enqueue_finish(fdm_solver* s)
{
  FDM_CUDA(cudaEventRecord(s->adv_stop, s->stream));
  if (s->cfg.check_nan && s->n_nodes > 0) {
    FDM_CUDA(cudaMemsetAsync(s->nonfinite.p, 0, sizeof(int), s->stream));
    FDM_CUDA(launch_count_nonfinite(s->vm.p, s->n_nodes, s->nonfinite.p, s->stream));
  }
  return FDM_OK;
}

// waits for the advance's device work, then adds up its timing and reads the non-finite count
static int complete_finish(fdm_solver* s)
{
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  float ms = 0;
  FDM_CUDA(cudaEventElapsedTime(&ms, s->adv_start, s->adv_stop));
  s->adv_ms += ms;
  for (size_t i = 0; i + 1 < s->ev_used; i += 2) {
    float m2 = 0;
    FDM_CUDA(cudaEventElapsedTime(&m2, s->ev_pool[i], s->ev_pool[i + 1]));
    s->main_ms += m2;
    s->main_launches++;
  }
  if (s->cfg.check_nan && s->n_nodes > 0) {
    int bad = 0;
    FDM_CUDA(cudaMemcpy(&bad, s->nonfinite.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (bad)
      return fail(s, FDM_ERR_NAN, "fdm_advance: " + std::to_string(bad) + " non-finite Vm values");
  }
  return FDM_OK;
}

static int finish_advance(fdm_solver* s)
{
  const int r = enqueue_finish(s);
  return r ? r : complete_finish(s);
}

extern "C" int fdm_wait(fdm_solver* s)
{
  if (!s)
    return fail(s, FDM_ERR_ARG, "fdm_wait: null solver");
  if (!s->finish_pending)
    return FDM_OK;
  FDM_BIND(s);
  s->finish_pending = false;
  return complete_finish(s);
}

extern "C" int fdm_wait_for(fdm_solver* s, double timeout_seconds)
{
  if (!s || !(timeout_seconds >= 0))
    return fail(s, FDM_ERR_ARG, "fdm_wait_for: bad argument");
  if (!s->finish_pending)
    return FDM_OK;
  FDM_BIND(s);
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t q = cudaStreamQuery(s->stream);
    if (q == cudaSuccess)
      break;
    if (q != cudaErrorNotReady) {
      s->finish_pending = false;
      return cuda_fail(s, q, "fdm_wait_for");
    }
    const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (waited >= timeout_seconds)
      return fail(s, FDM_ERR_TIMEOUT, "fdm_wait_for: the advance is still running after " +
                                          std::to_string(waited) + " s; it stays enqueued (fdm_wait completes it)");
    std::this_thread::sleep_for(std::chrono::microseconds(waited < 1e-3 ? 20 : 200));
  }
  return fdm_wait(s);
}

// the work of an advance, enqueued on the solver's stream (the host waits only where the window buffers of
// the step schedule are reused)
static int enqueue_advance(fdm_solver* s, double t_start, double t_end, const char* who, int64_t k_begin = 0,
                           int64_t k_end = -1)
{
  if (!s)
    return fail(s, FDM_ERR_ARG, std::string(who) + ": null solver");
  FDM_BIND(s);
  if (!(t_end >= t_start))
    return fail(s, FDM_ERR_ARG, std::string(who) + ": t_end must be >= t_start");
  if (s->n_fibers > 0 && !s->stimulation_set)
    return fail(s, FDM_ERR_ARG, std::string(who) + ": call fdm_set_stimulation first");
  int r = fdm_wait(s);     // the timing and the NaN check of an earlier asynchronous advance
  if (r)
    return r;
  s->ev_used = 0;
  FDM_CUDA(cudaEventRecord(s->adv_start, s->stream));
  std::vector<SplitStep> steps;
  std::vector<double> dt1s;
  plan_advance(s, t_start, t_end, steps, dt1s, k_begin, k_end);
  return run_planned(s, steps, dt1s, 0, steps.size(), true);
}

extern "C" int fdm_advance(fdm_solver* s, double t_start, double t_end)
{
  const int r = enqueue_advance(s, t_start, t_end, "fdm_advance");
  if (r)
    return r;
  return finish_advance(s);
}

extern "C" int fdm_advance_async(fdm_solver* s, double t_start, double t_end)
{
  int r = enqueue_advance(s, t_start, t_end, "fdm_advance_async");
  if (r)
    return r;
  r = enqueue_finish(s);
  if (r)
    return r;
  s->finish_pending = true;
  return FDM_OK;
}

// Strang steps given explicitly, as the reference's generated computeMonodomain receives them
// (fast_monodomain_solver_gpu.tpp:478-481, 505-515): currentTime = startTime + j*dtSplit, substeps at
// currentTime + k*dt0D and midTime + k*dt0D, one diffusion solve with dt1D per step.
static int advance_explicit(fdm_solver* s, double start, double dts, int ns, double dt0, int n0, double dt1)
{
  { // an asynchronous advance still owes its timing and NaN check
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  s->ev_used = 0;
  FDM_CUDA(cudaEventRecord(s->adv_start, s->stream));
  std::vector<SplitStep> steps(ns);
  std::vector<double> dt1s(ns, dt1);
  for (int j = 0; j < ns; j++) {
    const double tc = start + j * dts;
    steps[j].t = tc;
    steps[j].mid = tc + 0.5 * dts;
    steps[j].dt0 = dt0;
    steps[j].n0 = n0;
    steps[j].global_no = (int)std::min<int64_t>(std::max<int64_t>(s->split_no - s->trace_base, 0), 2147483647);
    s->split_no++;
  }
  int r = run_planned(s, steps, dt1s, 0, steps.size(), true);
  if (r)
    return r;
  return finish_advance(s);
}

extern "C" int fdm_repeated_call_plan(fdm_solver* s, double t_start, double t_end, int64_t* n_pieces,
                                      int* steps_per_piece)
{
  if (!s || !n_pieces || !(t_end >= t_start))
    return fail(s, FDM_ERR_ARG, "fdm_repeated_call_plan: bad argument");
  *n_pieces = repeated_call_pieces(s, t_start, t_end);
  if (steps_per_piece) { // a dry run of the plan: the time-stepping state is put back
    const Tss strang = s->strang, heun = s->heun, diff = s->diff;
    const bool tss_init = s->tss_init;
    const int64_t split_no = s->split_no;
    std::vector<SplitStep> steps;
    std::vector<double> dt1s;
    plan_advance(s, t_start, t_end, steps, dt1s, 0, -1, steps_per_piece);
    s->strang = strang;
    s->heun = heun;
    s->diff = diff;
    s->tss_init = tss_init;
    s->split_no = split_no;
  }
  return FDM_OK;
}

extern "C" int fdm_advance_pieces(fdm_solver* s, double t_start, double t_end, int64_t k_begin, int64_t k_end)
{
  if (!s)
    return fail(s, FDM_ERR_ARG, "fdm_advance_pieces: null solver");
  if (!(t_end >= t_start) || k_begin < 0 || k_end < k_begin || k_end > repeated_call_pieces(s, t_start, t_end))
    return fail(s, FDM_ERR_ARG, "fdm_advance_pieces: need 0 <= k_begin <= k_end <= the number of pieces");
  const int r = enqueue_advance(s, t_start, t_end, "fdm_advance_pieces", k_begin, k_end);
  if (r)
    return r;
  return finish_advance(s);
}

extern "C" int64_t fdm_split_steps(const fdm_solver* s) { return s ? s->split_no : 0; }

extern "C" int fdm_debug_fail_allocation(int64_t k)
{
  if (k < 0)
    return fail(nullptr, FDM_ERR_ARG, "fdm_debug_fail_allocation: k must be >= 0");
  g_fail_countdown.store(k);
  return FDM_OK;
}


extern "C" int fdm_set_stimulation_log(fdm_solver* s, int64_t capacity)
{
  if (!s || capacity < 0)
    return fail(s, FDM_ERR_ARG, "fdm_set_stimulation_log: bad argument");
  FDM_BIND(s);
  {
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  if (capacity == 0) {
    s->log_t.release();
    s->log_f.release();
    s->log_n.release();
    s->log_cap = 0;
    s->log_dropped = 0;
    return FDM_OK;
  }
  if (s->log_cap == 0) {
    FDM_CUDA(s->log_n.alloc(1));
    FDM_CUDA(cudaMemsetAsync(s->log_n.p, 0, sizeof(unsigned long long), s->stream));
  }
  if (capacity > s->log_cap) { // grow, keeping the entries recorded so far
    DevBuf<double> t;
    DevBuf<int> f;
    cudaError_t e = t.alloc((size_t)capacity);
    if (e == cudaSuccess)
      e = f.alloc((size_t)capacity);
    if (e == cudaSuccess && s->log_cap > 0) {
      e = cudaMemcpyAsync(t.p, s->log_t.p, sizeof(double) * s->log_cap, cudaMemcpyDeviceToDevice, s->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(f.p, s->log_f.p, sizeof(int) * s->log_cap, cudaMemcpyDeviceToDevice, s->stream);
    }
    // the counter may have run past the old capacity (those begins were counted, not stored): the new
    // entries must follow the stored ones, so the counter restarts at the stored count and the excess is
    // kept aside, where fdm_get_stimulation_log reports it
    unsigned long long n = 0;
    if (e == cudaSuccess && s->log_cap > 0)
      e = cudaMemcpyAsync(&n, s->log_n.p, sizeof(n), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess && n > (unsigned long long)s->log_cap) {
      const unsigned long long stored = (unsigned long long)s->log_cap;
      e = cudaMemcpyAsync(s->log_n.p, &stored, sizeof(stored), cudaMemcpyHostToDevice, s->stream);
      if (e == cudaSuccess)
        e = cudaStreamSynchronize(s->stream);
      if (e == cudaSuccess)
        s->log_dropped += (int64_t)(n - stored);
    }
    if (e != cudaSuccess) { // the log stays as it was
      t.release();
      f.release();
      return cuda_fail(s, e, "fdm_set_stimulation_log");
    }
    s->log_t.release();
    s->log_f.release();
    s->log_t = t;
    s->log_f = f;
    t.p = nullptr;
    f.p = nullptr;
    s->log_cap = capacity;
  }
  return FDM_OK;
}

extern "C" int fdm_get_stimulation_log(fdm_solver* s, int64_t* n_total, double* times, int* fibers)
{
  if (!s || !n_total)
    return fail(s, FDM_ERR_ARG, "fdm_get_stimulation_log: bad argument");
  FDM_BIND(s);
  {
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  *n_total = 0;
  if (s->log_cap == 0)
    return FDM_OK;
  unsigned long long n = 0;
  FDM_CUDA(cudaMemcpyAsync(&n, s->log_n.p, sizeof(n), cudaMemcpyDeviceToHost, s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  *n_total = (int64_t)n + s->log_dropped;
  if (!times && !fibers)
    return FDM_OK;
  if (s->log_dropped > 0 || *n_total > s->log_cap)
    return fail(s, FDM_ERR_ARG, "fdm_get_stimulation_log: " + std::to_string(*n_total) +
                                    " stimulation begins were recorded but the log kept only " +
                                    std::to_string(std::min<int64_t>(*n_total - s->log_dropped, s->log_cap)) +
                                    "; the log is incomplete (grow its capacity before each advance)");
  const size_t k = (size_t)n;
  if (k > 0 && times)
    FDM_CUDA(cudaMemcpyAsync(times, s->log_t.p, sizeof(double) * k, cudaMemcpyDeviceToHost, s->stream));
  if (k > 0 && fibers)
    FDM_CUDA(cudaMemcpyAsync(fibers, s->log_f.p, sizeof(int) * k, cudaMemcpyDeviceToHost, s->stream));
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  return FDM_OK;
}

extern "C" int fdm_get_timing(const fdm_solver* s, double* main_ms, int64_t* main_launches, double* adv_ms,
                              int64_t* launches)
{
  if (!s)
    return FDM_ERR_ARG;
  if (main_ms)
    *main_ms = s->main_ms;
  if (main_launches)
    *main_launches = s->main_launches;
  if (adv_ms)
    *adv_ms = s->adv_ms;
  if (launches)
    *launches = s->launches;
  return FDM_OK;
}

extern "C" int fdm_reset_timing(fdm_solver* s)
{
  if (!s)
    return FDM_ERR_ARG;
  s->main_ms = s->adv_ms = s->adj_ms = 0;
  s->main_launches = s->launches = 0;
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// checkpoint (saveFiberDataCheckpoint / restoreFiberDataCheckpoint): device-to-device snapshot
// ---------------------------------------------------------------------------------------------
extern "C" int fdm_checkpoint_save(fdm_solver* s)
{
  if (!s)
    return FDM_ERR_ARG;
  FDM_BIND(s);
  const int64_t N = s->n_nodes;
  const int NS = s->model->n_states;
  const int nf = s->n_fibers;
  s->ck_valid = false;   // until the snapshot below is complete
  s->eq.ck_valid = false;
  FDM_CUDA(s->ck_vm.alloc(std::max<int64_t>(N, 1)));
  FDM_CUDA(s->ck_states.alloc((size_t)std::max<int64_t>(N, 1) * std::max(NS - 1, 1) * s->real_bytes));
  FDM_CUDA(s->ck_last.alloc(std::max(nf, 1)));
  FDM_CUDA(s->ck_jit.alloc(std::max(nf, 1)));
  FDM_CUDA(s->ck_jidx.alloc(std::max(nf, 1)));
  FDM_CUDA(s->ck_hbs.alloc(std::max(nf, 1)));
  FDM_CUDA(s->ck_cur.alloc(std::max(nf, 1)));
  if (N > 0) {
    FDM_CUDA(cudaMemcpyAsync(s->ck_vm.p, s->vm.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream));
    if (NS > 1)
      FDM_CUDA(cudaMemcpyAsync(s->ck_states.p, s->states.p, (size_t)N * (NS - 1) * s->real_bytes,
                               cudaMemcpyDeviceToDevice, s->stream));
    if (NS > 1 && s->real_bytes == 4) {
      FDM_CUDA(s->ck_states_lo.alloc((size_t)N * (NS - 1) * 4));
      FDM_CUDA(cudaMemcpyAsync(s->ck_states_lo.p, s->states_lo.p, (size_t)N * (NS - 1) * 4,
                               cudaMemcpyDeviceToDevice, s->stream));
    }
  }
  if (nf > 0 && s->stimulation_set) {
    FDM_CUDA(cudaMemcpyAsync(s->ck_last.p, s->last_check.p, sizeof(double) * nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->ck_jit.p, s->cur_jitter.p, sizeof(double) * nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->ck_jidx.p, s->jitter_idx.p, sizeof(int) * nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->ck_hbs.p, s->hbs.p, nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->ck_cur.p, s->cur_stim.p, nf, cudaMemcpyDeviceToDevice, s->stream));
  }
  if (s->eq.on) {
    auto& E = s->eq;
    const size_t nsb = (size_t)std::max(NS - 1, 1) * std::max(E.n_pad, 1) * s->real_bytes;
    FDM_CUDA(E.ck_st.alloc(std::max<int64_t>(E.n_buffers, 1)));
    FDM_CUDA(E.ck_counter.alloc(s->cfg.n_ranks));
    FDM_CUDA(E.ck_vm_pad.alloc(std::max(E.n_pad, 1)));
    FDM_CUDA(E.ck_states_pad.alloc(nsb));
    FDM_CUDA(E.ck_states_lo_pad.alloc(nsb));
    FDM_CUDA(cudaMemcpyAsync(E.ck_st.p, E.st[0].p, std::max<int64_t>(E.n_buffers, 1), cudaMemcpyDeviceToDevice,
                             s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.ck_counter.p, E.counter.p, sizeof(int) * s->cfg.n_ranks, cudaMemcpyDeviceToDevice,
                             s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.ck_vm_pad.p, E.vm_pad.p, sizeof(double) * std::max(E.n_pad, 1),
                             cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.ck_states_pad.p, E.states_pad.p, nsb, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.ck_states_lo_pad.p, E.states_lo_pad.p, nsb, cudaMemcpyDeviceToDevice, s->stream));
    E.ck_valid = true;
  }
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->ck_strang = s->strang;
  s->ck_heun = s->heun;
  s->ck_diff = s->diff;
  s->ck_tss_init = s->tss_init;
  s->ck_split = s->split_no;
  s->ck_valid = true;
  return FDM_OK;
}

extern "C" int fdm_checkpoint_restore(fdm_solver* s)
{
  if (!s || !s->ck_valid)
    return fail(s, FDM_ERR_ARG, "fdm_checkpoint_restore: no checkpoint saved");
  FDM_BIND(s);
  const int64_t N = s->n_nodes;
  const int NS = s->model->n_states;
  const int nf = s->n_fibers;
  if (N > 0) {
    FDM_CUDA(cudaMemcpyAsync(s->vm.p, s->ck_vm.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s->stream));
    if (NS > 1)
      FDM_CUDA(cudaMemcpyAsync(s->states.p, s->ck_states.p, (size_t)N * (NS - 1) * s->real_bytes,
                               cudaMemcpyDeviceToDevice, s->stream));
    if (NS > 1 && s->real_bytes == 4)
      FDM_CUDA(cudaMemcpyAsync(s->states_lo.p, s->ck_states_lo.p, (size_t)N * (NS - 1) * 4,
                               cudaMemcpyDeviceToDevice, s->stream));
  }
  if (nf > 0 && s->stimulation_set) {
    FDM_CUDA(cudaMemcpyAsync(s->last_check.p, s->ck_last.p, sizeof(double) * nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->cur_jitter.p, s->ck_jit.p, sizeof(double) * nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->jitter_idx.p, s->ck_jidx.p, sizeof(int) * nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->hbs.p, s->ck_hbs.p, nf, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->cur_stim.p, s->ck_cur.p, nf, cudaMemcpyDeviceToDevice, s->stream));
  }
  if (s->eq.on && s->eq.ck_valid) {
    auto& E = s->eq;
    const size_t nsb = (size_t)std::max(NS - 1, 1) * std::max(E.n_pad, 1) * s->real_bytes;
    FDM_CUDA(cudaMemcpyAsync(E.st[0].p, E.ck_st.p, std::max<int64_t>(E.n_buffers, 1), cudaMemcpyDeviceToDevice,
                             s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.counter.p, E.ck_counter.p, sizeof(int) * s->cfg.n_ranks, cudaMemcpyDeviceToDevice,
                             s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.vm_pad.p, E.ck_vm_pad.p, sizeof(double) * std::max(E.n_pad, 1),
                             cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.states_pad.p, E.ck_states_pad.p, nsb, cudaMemcpyDeviceToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(E.states_lo_pad.p, E.ck_states_lo_pad.p, nsb, cudaMemcpyDeviceToDevice, s->stream));
  }
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  s->strang = s->ck_strang;
  s->heun = s->ck_heun;
  s->diff = s->ck_diff;
  s->tss_init = s->ck_tss_init;
  s->split_no = s->ck_split;
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// compute1D as a standalone operator on device arrays
// ---------------------------------------------------------------------------------------------
#include <mutex>

namespace {
struct ScratchPool {
  std::mutex mu;
  double* p[64] = {};
  size_t n[64] = {};
};
ScratchPool g_scratch;
} // namespace

extern "C" int fdm_diffusion_solve(int n_fibers, int64_t n_nodes, const int64_t* d_fiber_offsets,
                                   const double* d_element_lengths, const double* d_prefactor, double dt,
                                   int diffusion_scheme, double* d_vm, void* stream)
{
  fdm_solver* s = nullptr;
  if (n_fibers < 0 || n_nodes < 0 || (n_fibers > 0 && (!d_fiber_offsets || !d_element_lengths || !d_prefactor || !d_vm)))
    return fail(s, FDM_ERR_ARG, "fdm_diffusion_solve: bad argument");
  if (!(dt > 0) || (diffusion_scheme != FDM_IMPLICIT_EULER && diffusion_scheme != FDM_CRANK_NICOLSON))
    return fail(s, FDM_ERR_ARG, "fdm_diffusion_solve: dt must be positive and the scheme IE or CN");
  if (n_fibers == 0)
    return FDM_OK;
  int dev = 0;
  FDM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64)
    return fail(s, FDM_ERR_ARG, "fdm_diffusion_solve: device ordinal beyond 63");
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lock(g_scratch.mu);
  // scratch: 6 factorization doubles + 1 forward-sweep double per node, allocated by the library
  const size_t need = (size_t)7 * (size_t)n_nodes;
  if (g_scratch.n[dev] < need) {
    if (g_scratch.p[dev])
      FDM_CUDA(cudaFree(g_scratch.p[dev]));
    g_scratch.p[dev] = nullptr;
    g_scratch.n[dev] = 0;
    FDM_CUDA(cudaMalloc((void**)&g_scratch.p[dev], need * sizeof(double)));
    g_scratch.n[dev] = need;
  }
  double* coef = g_scratch.p[dev];
  double* fwd = coef + 6 * (size_t)n_nodes;
  FDM_CUDA(launch_coefficients(n_fibers, d_fiber_offsets, d_element_lengths, d_prefactor, dt,
                               diffusion_scheme == FDM_IMPLICIT_EULER, coef, n_nodes, st));
  FDM_CUDA(launch_diffusion(n_fibers, d_fiber_offsets, coef, n_nodes, d_vm, fwd, st));
  FDM_CUDA(cudaStreamSynchronize(st));
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// compatibility export of the reference's generated-library ABI
// (fast_monodomain_solver_gpu.tpp:361-365 initializeArrays, :478-481 computeMonodomain)
// ---------------------------------------------------------------------------------------------
namespace {
struct Compat {
  fdm_solver* s = nullptr;
  int n_fibers = 0, n_per_fiber = 0, n_params = 0, rows = 0, cols = 0, n_jitter = 0;
  int n_alg = 0, n_states_tr = 0;
  std::vector<int> alg_idx, state_idx;
  std::vector<float> last_params, last_lengths;
  double last_prefactor = -1;
  bool initialized = false;
};
Compat g_compat;
std::mutex g_compat_mu;
} // namespace

// ---------------------------------------------------------------------------------------------
// the CellmlAdapter's generic right-hand side (04_generator_gpu.cpp:13-113)
// ---------------------------------------------------------------------------------------------
extern "C" int fdm_cellml_rhs_device(int model, int approximate_exponential_function, int64_t n_instances, double t,
                                     const double* states, const double* parameters, double* rates,
                                     double* algebraics, void* stream)
{
  const ModelDesc* m = model_desc(model);
  if (!m || n_instances < 0 || (n_instances > 0 && (!states || !rates || (m->n_parameters > 0 && !parameters))))
    return fail(nullptr, FDM_ERR_ARG, "fdm_cellml_rhs_device: bad argument");
  const cudaError_t e = launch_cellml_rhs(model, approximate_exponential_function ? MATH_APPROX : MATH_EXACT,
                                          n_instances, t, states, parameters, rates, algebraics,
                                          (cudaStream_t)stream);
  if (e != cudaSuccess)
    return fail(nullptr, FDM_ERR_CUDA, std::string("fdm_cellml_rhs_device: ") + cudaGetErrorString(e));
  return FDM_OK;
}

extern "C" int fdm_model_equilibrium(int model, int device, int approximate_exponential_function,
                                     const double* parameters, double dt, double* states, int64_t* iterations,
                                     double* max_increment, double* dt_final)
{
  const ModelDesc* m = model_desc(model);
  if (!m || !states || !(dt > 0) || (m->n_parameters > 0 && !parameters))
    return fail(nullptr, FDM_ERR_ARG, "fdm_model_equilibrium: bad argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, FDM_ERR_NO_DEVICE, "fdm_model_equilibrium: no CUDA device");
  if (device < 0 || device >= ndev)
    return fail(nullptr, FDM_ERR_ARG, "fdm_model_equilibrium: device ordinal out of range");
  if (cudaSetDevice(device) != cudaSuccess)
    return fail(nullptr, FDM_ERR_CUDA, "fdm_model_equilibrium: cudaSetDevice failed");
  const int NS = m->n_states, NP = std::max(m->n_parameters, 1);
  // 03_cellml_adapter.tpp:469: at most 1e7 RK4 steps, here in launches of bounded length
  const int64_t limit = 10000000, chunk = NS <= 8 ? 100000 : 5000;
  DevBuf<double> u, u0, P;
  DevBuf<EquilibriumSearch> es;
  cudaStream_t st = nullptr;
  std::string err;
  auto run = [&]() -> cudaError_t {
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess || (e = u.alloc(NS)) ||
        (e = u0.alloc(NS)) || (e = P.alloc(NP)) || (e = es.alloc(1)))
      return e;
    EquilibriumSearch h{dt, 0.0, 0, 0, 0};
    if ((e = cudaMemcpyAsync(u.p, states, sizeof(double) * NS, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(u0.p, states, sizeof(double) * NS, cudaMemcpyHostToDevice, st)) ||
        (m->n_parameters > 0 &&
         (e = cudaMemcpyAsync(P.p, parameters, sizeof(double) * m->n_parameters, cudaMemcpyHostToDevice, st))) ||
        (e = cudaMemcpyAsync(es.p, &h, sizeof(h), cudaMemcpyHostToDevice, st)))
      return e;
    for (int64_t done = 0; done < limit && !h.done; done += chunk) {
      if ((e = launch_equilibrium_search(model, approximate_exponential_function ? MATH_APPROX : MATH_EXACT, u.p,
                                         u0.p, P.p, es.p, std::min(chunk, limit - done), st)) ||
          (e = cudaMemcpyAsync(&h, es.p, sizeof(h), cudaMemcpyDeviceToHost, st)) || (e = cudaStreamSynchronize(st)))
        return e;
    }
    if ((e = cudaMemcpyAsync(states, u.p, sizeof(double) * NS, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
      return e;
    if (iterations)
      *iterations = h.iterations;
    if (max_increment)
      *max_increment = h.max_increment;
    if (dt_final)
      *dt_final = h.dt;
    return cudaSuccess;
  };
  const cudaError_t e = run();
  u.release();
  u0.release();
  P.release();
  es.release();
  if (st)
    cudaStreamDestroy(st);
  if (e != cudaSuccess)
    return fail(nullptr, FDM_ERR_CUDA, std::string("fdm_model_equilibrium: ") + cudaGetErrorString(e));
  return FDM_OK;
}

namespace {
struct CellmlRhs {
  int model = -1, approx = 0, device = 0;
  int64_t n = 0;
  double *states = nullptr, *params = nullptr, *rates = nullptr, *alg = nullptr;
  cudaStream_t stream = nullptr;
  void release()
  {
    for (double* p : {states, params, rates, alg})
      if (p)
        cudaFree(p);
    states = params = rates = alg = nullptr;
    if (stream)
      cudaStreamDestroy(stream);
    stream = nullptr;
    model = -1;
  }
};
CellmlRhs g_rhs;
std::mutex g_rhs_mu;
} // namespace

extern "C" int fdm_cellml_rhs_configure(int model, int64_t n_instances, int approximate_exponential_function,
                                        int device)
{
  std::lock_guard<std::mutex> lock(g_rhs_mu);
  const ModelDesc* m = model_desc(model);
  if (!m || n_instances < 0)
    return fail(nullptr, FDM_ERR_ARG, "fdm_cellml_rhs_configure: bad argument");
  if (cudaSetDevice(device) != cudaSuccess)
    return fail(nullptr, FDM_ERR_NO_DEVICE, "fdm_cellml_rhs_configure: no such CUDA device");
  g_rhs.release();
  const size_t n = (size_t)std::max<int64_t>(n_instances, 1);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&g_rhs.states, sizeof(double) * n * m->n_states);
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&g_rhs.params, sizeof(double) * n * std::max(m->n_parameters, 1));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&g_rhs.rates, sizeof(double) * n * m->n_states);
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&g_rhs.alg, sizeof(double) * n * std::max(m->n_algebraics, 1));
  if (e == cudaSuccess)
    e = cudaStreamCreateWithFlags(&g_rhs.stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    g_rhs.release();
    return fail(nullptr, FDM_ERR_CUDA, std::string("fdm_cellml_rhs_configure: ") + cudaGetErrorString(e));
  }
  g_rhs.model = model;
  g_rhs.n = n_instances;
  g_rhs.approx = approximate_exponential_function;
  g_rhs.device = device;
  return FDM_OK;
}

// host arrays in and out, as the reference's OpenMP-offload code maps them (map(to: states, parameters)
// map(from: rates, algebraics)); a failure is reported through fdm_last_error(NULL) and leaves rates untouched
extern "C" void computeCellMLRightHandSide(void* context, double t, double* states, double* rates, double* algebraics,
                                           double* parameters)
{
  (void)context;
  std::lock_guard<std::mutex> lock(g_rhs_mu);
  if (g_rhs.model < 0 || !states || !rates) {
    fail(nullptr, FDM_ERR_ARG, "computeCellMLRightHandSide: call fdm_cellml_rhs_configure first");
    return;
  }
  const ModelDesc* m = model_desc(g_rhs.model);
  const int64_t n = g_rhs.n;
  cudaSetDevice(g_rhs.device);
  cudaStream_t st = g_rhs.stream;
  cudaError_t e = cudaMemcpyAsync(g_rhs.states, states, sizeof(double) * n * m->n_states, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && m->n_parameters > 0 && parameters)
    e = cudaMemcpyAsync(g_rhs.params, parameters, sizeof(double) * n * m->n_parameters, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = launch_cellml_rhs(g_rhs.model, g_rhs.approx ? MATH_APPROX : MATH_EXACT, n, t, g_rhs.states, g_rhs.params,
                          g_rhs.rates, algebraics ? g_rhs.alg : nullptr, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rates, g_rhs.rates, sizeof(double) * n * m->n_states, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && algebraics && m->n_algebraics > 0)
    e = cudaMemcpyAsync(algebraics, g_rhs.alg, sizeof(double) * n * m->n_algebraics, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    fail(nullptr, FDM_ERR_CUDA, std::string("computeCellMLRightHandSide: ") + cudaGetErrorString(e));
}

extern "C" int fdm_compat_configure(int model, int n_fibers, int n_instances_per_fiber, int n_parameters_per_instance,
                                    int firing_rows, int firing_cols, int n_jitter_per_fiber,
                                    int n_algebraics_for_transfer, int n_states_for_transfer, int diffusion_scheme,
                                    int approximate_exponential_function, int reaction_precision, int method)
{
  std::lock_guard<std::mutex> lock(g_compat_mu);
  const ModelDesc* m = model_desc(model);
  if (!m || n_fibers < 1 || n_instances_per_fiber < 2 || n_parameters_per_instance < 0 ||
      n_parameters_per_instance > m->n_parameters || firing_rows < 1 || firing_cols < 1 || n_jitter_per_fiber < 0 ||
      n_algebraics_for_transfer < 0 || n_states_for_transfer < 1)
    return fail(nullptr, FDM_ERR_ARG, "fdm_compat_configure: bad sizes");
  if (g_compat.s) {
    fdm_destroy(g_compat.s);
    g_compat.s = nullptr;
  }
  fdm_config c;
  fdm_config_default(&c);
  c.model = model;
  c.diffusion_scheme = diffusion_scheme;
  c.approximate_exponential_function = approximate_exponential_function;
  c.reaction_precision = reaction_precision;
  c.method = method;
  c.clamp_rule = FDM_CLAMP_CENTER; // the clamp set of the reference's GPU code
  fdm_solver* s = nullptr;
  int rc = fdm_create(&c, &s);
  if (rc)
    return rc;
  g_compat = Compat();
  g_compat.s = s;
  g_compat.n_fibers = n_fibers;
  g_compat.n_per_fiber = n_instances_per_fiber;
  g_compat.n_params = n_parameters_per_instance;
  g_compat.rows = firing_rows;
  g_compat.cols = firing_cols;
  g_compat.n_jitter = n_jitter_per_fiber;
  g_compat.n_alg = n_algebraics_for_transfer;
  g_compat.n_states_tr = n_states_for_transfer;
  // fibers of equal length and unit element length until computeMonodomain passes the real lengths
  std::vector<int64_t> off(n_fibers + 1);
  for (int f = 0; f <= n_fibers; f++)
    off[f] = (int64_t)f * n_instances_per_fiber;
  std::vector<double> h((size_t)n_fibers * (n_instances_per_fiber - 1), 1.0), pf(n_fibers, 1.0);
  return fdm_set_fibers(s, n_fibers, off.data(), h.data(), pf.data());
}

extern "C" void initializeArrays(const double* statesOneInstance, const int* algebraicsForTransferIndices,
                                 const int* statesForTransferIndices, const char* firingEvents,
                                 const double* setSpecificStatesFrequencyJitter, const int* motorUnitNo,
                                 const int* fiberStimulationPointIndex, const double* lastStimulationCheckTime,
                                 const double* setSpecificStatesCallFrequency,
                                 const double* setSpecificStatesRepeatAfterFirstCall,
                                 const double* setSpecificStatesCallEnableBegin)
{
  std::lock_guard<std::mutex> lock(g_compat_mu);
  Compat& g = g_compat;
  fdm_solver* s = g.s;
  if (!s) {
    fail(nullptr, FDM_ERR_ARG, "initializeArrays: call fdm_compat_configure first");
    return;
  }
  const int NS = s->model->n_states;
  const int64_t N = s->n_nodes;
  std::vector<double> st((size_t)NS * N);
  for (int k = 0; k < NS; k++)
    std::fill(st.begin() + (size_t)k * N, st.begin() + (size_t)(k + 1) * N, statesOneInstance[k]);
  if (fdm_set_states(s, st.data()))
    return;
  g.alg_idx.assign(algebraicsForTransferIndices, algebraicsForTransferIndices + g.n_alg);
  g.state_idx.assign(statesForTransferIndices, statesForTransferIndices + g.n_states_tr);
  if (fdm_set_algebraics_for_transfer(s, g.n_alg, g.alg_idx.data()))
    return;
  std::vector<uint8_t> fe((size_t)g.rows * g.cols);
  for (size_t i = 0; i < fe.size(); i++)
    fe[i] = firingEvents[i] ? 1 : 0;
  if (fdm_set_stimulation(s, fe.data(), g.rows, g.cols, motorUnitNo, fiberStimulationPointIndex,
                          setSpecificStatesCallFrequency, setSpecificStatesRepeatAfterFirstCall,
                          setSpecificStatesCallEnableBegin, setSpecificStatesFrequencyJitter, g.n_jitter))
    return;
  // the caller's initial check times replace the default ones (initialization.tpp:344 computes the same)
  if (cudaSetDevice(s->cfg.device) != cudaSuccess)
    return;
  cudaMemcpy(s->last_check.p, lastStimulationCheckTime, sizeof(double) * g.n_fibers, cudaMemcpyHostToDevice);
  g.last_params.clear();
  g.last_lengths.clear();
  g.last_prefactor = -1;
  g.initialized = true;
}

extern "C" void computeMonodomain(const float* parameters, double* algebraicsForTransfer, double* statesForTransfer,
                                  const float* elementLengths, double startTime, double timeStepWidthSplitting,
                                  int nTimeStepsSplitting, double dt0D, int nTimeSteps0D, double dt1D,
                                  int nTimeSteps1D, double prefactor, double valueForStimulatedPoint)
{
  (void)nTimeSteps1D; // the reference solves once per split step with dt1D (gpu.tpp:622, compute.tpp:284)
  std::lock_guard<std::mutex> lock(g_compat_mu);
  Compat& g = g_compat;
  fdm_solver* s = g.s;
  if (!s || !g.initialized) {
    fail(nullptr, FDM_ERR_ARG, "computeMonodomain: call fdm_compat_configure and initializeArrays first");
    return;
  }
  if (cudaSetDevice(s->cfg.device) != cudaSuccess)
    return;
  const int64_t N = s->n_nodes;
  const int NP = s->model->n_parameters;
  // element lengths and prefactor (re-sent by the reference at every call)
  const size_t ne = (size_t)g.n_fibers * (g.n_per_fiber - 1);
  if (g.last_lengths.size() != ne || std::memcmp(g.last_lengths.data(), elementLengths, ne * sizeof(float)) ||
      g.last_prefactor != prefactor) {
    g.last_lengths.assign(elementLengths, elementLengths + ne);
    g.last_prefactor = prefactor;
    std::vector<double> h(ne), pf(g.n_fibers, prefactor);
    for (size_t i = 0; i < ne; i++)
      h[i] = elementLengths[i];
    if (cudaMemcpy(s->elem_d.p, h.data(), sizeof(double) * ne, cudaMemcpyHostToDevice) != cudaSuccess)
      return;
    if (fdm_set_prefactor(s, pf.data()))
      return;
  }
  // parameters: the caller's per-instance values fill the model's first parameter slots
  const size_t npv = (size_t)g.n_params * N;
  if (g.last_params.size() != npv || std::memcmp(g.last_params.data(), parameters, npv * sizeof(float))) {
    g.last_params.assign(parameters, parameters + npv);
    std::vector<double> p((size_t)NP * N);
    for (int q = 0; q < NP; q++)
      for (int64_t i = 0; i < N; i++)
        p[(size_t)q * N + i] = q < g.n_params ? (double)parameters[(size_t)q * N + i] : s->model->parameter_defaults[q];
    if (fdm_set_parameters(s, p.data()))
      return;
  }
  if (s->cfg.value_for_stimulated_point != valueForStimulatedPoint)
    invalidate_graphs(s);
  s->cfg.value_for_stimulated_point = valueForStimulatedPoint;
  if (advance_explicit(s, startTime, timeStepWidthSplitting, nTimeStepsSplitting, dt0D, nTimeSteps0D, dt1D))
    return;
  // transfer outputs (gpu.tpp:1086-1115 reads them as [k * nInstances + instance])
  std::vector<double> st((size_t)s->model->n_states * N);
  if (fdm_get_states(s, st.data()))
    return;
  for (int k = 0; k < g.n_states_tr; k++) {
    const int idx = g.state_idx[k];
    std::memcpy(statesForTransfer + (size_t)k * N, st.data() + (size_t)idx * N, sizeof(double) * N);
  }
  if (g.n_alg > 0 && algebraicsForTransfer)
    fdm_get_algebraics(s, algebraicsForTransfer);
}

extern "C" int fdm_compat_release(void)
{
  std::lock_guard<std::mutex> lock(g_compat_mu);
  if (g_compat.s)
    fdm_destroy(g_compat.s);
  g_compat = Compat();
  return FDM_OK;
}

// ---------------------------------------------------------------------------------------------
// adjoint: discrete reverse mode of the FP64 split path with checkpointing
// ---------------------------------------------------------------------------------------------

// device copies of the evolving state: Vm, the other states (FP64) and the stimulation machine
static int copy_state(fdm_solver* s, double* vm, double* st, double* last, double* jit, int* jidx, uint8_t* hbs,
                      bool to_snapshot)
{
  const int64_t N = s->n_nodes;
  const int NS = s->model->n_states;
  const int nf = s->n_fibers;
  auto cp = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s->stream);
  };
  if (to_snapshot) {
    FDM_CUDA(cp(vm, s->vm.p, sizeof(double) * N));
    if (NS > 1)
      FDM_CUDA(cp(st, s->states.p, sizeof(double) * N * (NS - 1)));
    FDM_CUDA(cp(last, s->last_check.p, sizeof(double) * nf));
    FDM_CUDA(cp(jit, s->cur_jitter.p, sizeof(double) * nf));
    FDM_CUDA(cp(jidx, s->jitter_idx.p, sizeof(int) * nf));
    FDM_CUDA(cp(hbs, s->hbs.p, nf));
  } else {
    FDM_CUDA(cp(s->vm.p, vm, sizeof(double) * N));
    if (NS > 1)
      FDM_CUDA(cp(s->states.p, st, sizeof(double) * N * (NS - 1)));
    FDM_CUDA(cp(s->last_check.p, last, sizeof(double) * nf));
    FDM_CUDA(cp(s->cur_jitter.p, jit, sizeof(double) * nf));
    FDM_CUDA(cp(s->jitter_idx.p, jidx, sizeof(int) * nf));
    FDM_CUDA(cp(s->hbs.p, hbs, nf));
  }
  return FDM_OK;
}

extern "C" int fdm_adjoint_forward(fdm_solver* s, double t_start, double t_end, int checkpoint_every, int n_sensors,
                                   const int64_t* sensor_nodes)
{
  if (s && s->eq.on)
    return fail(s, FDM_ERR_UNSUPPORTED, "fdm_adjoint_forward: the equilibrium skip's decisions are not differentiable; "
                                        "switch it off for the adjoint");
  if (!s || checkpoint_every < 1 || n_sensors < 0 || (n_sensors > 0 && !sensor_nodes))
    return fail(s, FDM_ERR_ARG, "fdm_adjoint_forward: bad argument");
  FDM_BIND(s);
  if (s->cfg.method != FDM_METHOD_SPLIT || s->real_bytes != 8)
    return fail(s, FDM_ERR_UNSUPPORTED, "fdm_adjoint_forward: the adjoint runs on the FP64 split path "
                                        "(method FDM_METHOD_SPLIT, reaction_precision FDM_FP64)");
  if (s->n_fibers == 0 || !s->stimulation_set)
    return fail(s, FDM_ERR_ARG, "fdm_adjoint_forward: set fibers and stimulation first");
  auto& A = s->adj;
  A.release();
  A.steps.clear();
  A.dt1s.clear();
  plan_advance(s, t_start, t_end, A.steps, A.dt1s);
  const int64_t NT = (int64_t)A.steps.size();
  for (int64_t j = 0; j < NT; j++)
    A.steps[j].global_no = (int)j; // trace rows of this run
  int rc = fdm_set_trace(s, n_sensors, sensor_nodes, NT);
  if (rc)
    return rc;
  s->trace_base = s->split_no - NT;   // the rows are this run's steps (planned above)
  const int64_t N = s->n_nodes;
  const int NS = s->model->n_states;
  const int nf = s->n_fibers;
  A.kc = checkpoint_every;
  A.n_seg = (int)((NT + A.kc - 1) / A.kc);
  A.n_sensors = n_sensors;
  A.n0max = 1;
  for (auto& st : A.steps)
    A.n0max = std::max(A.n0max, st.n0);
  const size_t segs = std::max(A.n_seg, 1);
  FDM_CUDA(A.ck_vm.alloc(segs * N));
  FDM_CUDA(A.ck_states.alloc(segs * N * std::max(NS - 1, 1)));
  FDM_CUDA(A.ck_last.alloc(segs * nf));
  FDM_CUDA(A.ck_jit.alloc(segs * nf));
  FDM_CUDA(A.ck_jidx.alloc(segs * nf));
  FDM_CUDA(A.ck_hbs.alloc(segs * nf));
  FDM_CUDA(A.fin_vm.alloc(N));
  FDM_CUDA(A.fin_states.alloc((size_t)N * std::max(NS - 1, 1)));
  FDM_CUDA(A.fin_last.alloc(nf));
  FDM_CUDA(A.fin_jit.alloc(nf));
  FDM_CUDA(A.fin_jidx.alloc(nf));
  FDM_CUDA(A.fin_hbs.alloc(nf));
  { // an asynchronous advance still owes its timing and NaN check
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  s->ev_used = 0;
  FDM_CUDA(cudaEventRecord(s->adv_start, s->stream));
  // the replay in fdm_adjoint_backward runs the one-thread-per-node reaction kernel; the forward runs it too,
  // so that the replay reproduces it bit for bit (window graphs captured with the other kernel are dropped)
  invalidate_graphs(s);
  s->adj_forward = true;
  for (int c = 0; c < A.n_seg && !rc; c++) {
    rc = copy_state(s, A.ck_vm.p + (size_t)c * N, A.ck_states.p + (size_t)c * N * (NS - 1), A.ck_last.p + (size_t)c * nf,
                    A.ck_jit.p + (size_t)c * nf, A.ck_jidx.p + (size_t)c * nf, A.ck_hbs.p + (size_t)c * nf, true);
    if (rc)
      break;
    const size_t b = (size_t)c * A.kc, e = std::min<size_t>(b + A.kc, NT);
    rc = run_planned(s, A.steps, A.dt1s, b, e, c == A.n_seg - 1);
  }
  s->adj_forward = false;
  invalidate_graphs(s);
  if (rc)
    return rc;
  rc = copy_state(s, A.fin_vm.p, A.fin_states.p, A.fin_last.p, A.fin_jit.p, A.fin_jidx.p, A.fin_hbs.p, true);
  if (rc)
    return rc;
  A.fin_strang = s->strang;
  A.fin_heun = s->heun;
  A.fin_diff = s->diff;
  A.fin_split = s->split_no;
  rc = finish_advance(s);
  if (rc)
    return rc;
  A.ready = true;
  return FDM_OK;
}

extern "C" int fdm_adjoint_backward(fdm_solver* s, const double* trace_grad, double* grad_prefactor,
                                    double* grad_parameters, double* grad_states0)
{
  if (!s || !trace_grad)
    return fail(s, FDM_ERR_ARG, "fdm_adjoint_backward: bad argument");
  FDM_BIND(s);
  auto& A = s->adj;
  if (!A.ready)
    return fail(s, FDM_ERR_ARG, "fdm_adjoint_backward: call fdm_adjoint_forward first");
  const int64_t N = s->n_nodes;
  const int NS = s->model->n_states;
  const int NP = s->model->n_parameters;
  const int nf = s->n_fibers;
  const int64_t NT = (int64_t)A.steps.size();
  const size_t hstride = (size_t)A.n0max * NS * N; // one half step of stored substep states
  int max_words = 1;
  for (int c = 0; c < A.n_seg; c++) {
    const size_t b = (size_t)c * A.kc, e = std::min<size_t>(b + A.kc, NT);
    int nsub = 1;
    for (size_t j = b; j < e; j++)
      nsub = std::max(nsub, A.steps[j].n0);
    max_words = std::max(max_words, (int)(((e - b) * 2 * nsub + 31) / 32));
  }
  {
    int rc = ensure_step_capacity(s, A.kc);
    if (rc)
      return rc;
  }
  for (int k = 0; k < 2; k++) {
    if (s->gate_set)
      FDM_CUDA(A.gates[k].alloc((size_t)std::max(nf, 1) * 2 * s->step_capacity));
    FDM_CUDA(A.H[k].alloc((size_t)A.kc * 2 * hstride));
    FDM_CUDA(A.U[k].alloc((size_t)A.kc * N));
    FDM_CUDA(A.flags[k].alloc((size_t)max_words * std::max(nf, 1)));
    if (!A.replayed[k])
      FDM_CUDA(cudaEventCreateWithFlags(&A.replayed[k], cudaEventDisableTiming));
    if (!A.reversed[k])
      FDM_CUDA(cudaEventCreateWithFlags(&A.reversed[k], cudaEventDisableTiming));
  }
  if (!A.rstream)
    FDM_CUDA(cudaStreamCreateWithFlags(&A.rstream, cudaStreamNonBlocking));
  FDM_CUDA(A.lam.alloc((size_t)NS * N));
  FDM_CUDA(A.gP.alloc((size_t)std::max(NP, 1) * N));
  FDM_CUDA(A.gpf.alloc(nf));
  FDM_CUDA(A.mu.alloc(N));
  FDM_CUDA(A.ascratch.alloc(N));
  FDM_CUDA(A.tgrad.alloc(std::max<size_t>((size_t)NT * A.n_sensors, 1)));
  FDM_CUDA(cudaMemsetAsync(A.lam.p, 0, sizeof(double) * NS * N, s->stream));
  FDM_CUDA(cudaMemsetAsync(A.gP.p, 0, sizeof(double) * std::max(NP, 1) * N, s->stream));
  FDM_CUDA(cudaMemsetAsync(A.gpf.p, 0, sizeof(double) * nf, s->stream));
  if (NT * A.n_sensors > 0)
    FDM_CUDA(cudaMemcpyAsync(A.tgrad.p, trace_grad, sizeof(double) * NT * A.n_sensors, cudaMemcpyHostToDevice,
                             s->stream));
  const MathKind mk = s->cfg.approximate_exponential_function ? MATH_APPROX : MATH_EXACT;
  const int ie = s->cfg.diffusion_scheme == FDM_IMPLICIT_EULER;
  // The diffusion step width dt1D = ((t + dtSplit) - t)/n1D drifts in its last bits as t grows; the
  // factorization in use is replaced when dt1D leaves a relative 1e-12 of it (ensure_coefficients).  The
  // same rule applied to the run's step widths gives the factorizations ("epochs") of every split step;
  // each is computed once into its own buffer, so that replay and reverse sweeps, which both read them,
  // can run on two streams.  With many epochs (a step width changing at every step) everything runs in
  // order on one stream and the coefficients are refactorized where the width changes.
  std::vector<int> epoch(NT, 0);
  std::vector<double> edt;
  for (int64_t j = 0; j < NT; j++) {
    if (edt.empty() || std::fabs(A.dt1s[j] - edt.back()) > 1e-12 * std::fabs(edt.back()))
      edt.push_back(A.dt1s[j]);
    epoch[j] = (int)edt.size() - 1;
  }
  const bool pipelined = !edt.empty() && edt.size() <= 16;
  cudaStream_t rs = pipelined ? A.rstream : s->stream;
  if (pipelined) {
    FDM_CUDA(A.coefs.alloc(edt.size() * 6 * (size_t)N));
    for (size_t e = 0; e < edt.size(); e++) {
      FDM_CUDA(launch_coefficients(nf, s->off_d.p, s->elem_d.p, s->prefactor_d.p, edt[e], ie, A.coefs.p + e * 6 * N, N,
                                   s->stream));
      s->launches++;
    }
  }
  auto coef_of = [&](size_t j) -> const double* { return pipelined ? A.coefs.p + (size_t)epoch[j] * 6 * N : s->coef.p; };
  { // an asynchronous advance still owes its timing and NaN check
    const int rw = fdm_wait(s);
    if (rw)
      return rw;
  }
  s->ev_used = 0;
  FDM_CUDA(cudaEventRecord(s->adv_start, s->stream));
  std::vector<WindowInfo> win(A.n_seg);

  // replay of segment c into buffer k (stream s->stream): every substep's input state and Vm before each
  // diffusion solve
  auto replay = [&](int c, int k) -> int {
    FDM_CUDA(cudaStreamWaitEvent(s->stream, A.reversed[k], 0));
    int rc = copy_state(s, A.ck_vm.p + (size_t)c * N, A.ck_states.p + (size_t)c * N * (NS - 1),
                        A.ck_last.p + (size_t)c * nf, A.ck_jit.p + (size_t)c * nf, A.ck_jidx.p + (size_t)c * nf,
                        A.ck_hbs.p + (size_t)c * nf, false);
    if (rc)
      return rc;
    const size_t b = (size_t)c * A.kc, e = std::min<size_t>(b + A.kc, NT);
    const int len = (int)(e - b);
    rc = prepare_window(s, A.steps.data() + b, len, &win[c], A.flags[k].p, s->gate_set ? A.gates[k].p : nullptr);
    if (rc)
      return rc;
    ReactionArgs ra{};
    ra.n_nodes = N;
    ra.stride = N;
    ra.vm = s->vm.p;
    ra.states = s->states.p;
    ra.params = s->params.p;
    ra.clamp_fiber = s->clamp_fiber.p;
    ra.flags = A.flags[k].p;
    ra.words_per_fiber = win[c].words;
    ra.gate = s->gate_set ? s->gate.p : nullptr;
    ra.gate_start = win[c].gate_start;
    ra.gate_stride = win[c].gate_stride;
    ra.nsub_stride = win[c].nsub;
    ra.vstim = s->cfg.value_for_stimulated_point;
    ra.stimulus_mode = s->cfg.stimulus_mode;
    ra.stimulus_parameter = s->cfg.stimulus_parameter;
    ra.stimulus_value = s->cfg.stimulus_value;
    ra.steps = s->steps_d.p;
    for (int jj = 0; jj < len; jj++) {
      if (!pipelined) {
        rc = ensure_coefficients(s, A.dt1s[b + jj]);
        if (rc)
          return rc;
      }
      ra.step = jj;
      for (int half = 0; half < 2; half++) {
        ra.half = half;
        ra.store_states = A.H[k].p + ((size_t)jj * 2 + half) * hstride;
        // Vm before the diffusion solve (U) comes out of the first half step; Vm after it is the stored input
        // of the second half step's first substep
        ra.store_vm_out = half == 0 ? A.U[k].p + (size_t)jj * N : nullptr;
        FDM_CUDA(launch_reaction(s->cfg.model, REAL_F64, mk, ra, s->stream));
        s->launches++;
        if (half == 0) {
          FDM_CUDA(launch_diffusion(nf, s->off_d.p, coef_of(b + jj), N, s->vm.p, s->scratch.p, s->stream));
          s->launches++;
        }
      }
    }
    FDM_CUDA(cudaEventRecord(A.replayed[k], s->stream));
    return FDM_OK;
  };

  // reverse sweep of segment c from buffer k (stream A.rstream)
  auto reverse = [&](int c, int k) -> int {
    FDM_CUDA(cudaStreamWaitEvent(rs, A.replayed[k], 0));
    const size_t b = (size_t)c * A.kc, e = std::min<size_t>(b + A.kc, NT);
    const int len = (int)(e - b);
    AdjointArgs aa{};
    aa.n_nodes = N;
    aa.params = (const double*)s->params.p;
    aa.lam = A.lam.p;
    aa.grad_params = A.gP.p;
    aa.clamp_fiber = s->clamp_fiber.p;
    aa.flags = A.flags[k].p;
    aa.words_per_fiber = win[c].words;
    aa.gate = s->gate_set ? s->gate.p : nullptr;
    aa.gate_start = win[c].gate_start;
    aa.gate_stride = win[c].gate_stride;
    aa.nsub_stride = win[c].nsub;
    aa.vstim = s->cfg.value_for_stimulated_point;
    aa.stimulus_mode = s->cfg.stimulus_mode;
    aa.stimulus_parameter = s->cfg.stimulus_parameter;
    aa.stimulus_value = s->cfg.stimulus_value;
    aa.trace_slot = A.n_sensors > 0 ? s->trace_slot.p : nullptr;
    aa.trace_grad = A.tgrad.p;
    aa.n_trace = A.n_sensors;
    aa.use_tape = s->adjoint_tape;
    for (int jj = len - 1; jj >= 0; jj--) {
      const size_t j = b + jj;
      aa.step = A.steps[j];
      aa.step_in_window = jj;
      aa.half = 1;
      aa.trace_row = (int64_t)j;
      aa.states = A.H[k].p + ((size_t)jj * 2 + 1) * hstride;
      FDM_CUDA(launch_adjoint_half(s->cfg.model, mk, aa, rs));
      if (!pipelined) {
        int rc = ensure_coefficients(s, A.dt1s[j]);
        if (rc)
          return rc;
      }
      FDM_CUDA(launch_adjoint_diffusion(nf, s->off_d.p, s->elem_d.p, coef_of(j), N, A.lam.p, A.U[k].p + (size_t)jj * N,
                                        A.H[k].p + ((size_t)jj * 2 + 1) * hstride, ie, A.gpf.p, A.ascratch.p, A.mu.p,
                                        s->max_fiber_len, rs));
      aa.half = 0;
      aa.trace_row = -1;
      aa.states = A.H[k].p + ((size_t)jj * 2 + 0) * hstride;
      FDM_CUDA(launch_adjoint_half(s->cfg.model, mk, aa, rs));
      s->launches += 3;
    }
    FDM_CUDA(cudaEventRecord(A.reversed[k], rs));
    return FDM_OK;
  };

  // the reverse stream starts after the gradient buffers are cleared; buffers start free
  FDM_CUDA(cudaEventRecord(A.reversed[0], s->stream));
  FDM_CUDA(cudaEventRecord(A.reversed[1], s->stream));
  FDM_CUDA(cudaStreamWaitEvent(rs, A.reversed[0], 0));
  if (A.n_seg > 0) {
    int rc = replay(A.n_seg - 1, (A.n_seg - 1) & 1);
    if (rc)
      return rc;
  }
  for (int c = A.n_seg - 1; c >= 0; c--) {
    if (c > 0) {
      int rc = replay(c - 1, (c - 1) & 1);
      if (rc)
        return rc;
    }
    int rc = reverse(c, c & 1);
    if (rc)
      return rc;
  }
  // join: the gradients are complete when the last reverse sweep is
  FDM_CUDA(cudaEventRecord(A.reversed[0], rs));
  FDM_CUDA(cudaStreamWaitEvent(s->stream, A.reversed[0], 0));
  FDM_CUDA(cudaEventRecord(s->adv_stop, s->stream));
  if (grad_parameters && NP > 0)
    FDM_CUDA(cudaMemcpyAsync(grad_parameters, A.gP.p, sizeof(double) * NP * N, cudaMemcpyDeviceToHost, s->stream));
  if (grad_prefactor)
    FDM_CUDA(cudaMemcpyAsync(grad_prefactor, A.gpf.p, sizeof(double) * nf, cudaMemcpyDeviceToHost, s->stream));
  if (grad_states0)
    FDM_CUDA(cudaMemcpyAsync(grad_states0, A.lam.p, sizeof(double) * NS * N, cudaMemcpyDeviceToHost, s->stream));
  // the solver continues from the state the forward run ended in
  int rc = copy_state(s, A.fin_vm.p, A.fin_states.p, A.fin_last.p, A.fin_jit.p, A.fin_jidx.p, A.fin_hbs.p, false);
  if (rc)
    return rc;
  FDM_CUDA(cudaStreamSynchronize(s->stream));
  float ms = 0;
  FDM_CUDA(cudaEventElapsedTime(&ms, s->adv_start, s->adv_stop));
  s->adj_ms += ms;
  s->strang = A.fin_strang;
  s->heun = A.fin_heun;
  s->diff = A.fin_diff;
  s->split_no = A.fin_split;
  return FDM_OK;
}

extern "C" int fdm_adjoint_release(fdm_solver* s)
{
  if (!s)
    return FDM_ERR_ARG;
  FDM_BIND(s);
  s->adj.release();
  return FDM_OK;
}

extern "C" int fdm_adjoint_timing(const fdm_solver* s, double* backward_ms)
{
  if (!s || !backward_ms)
    return FDM_ERR_ARG;
  *backward_ms = s->adj_ms;
  return FDM_OK;
}

// back to the start: time-stepping objects, Strang step counter and the stimulation machine as after
// fdm_set_stimulation (the states are left as they are)
extern "C" int fdm_rewind(fdm_solver* s)
{
  if (!s)
    return FDM_ERR_ARG;
  FDM_BIND(s);
  s->tss_init = false;
  s->split_no = 0;
  s->trace_base = 0;
  s->ck_valid = false;
  const int nf = s->n_fibers;
  if (s->stimulation_set && nf > 0) {
    std::vector<double> last(nf), cj(nf, 0.0);
    std::vector<int> ji(nf, 0);
    std::vector<uint8_t> h0(nf, 0);
    for (int f = 0; f < nf; f++)
      last[f] = s->stim_begin[f] - 1e-13 - 1. / (s->stim_freq[f] + cj[f]);
    FDM_CUDA(cudaMemcpyAsync(s->last_check.p, last.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->cur_jitter.p, cj.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->jitter_idx.p, ji.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->hbs.p, h0.data(), nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaMemcpyAsync(s->cur_stim.p, h0.data(), nf, cudaMemcpyHostToDevice, s->stream));
    FDM_CUDA(cudaStreamSynchronize(s->stream));
  }
  if (s->eq.on) {
    int rc = eq_reset(s);
    if (rc)
      return rc;
  }
  return FDM_OK;
}
