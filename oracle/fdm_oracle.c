/* CPU oracle for the fiber monodomain hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C and FP64, what the reference's
 * FastMonodomainSolver computes with optimizationType "vc".  It is the checker for the CUDA
 * product (tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg use it); the product
 * never links or calls it.
 *
 * Followed reference code (paths relative to the opendihu source tree):
 *   time stepping rule      core/src/time_stepping_scheme/00_time_stepping_scheme.cpp:15-68
 *   RepeatedCall loop       core/src/time_stepping_scheme/repeated_call.tpp:43-80
 *   Strang loop             core/src/specialized_solver/fast_monodomain_solver/fast_monodomain_solver_compute.tpp:48-129
 *   compute0D               ...compute.tpp:131-254  (point buffers of W lanes, centre detection :158-166)
 *   Heun step + clamps      core/src/cellml/source_code_generator/03_generator_vc.cpp:1017-1163
 *   compute1D (Thomas)      ...compute.tpp:256-507  (consistent mass, IE or CN)
 *   stimulation machine     ...compute.tpp:509-627
 *   initial check time      ...fast_monodomain_solver_initialization.tpp:342-347
 *   ExplicitEuler           core/src/time_stepping_scheme/explicit_euler.tpp:20-60
 * Model right-hand sides come from generated/ (emitted from the reference's OpenCOR C inputs).
 *
 * Floating point: compile with -ffp-contract=off so that every expression is evaluated exactly
 * as written (no fused multiply-add), which is the canonical semantics the product's discrete
 * decisions (stimulation times) are checked against.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_math.h"
#include "generated/hodgkin_huxley_1952_anone_c2_3_4.h"
#include "generated/shorten_ocallaghan_davidson_soboleva_2007_a32_c65.h"

typedef void (*oracle_rates_fn)(double, const double *, const double *, double *, double *, int);

typedef struct {
  const char *name;
  int n_states, n_algebraics, n_parameters;
  oracle_rates_fn rates;
  const double *states_initial;
} oracle_model;

static const oracle_model oracle_models[] = {
  {"hodgkin_huxley_1952", 4, 9, 3, oracle_hodgkin_huxley_1952_anone_c2_3_4_rates,
   oracle_hodgkin_huxley_1952_anone_c2_3_4_states_initial},
  {"shorten_ocallaghan_davidson_soboleva_2007", 56, 71, 2,
   oracle_shorten_ocallaghan_davidson_soboleva_2007_a32_c65_rates,
   oracle_shorten_ocallaghan_davidson_soboleva_2007_a32_c65_states_initial},
};
#define ORACLE_N_MODELS ((int)(sizeof(oracle_models) / sizeof(oracle_models[0])))
#define ORACLE_MAX_STATES 64
#define ORACLE_MAX_VC_WIDTH 16
#define ORACLE_MAX_ALGEBRAICS 80
#define ORACLE_MAX_PARAMETERS 8

int oracle_model_info(int model, int *n_states, int *n_algebraics, int *n_parameters, double *states_initial)
{
  if (model < 0 || model >= ORACLE_N_MODELS)
    return -1;
  const oracle_model *m = &oracle_models[model];
  if (n_states) *n_states = m->n_states;
  if (n_algebraics) *n_algebraics = m->n_algebraics;
  if (n_parameters) *n_parameters = m->n_parameters;
  if (states_initial)
    memcpy(states_initial, m->states_initial, sizeof(double) * m->n_states);
  return 0;
}

/* one evaluation of the right-hand side (for unit tests of the model code) */
int oracle_rates(int model, double t, const double *states, const double *params, double *rates, double *algebraics,
                 int approx)
{
  if (model < 0 || model >= ORACLE_N_MODELS)
    return -1;
  double alg[ORACLE_MAX_ALGEBRAICS];
  oracle_models[model].rates(t, states, params, rates, algebraics ? algebraics : alg, approx);
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * ExplicitEuler over one cell (explicit_euler.tpp:38-60): y += dt f(t, y), t_k = t0 + k/N*span
 * ------------------------------------------------------------------------------------------- */
int oracle_explicit_euler_cell(int model, double *states, const double *params, double t0, double dt, int n_steps,
                               int approx)
{
  if (model < 0 || model >= ORACLE_N_MODELS)
    return -1;
  const oracle_model *m = &oracle_models[model];
  double rates[ORACLE_MAX_STATES], alg[ORACLE_MAX_ALGEBRAICS];
  const double span = dt * n_steps;
  double t = t0;
  for (int k = 0; k < n_steps;) {
    m->rates(t, states, params, rates, alg, approx);
    for (int s = 0; s < m->n_states; s++)
      states[s] = states[s] + dt * rates[s];
    k++;
    t = t0 + (double)k / n_steps * span;
  }
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * time stepping rule (00_time_stepping_scheme.cpp:15-68)
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  double start, end, dt, target;
  int n;
} oracle_tss;

static void tss_set_dt(oracle_tss *s, double dt)
{
  s->target = dt;
  long double n = ceill((long double)(s->end - s->start) / dt - 1e-1);
  s->n = n < 1 ? 1 : (int)n;
  s->dt = (s->end - s->start) / s->n;
}

static void tss_init(oracle_tss *s, double start, double end, double dt)
{
  s->start = start;
  s->end = end;
  s->dt = dt;
  s->target = dt;
}

static void tss_set_span(oracle_tss *s, double start, double end)
{
  s->start = start;
  s->end = end;
  if (s->target > end - start)
    s->dt = end - start;
  tss_set_dt(s, s->dt);
}

/* ---------------------------------------------------------------------------------------------
 * problem description
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  int model;
  int n_fibers;
  const int64_t *fiber_offsets;   /* n_fibers + 1 node offsets */
  const double *element_lengths;  /* fiber f: n_f - 1 lengths starting at fiber_offsets[f] - f */
  const double *prefactor;        /* per fiber */
  const double *parameters;       /* [p][node] */
  int diffusion_scheme;           /* 0 implicit Euler, 1 Crank-Nicolson */
  int approx_exp;
  int clamp_rule;                 /* 0: W-lane block of the vc path, 1: centre-1..centre+1 */
  int vc_width;
  int n_ranks;                    /* fibers go to rank fiberNo % n_ranks, each rank has its own buffers */
  int stimulus_mode;              /* 0: clamp Vm, 1: set parameter stimulus_parameter to stimulus_value */
  int stimulus_parameter;
  double stimulus_value;
  double value_for_stimulated_point;
  /* stimulation inputs */
  const uint8_t *firing_events;   /* [row][col] */
  int firing_rows, firing_cols;
  const int *motor_unit_no;       /* per fiber */
  const int *stimulation_point_index;
  const double *call_frequency, *repeat_after_first_call, *call_enable_begin;
  const double *jitter;           /* per fiber n_jitter values */
  int n_jitter;
  /* time */
  double t_start, t_end;
  double dt_repeated_call, dt_splitting, dt_0d, dt_1d;
  int n_threads;
  /* outputs */
  int n_algebraics_out;
  const int *algebraic_indices;
  double *algebraics_out;         /* [k][node] */
  int n_trace_nodes;
  const int64_t *trace_nodes;
  double *trace;                  /* [split step][trace node], Vm after each split step */
  int64_t trace_capacity;         /* number of split steps the trace buffer holds */
  /* onlyComputeIfHasBeenStimulated (compute.tpp:201-205): a point buffer is not computed while the
   * fiber it is attributed to has not been stimulated; the flag per fiber is in/out (NULL: all 0) */
  int only_if_stimulated;
  int *has_been_stimulated;
  /* disableComputationWhenStatesAreCloseToEquilibrium (compute.tpp:630-797): every point buffer carries a
   * status (0 inactive, 1 neighbor_is_active, 2 active), a rank counts its buffers set inactive, and a
   * rank whose count equals its number of buffers skips compute1D (compute.tpp:261-265).  In/out, per
   * rank: eq_status (the ranks' buffers one after the other; NULL: all active), eq_counter (NULL: 0),
   * pad_states [rank][lane][state] for the lanes of a rank's last buffer past its last node, which the
   * reference computes like the others and includes in the equilibrium test (NULL: initial values). */
  int equilibrium;
  uint8_t *eq_status;
  int *eq_counter;
  double *pad_states;
  /* stimulation log (StimulationLogging::logStimulationBegin, called at compute.tpp:603-607): the time and
   * fiber of every substep whose decision stimulates while the fiber's previous decision did not.
   * currently_stimulating per fiber is in/out (NULL: all 0); log_times/log_fibers hold log_capacity entries,
   * *log_count counts all (NULL: no log). */
  int *currently_stimulating;
  double *log_times;
  int *log_fibers;
  int64_t log_capacity;
  int64_t *log_count;
} oracle_problem;

enum { EQ_INACTIVE = 0, EQ_NEIGHBOR_IS_ACTIVE = 1, EQ_ACTIVE = 2 };

typedef struct {
  double last_check_time, current_jitter;
  int jitter_index;
  int has_been_stimulated;
  int currently_stimulating;
} oracle_fiber_state;

/* initial state of the stimulation machine (initialization.tpp:342-347) */
void oracle_stimulation_init(const oracle_problem *p, double *last_check_time, double *current_jitter,
                             int *jitter_index)
{
  for (int f = 0; f < p->n_fibers; f++) {
    current_jitter[f] = 0;
    jitter_index[f] = 0;
    last_check_time[f] = p->call_enable_begin[f] - 1e-13 - 1. / (p->call_frequency[f] + current_jitter[f]);
  }
}

/* isCurrentPointStimulated (compute.tpp:509-627) */
static int stimulation_machine(const oracle_problem *p, int f, oracle_fiber_state *st, double t)
{
  const double freq = p->call_frequency[f];
  const double repeat = p->repeat_after_first_call[f];
  const double begin = p->call_enable_begin[f];
  int check = 0;
  if (t >= st->last_check_time + 1. / (freq + st->current_jitter) && t >= begin - 1e-13) {
    check = 1;
    if (repeat != 0 && t - (st->last_check_time + 1. / (freq + st->current_jitter)) > repeat) {
      st->last_check_time += 1. / (freq + st->current_jitter);
      double jitter_factor = 0.0;
      if (p->n_jitter > 0)
        jitter_factor = p->jitter[(int64_t)f * p->n_jitter + st->jitter_index % p->n_jitter];
      st->current_jitter = jitter_factor * freq;
      st->jitter_index++;
      check = 0;
    }
  }
  int index = (int)round(t * freq);
  int row = index % p->firing_rows;
  if (row < 0)
    row += p->firing_rows;
  const int col = p->motor_unit_no[f] % p->firing_cols;
  const int stimulate = check && p->firing_events[(int64_t)row * p->firing_cols + col];
  if (stimulate)
    st->has_been_stimulated = 1;
  if (stimulate && !st->currently_stimulating && p->log_count) {
    int64_t i;
#pragma omp atomic capture
    i = (*p->log_count)++;
    if (i < p->log_capacity) {
      p->log_times[i] = t;
      p->log_fibers[i] = f;
    }
  }
  st->currently_stimulating = stimulate;
  return stimulate;
}

/* ---------------------------------------------------------------------------------------------
 * per-rank view: the fibers a rank computes, concatenated (valuesOffset), in point buffers
 * ------------------------------------------------------------------------------------------- */
typedef struct {
  int n_fibers;
  int *fibers;           /* global fiber numbers */
  int64_t *values_offset;/* offset of each local fiber in the rank's concatenated node list */
  int64_t n_values;
  int64_t n_buffers;
  int64_t *node_of;      /* rank-local index -> global node index */
  double *states;        /* [s][n_buffers*W], rank-local copy */
  double *params;        /* [p][n_buffers*W] */
  double *alg_out;       /* [k][n_buffers*W] */
  double *c_prime, *d_prime;
  uint8_t *eq_status;    /* n_buffers (points into the problem's eq_status or a local array) */
  int eq_counter;
} oracle_rank;

static void heun_step(const oracle_model *m, double *y, const double *prm, double t, double dt, int stimulate,
                      int clamp, double v_stim, int store, const oracle_problem *p, double *alg_store,
                      int64_t stride)
{
  /* 03_generator_vc.cpp:1017-1163 for a single lane */
  double rate[ORACLE_MAX_STATES], alg[ORACLE_MAX_ALGEBRAICS];
  double ys[ORACLE_MAX_STATES], rate2[ORACLE_MAX_STATES], alg2[ORACLE_MAX_ALGEBRAICS];
  m->rates(t, y, prm, rate, alg, p->approx_exp);
  for (int s = 0; s < m->n_states; s++)
    ys[s] = y[s] + dt * rate[s];
  if (stimulate && clamp)
    ys[0] = v_stim;
  m->rates(t, ys, prm, rate2, alg2, p->approx_exp);
  for (int s = 0; s < m->n_states; s++)
    y[s] += 0.5 * dt * (rate[s] + rate2[s]);
  if (stimulate && clamp)
    y[0] = v_stim;
  if (store)
    for (int k = 0; k < p->n_algebraics_out; k++)
      alg_store[k * stride] = alg2[p->algebraic_indices[k]];
}

/* n_steps Heun steps of one W-lane point buffer as compute0D calls the generated compute0DInstance
 * (03_generator_vc.cpp:913-1163): y[s * W + lane], params[q * W + lane]; step k at t0 + k * dt; when stimulate
 * is set the lanes 0..min(3, W)-1 are clamped to v_stim (the vc rule's lanes of the junction buffer); after
 * the last step the algebraics alg_indices[0..n_alg) of the second evaluation go to alg_out[k * W + lane].
 * Exported for the cross-check against the reference's own generated code. */
int oracle_heun_buffer(int model, int W, int approx, double *y, const double *params, double t0, double dt,
                       int n_steps, int stimulate, double v_stim, int n_alg, const int *alg_indices, double *alg_out)
{
  if (model < 0 || model >= ORACLE_N_MODELS || W < 1 || W > ORACLE_MAX_VC_WIDTH || n_alg < 0)
    return -1;
  const oracle_model *m = &oracle_models[model];
  oracle_problem p;
  memset(&p, 0, sizeof(p));
  p.approx_exp = approx;
  p.n_algebraics_out = n_alg;
  p.algebraic_indices = alg_indices;
  for (int lane = 0; lane < W; lane++) {
    double ys[ORACLE_MAX_STATES], prm[ORACLE_MAX_PARAMETERS];
    for (int s = 0; s < m->n_states; s++)
      ys[s] = y[s * W + lane];
    for (int q = 0; q < m->n_parameters; q++)
      prm[q] = params[q * W + lane];
    const int clamp = lane < (W < 3 ? W : 3);
    for (int k = 0; k < n_steps; k++)
      heun_step(m, ys, prm, t0 + k * dt, dt, stimulate, clamp, v_stim, k == n_steps - 1 && n_alg > 0, &p,
                alg_out ? alg_out + lane : NULL, W);
    for (int s = 0; s < m->n_states; s++)
      y[s * W + lane] = ys[s];
  }
  return 0;
}

/* equilibriumAccelerationUpdate (compute.tpp:630-762) for buffer b after its substeps: the buffer is at
 * equilibrium if no state of any lane changed by more than 1e-6 (relative, or absolute when the smallest
 * lane value of the state is below 1e-11 in magnitude); statuses and the rank's count follow the
 * reference's three-state rules */
static void equilibrium_update(const oracle_model *m, oracle_rank *r, int64_t b, int W, int64_t N,
                               const double *previous)
{
  uint8_t *st = r->eq_status;
  const int64_t nb = r->n_buffers;
  int at_equilibrium = 1;
  if (st[b] != EQ_INACTIVE) {
    for (int s = 0; s < m->n_states && at_equilibrium; s++) {
      double vmin = r->states[s * N + b * W];
      for (int lane = 1; lane < W; lane++)
        if (r->states[s * N + b * W + lane] < vmin)
          vmin = r->states[s * N + b * W + lane];
      double change = 0.0;
      for (int lane = 0; lane < W; lane++) {
        const double nv = r->states[s * N + b * W + lane], ov = previous[s * W + lane];
        const double c = fabs(vmin) < 1e-11 ? fabs(nv - ov) : fabs((nv - ov) / nv);
        if (c > change || c != c)
          change = c != c ? INFINITY : c;
      }
      if (change > 1e-6)
        at_equilibrium = 0;
    }
  }
  if (st[b] == EQ_NEIGHBOR_IS_ACTIVE && at_equilibrium) {
    if (b > 0 && st[b - 1] != EQ_ACTIVE && st[b] != EQ_INACTIVE) {
      st[b] = EQ_INACTIVE;
      r->eq_counter++;
    }
    if (b < nb - 1 && st[b + 1] != EQ_ACTIVE && st[b] != EQ_INACTIVE) {
      st[b] = EQ_INACTIVE;
      r->eq_counter++;
    }
  }
  if (st[b] == EQ_ACTIVE || st[b] == EQ_NEIGHBOR_IS_ACTIVE) {
    if (at_equilibrium) {
      st[b] = EQ_INACTIVE;
      r->eq_counter++;
    } else {
      st[b] = EQ_ACTIVE;
      if (b > 0 && st[b - 1] == EQ_INACTIVE) {
        r->eq_counter--;
        st[b - 1] = EQ_NEIGHBOR_IS_ACTIVE;
      }
      if (b < nb - 1 && st[b + 1] == EQ_INACTIVE) {
        r->eq_counter--;
        st[b + 1] = EQ_NEIGHBOR_IS_ACTIVE;
      }
    }
  }
}

/* compute0D for one rank (compute.tpp:131-254) */
static void compute0d(const oracle_problem *p, oracle_rank *r, oracle_fiber_state *fs, double t0, double dt,
                      int n_steps, int store)
{
  const oracle_model *m = &oracle_models[p->model];
  const int W = p->vc_width;
  const int64_t N = r->n_buffers * W;
  const double factor = (double)W / (double)(r->values_offset[1] - r->values_offset[0]);
  /* buffers are independent; each fiber's stimulation machine is advanced only by the one buffer
   * that holds its junction, so the loop runs in parallel without changing the result.  With
   * onlyComputeIfHasBeenStimulated a buffer reads the flag its fiber's junction buffer sets, so the
   * buffers run in the reference's order, one after the other. */
  const int eq = p->equilibrium != 0;
  const int serial = p->only_if_stimulated != 0 || eq;
  const int64_t nb = r->n_buffers;
  uint8_t *status = r->eq_status;
  if (eq && nb > 0) {
    /* compute.tpp:154-156: the first and the last buffer of the rank are set active (the count is not
     * adjusted) */
    status[0] = EQ_ACTIVE;
    status[nb - 1] = EQ_ACTIVE;
  }
#pragma omp parallel for num_threads(serial ? 1 : (p->n_threads > 0 ? p->n_threads : 1)) schedule(static)
  for (int64_t b = 0; b < r->n_buffers; b++) {
    double y[ORACLE_MAX_STATES], prm[ORACLE_MAX_PARAMETERS];
    double previous[ORACLE_MAX_STATES * ORACLE_MAX_VC_WIDTH];
    if (eq)
      for (int lane = 0; lane < W; lane++)
        for (int s = 0; s < m->n_states; s++)
          previous[s * W + lane] = r->states[s * N + b * W + lane];
    int local = (int)(b * factor);
    if (local >= r->n_fibers)
      local = r->n_fibers - 1;
    const int f = r->fibers[local];
    const int64_t index_in_fiber = b * W - r->values_offset[local];
    const int center = p->stimulation_point_index[f];
    int in_center;
    if (p->clamp_rule == 0)
      in_center = (unsigned long)((long)center - (long)index_in_fiber) < (unsigned long)W;
    else
      in_center = 0;
    for (int k = 0; k < n_steps; k++) {
      const double t = t0 + k * dt;
      int stim = 0;
      if (in_center)
        stim = stimulation_machine(p, f, &fs[f], t);
      if (eq) {
        /* isEquilibriumAccelerationCurrentPointDisabled (compute.tpp:764-797) */
        if (stim) {
          status[b] = EQ_ACTIVE;
          if (b > 0 && status[b - 1] == EQ_INACTIVE) {
            r->eq_counter--;
            status[b - 1] = EQ_NEIGHBOR_IS_ACTIVE;
          }
          if (b < nb - 1 && status[b + 1] == EQ_INACTIVE) {
            r->eq_counter--;
            status[b + 1] = EQ_NEIGHBOR_IS_ACTIVE;
          }
        }
        if (status[b] == EQ_INACTIVE)
          continue;
      }
      if (p->only_if_stimulated && !fs[f].has_been_stimulated)
        continue; /* compute.tpp:201-205 */
      const int store_now = store && k == n_steps - 1;
      for (int lane = 0; lane < W; lane++) {
        const int64_t i = b * W + lane;
        if (r->node_of[i] < 0 && !eq)
          continue; /* padding lane (computed by the reference, but it only matters to the equilibrium test) */
        for (int s = 0; s < m->n_states; s++)
          y[s] = r->states[s * N + i];
        for (int q = 0; q < m->n_parameters; q++)
          prm[q] = r->params[q * N + i];
        int clamp = 0;
        if (p->clamp_rule == 0) {
          clamp = lane < (W < 3 ? W : 3);
        }
        if (p->stimulus_mode == 1 && stim && clamp)
          prm[p->stimulus_parameter] = p->stimulus_value;
        heun_step(m, y, prm, t, dt, stim, p->stimulus_mode == 0 ? clamp : 0, p->value_for_stimulated_point, store_now,
                  p, r->alg_out + i, N);
        for (int s = 0; s < m->n_states; s++)
          r->states[s * N + i] = y[s];
      }
    }
    if (eq)
      equilibrium_update(m, r, b, W, N, previous);
  }
}

/* the centre-1..centre+1 rule: the machine is advanced once per fiber and substep, and the three
 * nodes around the centre are clamped (fast_monodomain_solver_gpu.tpp:538-540; the reference's
 * offload code advances it from three threads at once, here it is advanced once, in time order) */
static void compute0d_center(const oracle_problem *p, oracle_rank *r, oracle_fiber_state *fs, double t0, double dt,
                             int n_steps, int store)
{
  const oracle_model *m = &oracle_models[p->model];
  const int64_t N = r->n_buffers * p->vc_width;
#pragma omp parallel num_threads(p->n_threads > 0 ? p->n_threads : 1)
  {
  double y[ORACLE_MAX_STATES], prm[ORACLE_MAX_PARAMETERS], prm_stim[ORACLE_MAX_PARAMETERS];
  int *stim = (int *)malloc(sizeof(int) * (n_steps > 0 ? n_steps : 1));
  int *stim_seen = (int *)malloc(sizeof(int) * (n_steps > 0 ? n_steps : 1));
#pragma omp for schedule(dynamic, 1)
  for (int lf = 0; lf < r->n_fibers; lf++) {
    const int f = r->fibers[lf];
    const int64_t n = p->fiber_offsets[f + 1] - p->fiber_offsets[f];
    const int64_t center = p->stimulation_point_index[f];
    for (int k = 0; k < n_steps; k++) {
      stim[k] = stimulation_machine(p, f, &fs[f], t0 + k * dt);
      stim_seen[k] = fs[f].has_been_stimulated; /* the flag after the machine's substep k */
    }
    for (int64_t j = 0; j < n; j++) {
      const int64_t i = r->values_offset[lf] + j;
      for (int s = 0; s < m->n_states; s++)
        y[s] = r->states[s * N + i];
      for (int q = 0; q < m->n_parameters; q++)
        prm[q] = prm_stim[q] = r->params[q * N + i];
      const int clamp = (j >= center - 1 && j <= center + 1);
      if (p->stimulus_mode == 1)
        prm_stim[p->stimulus_parameter] = p->stimulus_value;
      for (int k = 0; k < n_steps; k++) {
        const double t = t0 + k * dt;
        if (p->only_if_stimulated && !stim_seen[k])
          continue;
        const int on = stim[k] && clamp;
        heun_step(m, y, (p->stimulus_mode == 1 && on) ? prm_stim : prm, t, dt, on, p->stimulus_mode == 0, p->value_for_stimulated_point,
                  store && k == n_steps - 1, p, r->alg_out + i, N);
      }
      for (int s = 0; s < m->n_states; s++)
        r->states[s * N + i] = y[s];
    }
  }
  free(stim);
  free(stim_seen);
  }
}

/* compute1D for one rank (compute.tpp:256-507): one Thomas solve per fiber of
 *   IE: (K - M/dt) u+ = -M/dt u        CN: (K/2 - M/dt) u+ = (-K/2 - M/dt) u
 * with the 1D linear stencils K = prefactor/h [-1 1; 1 -1] and consistent mass M = h [1/3 1/6; 1/6 1/3] */
static void compute1d(const oracle_problem *p, oracle_rank *r, double dt)
{
  const int ie = p->diffusion_scheme == 0;
  const int64_t N = r->n_buffers * p->vc_width;
  double *u = r->states; /* state 0 */
  int64_t max_len = 1;
  for (int lf = 0; lf < r->n_fibers; lf++) {
    const int f = r->fibers[lf];
    const int64_t n = p->fiber_offsets[f + 1] - p->fiber_offsets[f];
    if (n > max_len)
      max_len = n;
  }
#pragma omp parallel num_threads(p->n_threads > 0 ? p->n_threads : 1)
  {
  double *cp = (double *)malloc(sizeof(double) * max_len), *dp = (double *)malloc(sizeof(double) * max_len);
#pragma omp for schedule(dynamic, 1)
  for (int lf = 0; lf < r->n_fibers; lf++) {
    const int f = r->fibers[lf];
    const int64_t n = p->fiber_offsets[f + 1] - p->fiber_offsets[f];
    const double *h = p->element_lengths + (p->fiber_offsets[f] - f);
    const double prefactor = p->prefactor[f];
    const int64_t o = r->values_offset[lf];
    for (int64_t v = 0; v < n; v++) {
      double a = 0, b = 0, c = 0, d = 0;
      double u_prev = 0, u_center = u[o + v], u_next = 0;
      if (v > 0) {
        u_prev = u[o + v - 1];
        const double h_left = h[v - 1];
        const double k_left = 1. / h_left * (1) * prefactor;
        const double m_left = h_left * 1. / 6;
        if (ie)
          a = (k_left - 1 / dt * m_left);
        else
          a = (k_left / 2. - 1 / dt * m_left);
        const double k_right = 1. / h_left * (-1) * prefactor;
        const double m_right = h_left * 1. / 3;
        if (ie) {
          b += (k_right - 1 / dt * m_right);
          d += (-1 / dt * m_left) * u_prev + (-1 / dt * m_right) * u_center;
        } else {
          b += (k_right / 2. - 1 / dt * m_right);
          d += (-k_left / 2. - 1 / dt * m_left) * u_prev + (-k_right / 2. - 1 / dt * m_right) * u_center;
        }
      }
      if (v < n - 1) {
        u_next = u[o + v + 1];
        const double h_right = h[v];
        const double k_right = 1. / h_right * (1) * prefactor;
        const double m_right = h_right * 1. / 6;
        if (ie)
          c = (k_right - 1 / dt * m_right);
        else
          c = (k_right / 2. - 1 / dt * m_right);
        const double k_left = 1. / h_right * (-1) * prefactor;
        const double m_left = h_right * 1. / 3;
        if (ie) {
          b += (k_left - 1 / dt * m_left);
          d += (-1 / dt * m_left) * u_center + (-1 / dt * m_right) * u_next;
        } else {
          b += (k_left / 2. - 1 / dt * m_left);
          d += (-k_left / 2. - 1 / dt * m_left) * u_center + (-k_right / 2. - 1 / dt * m_right) * u_next;
        }
      }
      if (v == 0) {
        cp[0] = c / b;
        dp[0] = d / b;
      } else {
        if (v != n - 1)
          cp[v] = c / (b - cp[v - 1] * a);
        dp[v] = (d - dp[v - 1] * a) / (b - cp[v - 1] * a);
      }
    }
    u[o + n - 1] = dp[n - 1];
    double prev = dp[n - 1];
    for (int64_t v = n - 2; v >= 0; v--) {
      const double x = dp[v] - cp[v] * prev;
      u[o + v] = x;
      prev = x;
    }
  }
  free(cp);
  free(dp);
  }
  (void)N;
}

static void build_ranks(const oracle_problem *p, oracle_rank *ranks, const double *states)
{
  const oracle_model *m = &oracle_models[p->model];
  const int W = p->vc_width;
  for (int rk = 0; rk < p->n_ranks; rk++) {
    oracle_rank *r = &ranks[rk];
    memset(r, 0, sizeof(*r));
    for (int f = rk; f < p->n_fibers; f += p->n_ranks)
      r->n_fibers++;
    r->fibers = (int *)malloc(sizeof(int) * (r->n_fibers + 1));
    r->values_offset = (int64_t *)malloc(sizeof(int64_t) * (r->n_fibers + 2));
    int lf = 0;
    int64_t off = 0, max_len = 1;
    for (int f = rk; f < p->n_fibers; f += p->n_ranks, lf++) {
      r->fibers[lf] = f;
      r->values_offset[lf] = off;
      const int64_t n = p->fiber_offsets[f + 1] - p->fiber_offsets[f];
      off += n;
      if (n > max_len)
        max_len = n;
    }
    r->values_offset[lf] = off;
    r->values_offset[lf + 1] = off;
    r->n_values = off;
    r->n_buffers = (off + W - 1) / W;
    const int64_t N = r->n_buffers * W;
    r->node_of = (int64_t *)malloc(sizeof(int64_t) * (N > 0 ? N : 1));
    r->states = (double *)calloc((size_t)(N > 0 ? N : 1) * m->n_states, sizeof(double));
    r->params = (double *)calloc((size_t)(N > 0 ? N : 1) * (m->n_parameters > 0 ? m->n_parameters : 1), sizeof(double));
    r->alg_out = (double *)calloc((size_t)(N > 0 ? N : 1) * (p->n_algebraics_out > 0 ? p->n_algebraics_out : 1), sizeof(double));
    r->c_prime = (double *)malloc(sizeof(double) * max_len);
    r->d_prime = (double *)malloc(sizeof(double) * max_len);
    for (int64_t i = 0; i < N; i++)
      r->node_of[i] = -1;
    const int64_t n_nodes = p->fiber_offsets[p->n_fibers];
    for (lf = 0; lf < r->n_fibers; lf++) {
      const int f = r->fibers[lf];
      const int64_t n = p->fiber_offsets[f + 1] - p->fiber_offsets[f];
      for (int64_t j = 0; j < n; j++) {
        const int64_t i = r->values_offset[lf] + j, g = p->fiber_offsets[f] + j;
        r->node_of[i] = g;
        for (int s = 0; s < m->n_states; s++)
          r->states[s * N + i] = states[s * n_nodes + g];
        for (int q = 0; q < m->n_parameters; q++)
          r->params[q * N + i] = p->parameters[q * n_nodes + g];
      }
    }
    /* padding lanes hold the initial values (initializeStates runs on every buffer) or, for the
     * equilibrium test, the values they reached in earlier runs; their parameters are those of the rank's
     * first instance (initialization.tpp:436-441 fills every lane with them before the fibers' values) */
    for (int64_t i = 0; i < N; i++)
      if (r->node_of[i] < 0) {
        const int lane = (int)(i % W);
        for (int s = 0; s < m->n_states; s++)
          r->states[s * N + i] = (p->equilibrium && p->pad_states)
                                     ? p->pad_states[((int64_t)rk * W + lane) * m->n_states + s]
                                     : m->states_initial[s];
        if (r->n_fibers > 0)
          for (int q = 0; q < m->n_parameters; q++)
            r->params[q * N + i] = p->parameters[q * n_nodes + p->fiber_offsets[r->fibers[0]]];
      }
  }
}

static void free_ranks(const oracle_problem *p, oracle_rank *ranks)
{
  for (int rk = 0; rk < p->n_ranks; rk++) {
    free(ranks[rk].fibers);
    free(ranks[rk].values_offset);
    free(ranks[rk].node_of);
    free(ranks[rk].states);
    free(ranks[rk].params);
    free(ranks[rk].alg_out);
    free(ranks[rk].c_prime);
    free(ranks[rk].d_prime);
  }
}

/* Run RepeatedCall<FastMonodomainSolver> over [t_start, t_end].
 * states: [s][node] in/out.  last_check_time / current_jitter / jitter_index: per fiber stimulation
 * machine state, in/out (initialise with oracle_stimulation_init).  Returns the number of split steps. */
int64_t oracle_run(const oracle_problem *p, double *states, double *last_check_time, double *current_jitter,
                   int *jitter_index)
{
  if (p->model < 0 || p->model >= ORACLE_N_MODELS || p->n_ranks < 1 || p->vc_width < 1)
    return -1;
  const oracle_model *m = &oracle_models[p->model];
  const int64_t n_nodes = p->fiber_offsets[p->n_fibers];
  if (p->equilibrium && p->vc_width > ORACLE_MAX_VC_WIDTH)
    return -1;
  oracle_rank *ranks = (oracle_rank *)calloc(p->n_ranks, sizeof(oracle_rank));
  build_ranks(p, ranks, states);
  uint8_t *local_status = NULL;
  if (p->equilibrium) {
    int64_t total_buffers = 0;
    for (int rk = 0; rk < p->n_ranks; rk++)
      total_buffers += ranks[rk].n_buffers;
    uint8_t *st = p->eq_status;
    if (!st) {
      local_status = (uint8_t *)malloc(total_buffers > 0 ? total_buffers : 1);
      memset(local_status, EQ_ACTIVE, total_buffers > 0 ? total_buffers : 1);
      st = local_status;
    }
    int64_t o = 0;
    for (int rk = 0; rk < p->n_ranks; rk++) {
      ranks[rk].eq_status = st + o;
      ranks[rk].eq_counter = p->eq_counter ? p->eq_counter[rk] : 0;
      o += ranks[rk].n_buffers;
    }
  }
  oracle_fiber_state *fs = (oracle_fiber_state *)calloc(p->n_fibers > 0 ? p->n_fibers : 1, sizeof(oracle_fiber_state));
  for (int f = 0; f < p->n_fibers; f++) {
    fs[f].last_check_time = last_check_time[f];
    fs[f].current_jitter = current_jitter[f];
    fs[f].jitter_index = jitter_index[f];
    fs[f].has_been_stimulated = p->has_been_stimulated ? p->has_been_stimulated[f] : 0;
    fs[f].currently_stimulating = p->currently_stimulating ? p->currently_stimulating[f] : 0;
  }

  /* RepeatedCall (repeated_call.tpp:43-75) */
  oracle_tss rc;
  tss_init(&rc, p->t_start, p->t_end, p->dt_repeated_call);
  tss_set_dt(&rc, p->dt_repeated_call);
  const double span = rc.end - rc.start;
  oracle_tss strang, heun, diff;
  tss_init(&strang, p->t_start, p->t_start + p->dt_splitting, p->dt_splitting);
  tss_init(&heun, p->t_start, p->t_start + p->dt_0d, p->dt_0d);
  tss_init(&diff, p->t_start, p->t_start + p->dt_1d, p->dt_1d);
  int64_t split_no = 0;
  double t = rc.start;
  for (int k = 0; k < rc.n;) {
    tss_set_span(&strang, t, t + rc.dt);
    /* computeMonodomain (compute.tpp:64-129) */
    const double start = strang.start;
    const double dts = strang.dt;
    const int ns = strang.n;
    tss_set_span(&heun, start, start + 0.5 * dts);
    tss_set_span(&diff, start, start + dts);
    const double dt0 = heun.dt, dt1 = diff.dt;
    const int n0 = heun.n;
    for (int j = 0; j < ns; j++) {
      const double tc = start + j * dts;
      const double mid = tc + 0.5 * dts;
      const int store = j == ns - 1;
      for (int rk = 0; rk < p->n_ranks; rk++) {
        oracle_rank *r = &ranks[rk];
        if (r->n_fibers == 0)
          continue;
        if (p->clamp_rule == 0)
          compute0d(p, r, fs, tc, dt0, n0, 0);
        else
          compute0d_center(p, r, fs, tc, dt0, n0, 0);
        /* compute.tpp:261-265: no 1D solve when every buffer of the rank is counted inactive */
        if (!(p->equilibrium && p->clamp_rule == 0 && r->eq_counter == (int)r->n_buffers))
          compute1d(p, r, dt1);
        if (p->clamp_rule == 0)
          compute0d(p, r, fs, mid, dt0, n0, store);
        else
          compute0d_center(p, r, fs, mid, dt0, n0, store);
      }
      if (p->n_trace_nodes > 0 && p->trace && split_no < p->trace_capacity) {
        for (int q = 0; q < p->n_trace_nodes; q++) {
          const int64_t g = p->trace_nodes[q];
          /* find the rank copy of node g */
          double v = NAN;
          for (int rk = 0; rk < p->n_ranks && isnan(v); rk++) {
            oracle_rank *r = &ranks[rk];
            for (int lf = 0; lf < r->n_fibers; lf++) {
              const int f = r->fibers[lf];
              if (g >= p->fiber_offsets[f] && g < p->fiber_offsets[f + 1]) {
                v = r->states[r->values_offset[lf] + (g - p->fiber_offsets[f])];
                break;
              }
            }
          }
          p->trace[split_no * p->n_trace_nodes + q] = v;
        }
      }
      split_no++;
    }
    k++;
    t = rc.start + (double)k / rc.n * span;
  }

  /* copy back */
  for (int rk = 0; rk < p->n_ranks; rk++) {
    oracle_rank *r = &ranks[rk];
    const int64_t N = r->n_buffers * p->vc_width;
    for (int64_t i = 0; i < N; i++) {
      const int64_t g = r->node_of[i];
      if (g < 0)
        continue;
      for (int s = 0; s < m->n_states; s++)
        states[s * n_nodes + g] = r->states[s * N + i];
      for (int q = 0; q < p->n_algebraics_out; q++)
        p->algebraics_out[q * n_nodes + g] = r->alg_out[q * N + i];
    }
  }
  for (int f = 0; f < p->n_fibers; f++) {
    last_check_time[f] = fs[f].last_check_time;
    current_jitter[f] = fs[f].current_jitter;
    jitter_index[f] = fs[f].jitter_index;
    if (p->has_been_stimulated)
      p->has_been_stimulated[f] = fs[f].has_been_stimulated;
    if (p->currently_stimulating)
      p->currently_stimulating[f] = fs[f].currently_stimulating;
  }
  if (p->equilibrium) {
    for (int rk = 0; rk < p->n_ranks; rk++) {
      oracle_rank *r = &ranks[rk];
      if (p->eq_counter)
        p->eq_counter[rk] = r->eq_counter;
      if (p->pad_states) {
        const int W = p->vc_width;
        const int64_t N = r->n_buffers * W;
        for (int64_t i = 0; i < N; i++)
          if (r->node_of[i] < 0)
            for (int s = 0; s < m->n_states; s++)
              p->pad_states[((int64_t)rk * W + (i % W)) * m->n_states + s] = r->states[s * N + i];
      }
    }
    free(local_status);
  }
  free_ranks(p, ranks);
  free(ranks);
  free(fs);
  return split_no;
}

/* The clamp set the vc rule produces for each fiber, for checking the product's host logic:
 * out_first[f] = first clamped global node (or -1), out_count[f] = number of clamped nodes. */
int oracle_vc_clamp_nodes(const oracle_problem *p, int64_t *out_first, int *out_count)
{
  const int W = p->vc_width;
  for (int f = 0; f < p->n_fibers; f++) {
    out_first[f] = -1;
    out_count[f] = 0;
  }
  for (int rk = 0; rk < p->n_ranks; rk++) {
    int nf = 0;
    for (int f = rk; f < p->n_fibers; f += p->n_ranks)
      nf++;
    if (nf == 0)
      continue;
    int *fib = (int *)malloc(sizeof(int) * nf);
    int64_t *vo = (int64_t *)malloc(sizeof(int64_t) * (nf + 1));
    int64_t off = 0;
    int lf = 0;
    for (int f = rk; f < p->n_fibers; f += p->n_ranks, lf++) {
      fib[lf] = f;
      vo[lf] = off;
      off += p->fiber_offsets[f + 1] - p->fiber_offsets[f];
    }
    vo[nf] = off;
    const int64_t nb = (off + W - 1) / W;
    const double factor = (double)W / (double)(vo[1] - vo[0]);
    for (int64_t b = 0; b < nb; b++) {
      int local = (int)(b * factor);
      if (local >= nf)
        local = nf - 1;
      const int f = fib[local];
      const int64_t index_in_fiber = b * W - vo[local];
      const int center = p->stimulation_point_index[f];
      if ((unsigned long)((long)center - (long)index_in_fiber) < (unsigned long)W) {
        /* lanes 0..min(3,W)-1 of buffer b, as rank-local indices, mapped to global nodes */
        const int cnt = W < 3 ? W : 3;
        int64_t first = -1;
        int c = 0;
        for (int lane = 0; lane < cnt; lane++) {
          const int64_t i = b * W + lane;
          /* map rank-local index to global */
          for (int l2 = 0; l2 < nf; l2++)
            if (i >= vo[l2] && i < vo[l2 + 1]) {
              const int64_t g = p->fiber_offsets[fib[l2]] + (i - vo[l2]);
              if (first < 0)
                first = g;
              c++;
              break;
            }
        }
        out_first[f] = first;
        out_count[f] = c;
      }
    }
    free(fib);
    free(vo);
  }
  return 0;
}
