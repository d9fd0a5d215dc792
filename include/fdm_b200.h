/* fdm_b200 — B200-native fiber monodomain solver, C ABI.
 *
 * This is the drop-in boundary for OpenDiHu's FastMonodomainSolver hot path
 * (core/src/specialized_solver/fast_monodomain_solver/).  Plain C types only: pointers, sizes and
 * int status codes; every array is a HOST array unless its name says "device".
 *
 * Reference interfaces replaced:
 *  - fdm_create / fdm_set_* / fdm_advance / fdm_get_* replace the generated-library ABI the reference
 *    loads with dlopen/dlsym, `initializeArrays(...)` and `computeMonodomain(...)`
 *    (fast_monodomain_solver_gpu.tpp:361-365, :478-481, :187-196), whose sizes the reference bakes into
 *    generated source (gpu.tpp:293-312); here sizes are run-time arguments.
 *  - fdm_advance(t_start, t_end) is RepeatedCall<FastMonodomainSolver>::advanceTimeSpan
 *    (repeated_call.tpp:43-80) driving FastMonodomainSolverBase::setTimeSpan + advanceTimeSpan
 *    (fast_monodomain_solver_compute.tpp:14-129).
 *  - fdm_checkpoint_save / fdm_checkpoint_restore are saveFiberDataCheckpoint /
 *    restoreFiberDataCheckpoint (fast_monodomain_solver_communication.tpp:497-509).
 *  - fdm_get_algebraics returns algebraicsForTransfer (03_generator_vc.cpp:1131-1160).
 *  - fdm_compat_configure + initializeArrays + computeMonodomain (end of this header) export the reference's
 *    generated-library symbols with their exact signatures (fast_monodomain_solver_gpu.tpp:361-365, :478-481).
 *
 * Errors: every function returns FDM_OK (0) or a positive FDM_ERR_* code; fdm_last_error() gives the
 * message.  Nothing aborts the process.  One solver handle must not be used from two host threads
 * at once; different handles are independent (each owns its CUDA stream and device memory).
 */
#ifndef FDM_B200_H
#define FDM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDM_OK 0
#define FDM_ERR_ARG 1          /* invalid argument or call order */
#define FDM_ERR_CUDA 2         /* a CUDA call failed (message has the CUDA error string) */
#define FDM_ERR_NAN 3          /* NaN or Inf in the transmembrane potential after an advance */
#define FDM_ERR_UNSUPPORTED 4  /* combination not built into this library */
#define FDM_ERR_NO_DEVICE 5    /* no CUDA device */
#define FDM_ERR_TIMEOUT 6      /* a wait gave up before the device finished (fdm_wait_for) */

#define FDM_MODEL_HODGKIN_HUXLEY_1952 0
#define FDM_MODEL_SHORTEN_2007 1

#define FDM_IMPLICIT_EULER 0
#define FDM_CRANK_NICOLSON 1

#define FDM_METHOD_SPLIT 0     /* reaction kernel + diffusion kernel per half/full step, states in HBM */
#define FDM_METHOD_FUSED 1     /* one persistent kernel per window, states resident on chip */

#define FDM_FP64 0
#define FDM_FP32_REACTION 1    /* rates and gates in FP32; Vm accumulation and diffusion in FP64 */

#define FDM_CLAMP_VC_LANES 0   /* lanes 0..min(3,W)-1 of the W-wide buffer holding the junction ("vc") */
#define FDM_CLAMP_CENTER 1     /* junction node and its two neighbours ("gpu") */

#define FDM_STIMULUS_CLAMP 0   /* Vm := valueForStimulatedPoint on stimulated nodes (reference) */
#define FDM_STIMULUS_CURRENT 1 /* parameter stimulus_parameter := stimulus_value on stimulated nodes */

typedef struct fdm_solver fdm_solver;

typedef struct fdm_config {
  int model;                     /* FDM_MODEL_* */
  int diffusion_scheme;          /* FDM_IMPLICIT_EULER / FDM_CRANK_NICOLSON */
  int method;                    /* FDM_METHOD_* */
  int reaction_precision;        /* FDM_FP64 / FDM_FP32_REACTION */
  int approximate_exponential_function; /* 1: exp(x) ~ (1+x/1024)^1024 as the reference's "vc" code */
  int clamp_rule;                /* FDM_CLAMP_* */
  int vc_width;                  /* W of the FDM_CLAMP_VC_LANES rule (4 = AVX2 build of the reference) */
  int n_ranks;                   /* fibers are laid out as on n_ranks ranks (fiberNo % n_ranks) for the clamp rule */
  int stimulus_mode;             /* FDM_STIMULUS_* */
  int stimulus_parameter;        /* parameter index for FDM_STIMULUS_CURRENT */
  double stimulus_value;
  double value_for_stimulated_point;   /* "valueForStimulatedPoint", default 20 */
  double dt_repeated_call;       /* RepeatedCall timeStepWidth */
  double dt_splitting;           /* Strang timeStepWidth */
  double dt_0d;                  /* Heun timeStepWidth */
  double dt_1d;                  /* ImplicitEuler / CrankNicolson timeStepWidth */
  int steps_per_launch;          /* split steps per launch window, 0 = default */
  int threads_per_block;         /* fused kernel CTA size, 0 = choose */
  int nodes_per_thread;          /* fused kernel nodes per thread, 0 = choose */
  int check_nan;                 /* 1: fdm_advance fails with FDM_ERR_NAN if Vm is not finite */
  int profile;                   /* 1: time the main kernel launches with CUDA events */
  int device;                    /* CUDA device ordinal the solver lives on */
  int use_graph;                 /* 1: the split path replays each window's launch sequence as a CUDA graph */
  int only_compute_if_stimulated; /* "onlyComputeIfHasBeenStimulated" (compute.tpp:201-205): a node's Heun
                                     substeps are skipped while the fiber its point buffer is attributed to
                                     has not been stimulated (0: every node computed, the parity setting) */
  int skip_close_to_equilibrium;  /* "disableComputationWhenStatesAreCloseToEquilibrium" (compute.tpp:130-265,
                                     630-797): point buffers whose states stop changing are skipped and a rank
                                     whose buffers are all counted inactive skips its diffusion solve; split
                                     method with the vc clamp rule only (0: off, the parity setting) */
  int cluster_size;               /* fused method: a fiber spread over this many CTAs of one thread-block cluster
                                     (2..8; HH, exact exponentials, every node computed), for few fibers that
                                     would leave most SMs idle; 0 = chosen automatically, 1 = off */
} fdm_config;

/* fills *cfg with the reference's defaults (HH, implicit Euler, FP64 split, vc rule W=4, 20 mV clamp) */
void fdm_config_default(fdm_config *cfg);

int fdm_create(const fdm_config *cfg, fdm_solver **out);
int fdm_destroy(fdm_solver *s);
/* message of the last failed call on s (or of the last failed fdm_create if s is NULL) */
const char *fdm_last_error(const fdm_solver *s);

/* Loads a run-time model module: a shared library compiled from a generated translation unit for one CellML
 * model or parameter variant that is not built into this library (opendihu_b200/csrc/fdm_model_module.cuh;
 * the Python settings layer generates and compiles it on demand, as the reference generates, compiles and
 * dlopens a library from the model file: fast_monodomain_solver_gpu.tpp:106-205, the CellmlAdapter's
 * libraryFilename option).  *model_id receives the number to pass as fdm_config.model (a module loaded again
 * keeps its number).  Module models run the split method, the equilibrium skip and the adjoint; the fused
 * method is built for the library's own models only. */
int fdm_register_model_library(const char *path, int *model_id);

/* model description: sizes and initial state values of the model's OpenCOR file */
int fdm_model_info(int model, int *n_states, int *n_algebraics, int *n_parameters, double *states_initial);
/* default value of every parameter slot: the raw CONSTANTS value for a constant parameter, 0 for an
 * algebraic one (00_source_code_generator_base.cpp:67-81 fills missing parameters the same way) */
int fdm_model_parameter_defaults(int model, double *defaults);

/* Fibers: fiber_offsets[n_fibers+1] node offsets (fiber f owns nodes [off[f], off[f+1]), at least 2 nodes);
 * element_lengths: fiber f's off[f+1]-off[f]-1 element lengths, concatenated in fiber order;
 * prefactor[n_fibers]: sigma/(Am*Cm) per fiber ("prefactor" of the diffusion FEM settings).
 * Resets states to the model's initial values and parameters to the model's defaults. */
int fdm_set_fibers(fdm_solver *s, int n_fibers, const int64_t *fiber_offsets, const double *element_lengths,
                   const double *prefactor);
int fdm_set_prefactor(fdm_solver *s, const double *prefactor);

/* parameters[p * n_nodes + node] (SoA, "parametersInitialValues" per instance) */
int fdm_set_parameters(fdm_solver *s, const double *parameters);
int fdm_get_parameters(fdm_solver *s, double *parameters);

/* states[state * n_nodes + node] (SoA); state 0 is Vm.  Host arrays from fdm_host_alloc are transferred
 * directly (the other states converted on the device); other host memory goes through pinned staging, with
 * the host copies overlapping the transfers.  Both forms give bit-identical results. */
int fdm_set_states(fdm_solver *s, const double *states);
int fdm_get_states(fdm_solver *s, double *states);

/* Page-locked host memory for state arrays (the reference keeps its fiber data in host vectors,
 * fast_monodomain_solver_initialization.tpp:145-347, and copies them in and out every call,
 * gpu.tpp:478-481): *ptr receives `bytes` of pinned memory the transfers use without staging.
 * fdm_host_free releases it (FDM_ERR_ARG for a pointer fdm_host_alloc did not return). */
int fdm_host_alloc(size_t bytes, void **ptr);
int fdm_host_free(void *ptr);
int fdm_get_vm(fdm_solver *s, double *vm);

/* Stimulation inputs (fast_monodomain_solver_initialization.tpp:145-347):
 *  firing_events[rows*cols] (0/1, the firingTimesFile), motor_unit_no[f], stimulation_point_index[f]
 *  (NMJ node within the fiber), call_frequency[f], repeat_after_first_call[f], call_enable_begin[f],
 *  jitter[f*n_jitter + k] (setSpecificStatesFrequencyJitter). Resets the stimulation state machine. */
int fdm_set_stimulation(fdm_solver *s, const uint8_t *firing_events, int rows, int cols, const int *motor_unit_no,
                        const int *stimulation_point_index, const double *call_frequency,
                        const double *repeat_after_first_call, const double *call_enable_begin,
                        const double *jitter, int n_jitter);
/* per fiber: first clamped node (global index, -1 if none), number of clamped nodes, machine evaluated */
int fdm_get_clamp_nodes(fdm_solver *s, int64_t *first_node, int *count, uint8_t *evaluated);
/* replaces the clamp nodes fdm_set_stimulation chose (e.g. with a selection made for a larger layout) */
int fdm_set_clamp_nodes(fdm_solver *s, const int64_t *first_node, const int *count, const uint8_t *evaluated);
/* disableComputationWhenStatesAreCloseToEquilibrium: the number of point buffers (all ranks, rank after rank),
 * their statuses (0 inactive, 1 neighbor_is_active, 2 active; may be NULL) and the per-rank counts of
 * inactive buffers (n_ranks entries; may be NULL) -- the "computeStateInformation" data of
 * fast_monodomain_solver_communication.tpp:280-290 */
int fdm_get_equilibrium_state(fdm_solver *s, int64_t *n_buffers, uint8_t *status, int *counter);
/* "computeStateInformation" per node (the extra transfer slot, communication.tpp:277-290): the status of the
 * node's point buffer (0 inactive, 1 neighbor_is_active, 2 active; 2 everywhere while the equilibrium skip
 * is off), -1 on the nodes of a fiber not stimulated yet under onlyComputeIfHasBeenStimulated */
int fdm_get_compute_state_information(fdm_solver *s, double *out /* [n_nodes] */);
/* host-only: per node, the code (attributed fiber) * 4 + class that onlyComputeIfHasBeenStimulated uses:
 * class 0/1/2 = the node's point buffer lies before / is / lies after the junction buffer of the fiber it
 * is attributed to (compute.tpp:158-205 processes buffers in order and the junction buffer sets the flag) */
int fdm_select_gate_codes(int clamp_rule, int vc_width, int n_ranks, int n_fibers, const int64_t *fiber_offsets,
                          const int *stimulation_point_index, int *codes);
/* replaces the codes fdm_set_stimulation chose (a selection made for a larger layout) */
int fdm_set_gate_codes(fdm_solver *s, const int *codes);
/* host-only: the clamp nodes of a fiber layout under a rule (the selection fdm_set_stimulation makes) */
int fdm_select_clamp_nodes(int clamp_rule, int vc_width, int n_ranks, int n_fibers, const int64_t *fiber_offsets,
                           const int *stimulation_point_index, int64_t *first_node, int *count, uint8_t *evaluated);

/* which algebraics to return after each advance ("algebraicsForTransfer") */
int fdm_set_algebraics_for_transfer(fdm_solver *s, int n, const int *algebraic_indices);
int fdm_get_algebraics(fdm_solver *s, double *out /* [k * n_nodes + node] */);

/* record Vm at the given nodes after every split step (for activation times); capacity in split steps; the
 * rows count the split steps from this call on (row 0 = the first step after it) */
int fdm_set_trace(fdm_solver *s, int n_nodes, const int64_t *nodes, int64_t capacity);
int fdm_get_trace(fdm_solver *s, double *out /* [step * n_nodes + k] */, int64_t *n_steps_recorded);
/* Activation recording on the traced nodes (no counterpart in the reference; its scripts find activation
 * times in the written Vm): after each Strang step, a traced node whose Vm rose above threshold (Vm after the
 * previous step <= threshold < Vm now) records the step's trace row (Strang steps since fdm_set_trace, 0 =
 * the first).  The first capacity_per_node rows per node are kept, every crossing is counted; the step right
 * after the recording starts never records.  0 turns it off; fdm_set_trace turns it off (call this after). */
int fdm_set_activation_recording(fdm_solver *s, double threshold, int capacity_per_node);
/* counts[k] = crossings of traced node k; steps[k * capacity_per_node + j] = its j-th row (-1: none) */
int fdm_get_activation_steps(fdm_solver *s, int *counts, int *steps);

/* RepeatedCall over [t_start, t_end]: blocking; returns after the device finished. */
int fdm_advance(fdm_solver *s, double t_start, double t_end);
/* the same, returning once the work is enqueued on the solver's stream (no counterpart in the reference,
 * whose calls are synchronous): the host can prepare other work meanwhile.  fdm_wait completes it (timing,
 * the NaN check of check_nan); every other call on the solver orders after the enqueued work, the next
 * advance waits first. */
int fdm_advance_async(fdm_solver *s, double t_start, double t_end);
int fdm_wait(fdm_solver *s);
/* fdm_wait with a limit (no counterpart in the reference, whose calls block without one): polls the solver's
 * stream for at most timeout_seconds; FDM_ERR_TIMEOUT if the advance is still running then (it stays enqueued
 * and the solver usable: a later fdm_wait or fdm_wait_for completes it), otherwise as fdm_wait.  For callers
 * that must notice a device that stopped making progress without blocking on it forever. */
int fdm_wait_for(fdm_solver *s, double timeout_seconds);
/* The RepeatedCall pieces of [t_start, t_end] (repeated_call.tpp:43-80: piece k is one call of
 * FastMonodomainSolver::advanceTimeSpan, after which the reference calls the diffusion's output writers,
 * fast_monodomain_solver_compute.tpp:35-44): their number, and, when steps_per_piece is not null, the number
 * of split steps of each (the writers' callCountIncrement), planned from the solver's current time-stepping
 * state without changing it. */
int fdm_repeated_call_plan(fdm_solver *s, double t_start, double t_end, int64_t *n_pieces, int *steps_per_piece);
/* advances the pieces k_begin <= k < k_end of that span (blocking): consecutive ranges covering all pieces
 * give the same steps, bit for bit, as one fdm_advance over the span, with the host free between them
 * (output at the reference's times) */
int fdm_advance_pieces(fdm_solver *s, double t_start, double t_end, int64_t k_begin, int64_t k_end);
/* Stimulation log (the reference's StimulationLogging, core/src/control/diagnostic_tool/stimulation_logging.cpp,
 * fed at fast_monodomain_solver_compute.tpp:603-607): from now on every substep at which a fiber's stimulation
 * begins (its decision stimulates, its previous decision did not) is recorded as (time, fiber), up to capacity
 * entries.  A larger capacity keeps the entries recorded so far; 0 turns the log off and drops them. */
int fdm_set_stimulation_log(fdm_solver *s, int64_t capacity);
/* *n_total = stimulation begins recorded; times/fibers (may be null) receive all n_total of them, in the order
 * they were recorded (fibers of one window in no fixed order).  If more begins happened than the capacity
 * held, *n_total still counts them all, nothing is copied and the call fails with FDM_ERR_ARG (the log is
 * incomplete): grow the capacity before each advance to what its span can need.  With times and fibers both
 * null the call only counts (it does not fail on an incomplete log). */
int fdm_get_stimulation_log(fdm_solver *s, int64_t *n_total, double *times, int *fibers);
/* number of split steps done by all advances so far */
int64_t fdm_split_steps(const fdm_solver *s);
/* Fault injection for tests (no counterpart in the reference): the k-th allocation of solver memory (device
 * buffers and pinned host staging, any solver of this process) from now on fails as if the device were out of
 * memory; k = 0 turns it off.  The call that meets the failure returns FDM_ERR_CUDA and leaves the solver safe:
 * a failed fdm_set_fibers leaves it without fibers, a failed fdm_set_stimulation, fdm_set_trace,
 * fdm_set_algebraics_for_transfer or fdm_checkpoint_save leaves that setting unset, a failed advance can be
 * repeated; fdm_destroy always releases what was allocated. */
int fdm_debug_fail_allocation(int64_t k);
/* summed device time and count of the main kernel launches (config.profile = 1), and of all GPU work
 * of the advances */
int fdm_get_timing(const fdm_solver *s, double *main_kernel_ms, int64_t *main_kernel_launches,
                   double *advance_ms, int64_t *kernel_launches);
int fdm_reset_timing(fdm_solver *s);

/* back to the start of the simulation: time-stepping state, Strang step counter and stimulation machine as
 * right after fdm_set_stimulation (states and parameters are kept) */
int fdm_rewind(fdm_solver *s);

int fdm_checkpoint_save(fdm_solver *s);
int fdm_checkpoint_restore(fdm_solver *s);

/* One diffusion solve of compute1D (fast_monodomain_solver_compute.tpp:256-507) for every fiber, as a
 * standalone operator on DEVICE arrays of the current CUDA device: d_fiber_offsets[n_fibers+1] (node offsets),
 * d_element_lengths (each fiber's n_f-1 lengths, concatenated), d_prefactor[n_fibers], d_vm[n_nodes] (in: u,
 * out: u+).  diffusion_scheme is FDM_IMPLICIT_EULER or FDM_CRANK_NICOLSON, dt the diffusion step width.
 * Scratch memory (7 doubles per node) is allocated by the library with cudaMalloc and kept for later calls.
 * stream is a cudaStream_t (NULL: the legacy default stream); the call returns after the solve. */
int fdm_diffusion_solve(int n_fibers, int64_t n_nodes, const int64_t *d_fiber_offsets, const double *d_element_lengths,
                        const double *d_prefactor, double dt, int diffusion_scheme, double *d_vm, void *stream);

/* fdm_diffusion_solve without any device allocation; no counterpart in the reference.  For callers that
 * cannot allocate device memory while they run (an application whose memory pool owns the whole GPU, a
 * coupled code that has reserved HBM for its own mesh, a stepping loop that must not synchronize on
 * cudaMalloc/cudaFree).  The scratch is one array compiled into the library, sized for at most
 * FDM_NOALLOC_MAX_NODES nodes (14.7 MB held on every GPU that loads the library until the process exits);
 * larger n_nodes fail with FDM_ERR_ARG.  The fiber offsets index that array: they must not decrease and must
 * lie in [0, n_nodes] (d_fiber_offsets[n_fibers] <= n_nodes); the call reads their first and last entry back
 * and fails with FDM_ERR_ARG when either end is outside.  The first call on a device looks the array's
 * address up; make it before any stream capture.  All calls share the array: calls that overlap on the GPU
 * race, so order them on one stream.  Arguments and result as fdm_diffusion_solve. */
#define FDM_NOALLOC_MAX_NODES 262144
int fdm_diffusion_solve_noalloc(int n_fibers, int64_t n_nodes, const int64_t *d_fiber_offsets,
                                const double *d_element_lengths, const double *d_prefactor, double dt,
                                int diffusion_scheme, double *d_vm, void *stream);

/* ---- adjoint (no counterpart in the reference: the differentiation extension) ----------------------
 * Discrete reverse mode of the FP64 split path (method FDM_METHOD_SPLIT, FDM_FP64).
 * fdm_adjoint_forward: advances over [t_start, t_end] like fdm_advance, records Vm at the sensor nodes after
 *   every Strang step (read with fdm_get_trace) and saves a checkpoint every checkpoint_every steps.
 * fdm_adjoint_backward: given trace_grad[step * n_sensors + k] = dL/dVm(sensor k, after step), returns
 *   dL/dprefactor[fiber], dL/dparameters[p * n_nodes + node] and dL/dstates(t_start)[s * n_nodes + node] (any of
 *   the three may be NULL).  Each checkpoint segment is replayed storing every Heun substep's input state, then
 *   reversed: Heun steps through the generated vector-Jacobian product of the model, the diffusion solve through
 *   the transposed (= same, symmetric) tridiagonal system.  The solver then continues from the forward run's end. */
int fdm_adjoint_forward(fdm_solver *s, double t_start, double t_end, int checkpoint_every, int n_sensors,
                        const int64_t *sensor_nodes);
int fdm_adjoint_backward(fdm_solver *s, const double *trace_grad, double *grad_prefactor, double *grad_parameters,
                         double *grad_states0);
int fdm_adjoint_release(fdm_solver *s);
/* device time of the adjoint backward passes so far (ms) */
int fdm_adjoint_timing(const fdm_solver *s, double *backward_ms);

/* number of the fused-kernel shapes built into the library and their (threads, nodes per thread) */
int fdm_fused_shapes(int *threads, int *nodes_per_thread, int capacity);
/* the same for the cluster mode of the fused kernel (a fiber spread over up to 8 CTAs of one cluster) */
int fdm_fused_cluster_shapes(int *threads, int *nodes_per_thread, int capacity);
/* the fused launch fdm_set_fibers chose: CTA size, nodes per thread, CTAs per fiber (1: bins of whole
 * fibers, > 1: cluster mode), number of CTAs */
int fdm_fused_layout(const fdm_solver *s, int *threads, int *nodes_per_thread, int *cluster_size, int *n_blocks);

/* ---- fibers -> 3D static bidomain (EMG) -------------------------------------------------------------
 * The caller downstream of the fiber solver in the reference's fibers_emg example (fast_fibers_emg.cpp:17-63:
 * Control::Coupling of the FastMonodomainSolver with TimeSteppingScheme::StaticBidomainSolver,
 * static_bidomain_solver.tpp).  Structured hexahedral mesh with trilinear elements: node_positions[n][3] for
 * the nx*ny*nz nodes numbered i + nx*(j + ny*k); element dofs in the reference's order (x fastest).
 * fdm_emg_potential_flow: Laplace with Dirichlet values ("PotentialFlow", static_bidomain_solver.tpp:102-130),
 *   nodal gradients averaged over adjacent elements and normalised into the fiber direction
 *   (08_field_variable_gradient.tpp:59-115); or fdm_emg_set_direction gives the directions.
 * fdm_emg_set_conductivity: "diffusionTensor" sigma_i and "extracellularDiffusionTensor" sigma_e (9 values,
 *   row-major, in fiber coordinates: first axis along the fiber), one for all elements or one per element;
 *   assembles K(sigma_i) and K(sigma_i + sigma_e) with the tensors rotated onto the interpolated direction
 *   (diffusion_tensor_directional.tpp:72-110) and gauss_points^3 Gauss points per element.
 * fdm_emg_set_fiber_mapping: positions[n_source][3] of the fiber nodes (in the fiber solver's node order);
 *   each node inside an element (xi outside [0,1] by at most xi_tolerance, <= 0: 0.1) adds phi_m(xi) times its
 *   value to the element's 8 nodes, each 3D node divides by its factor sum (|sum| <= 1e-12: default_value)
 *   (mapping_between_meshes 00_construct.tpp:90-160, 03_manager_implementation.tpp:239-300).
 * fdm_emg_map_fibers: maps the fiber solver's current Vm (on the device, ordered after its work);
 *   fdm_emg_map_values maps host values; fdm_emg_set_vm sets the 3D Vm directly.
 * fdm_emg_solve: K(sigma_i + sigma_e) phi_e = -K(sigma_i) Vm (static_bidomain_solver.tpp:37-55), constants as
 *   null space, conjugate gradients with a Jacobi preconditioner until ||r||_2 <= max(rtol ||b||_2, atol);
 *   phi_e is the zero-mean solution; initial_guess_nonzero starts from the previous phi_e. */
typedef struct fdm_emg fdm_emg;
#define FDM_EMG_PHI_E 0          /* extracellular potential phi_e [N] */
#define FDM_EMG_VM 1             /* transmembrane potential on the 3D mesh [N] */
#define FDM_EMG_RHS 2            /* -K(sigma_i) Vm [N] */
#define FDM_EMG_FLOW_POTENTIAL 3 /* potential flow solution [N] */
#define FDM_EMG_DIRECTION 4      /* fiber direction [N][3] */
int fdm_emg_create(int nx, int ny, int nz, const double *node_positions, int device, fdm_emg **out);
int fdm_emg_destroy(fdm_emg *m);
const char *fdm_emg_last_error(const fdm_emg *m);
int fdm_emg_potential_flow(fdm_emg *m, int64_t n_dirichlet, const int64_t *nodes, const double *values,
                           int gauss_points, double rtol, double atol, int max_iterations, int *iterations);
int fdm_emg_set_direction(fdm_emg *m, const double *direction /* [N][3] */);
int fdm_emg_set_conductivity(fdm_emg *m, int64_t n_sigma_i, const double *sigma_i, int64_t n_sigma_e,
                             const double *sigma_e, int gauss_points);
int fdm_emg_set_fiber_mapping(fdm_emg *m, int64_t n_source, const double *positions, double xi_tolerance,
                              double default_value, int64_t *n_mapped);
int fdm_emg_map_fibers(fdm_emg *m, fdm_solver *s);
int fdm_emg_map_values(fdm_emg *m, const double *fiber_values);
int fdm_emg_set_vm(fdm_emg *m, const double *vm);
int fdm_emg_solve(fdm_emg *m, double rtol, double atol, int max_iterations, int initial_guess_nonzero,
                  int *iterations, double *residual);
/* preconditioner of the bidomain solve ("preconditionerType"): Jacobi, or (default) a geometric multigrid
 * V-cycle (structured coarsening by 2, Galerkin coarse operators, two damped-Jacobi sweeps before and after);
 * levels: the number of grid levels (1 for Jacobi; the hierarchy is built once the operators exist) */
#define FDM_EMG_PRECOND_JACOBI 0
#define FDM_EMG_PRECOND_MULTIGRID 1
int fdm_emg_set_preconditioner(fdm_emg *m, int type, int *levels);
int fdm_emg_get(fdm_emg *m, int field, double *out);
/* the assembled stencils, coef[q * N + node] with q = (dx+1) + 3(dy+1) + 9(dz+1); which: 0 K(sigma_i),
 * 1 K(sigma_i + sigma_e) */
int fdm_emg_get_stencil(fdm_emg *m, int which, double *out /* [27 * N] */);
/* device time, iterations and residual norm of the last fdm_emg_solve */
int fdm_emg_timing(const fdm_emg *m, double *last_solve_ms, int *last_iterations, double *last_residual);

/* ---- compatibility export of the reference's generated-library ABI ---------------------------------
 * The reference's FastMonodomainSolver with optimizationType "gpu" dlopens a library and binds
 * initializeArrays and computeMonodomain (fast_monodomain_solver_gpu.tpp:185-196); pointing its
 * "libraryFilename" at libfdm_b200.so makes it use this solver.  The reference bakes the sizes into the
 * generated source (gpu.tpp:293-312); here fdm_compat_configure gives them first.  The nodes use the clamp set
 * of the reference's GPU code (junction node and its neighbours); parameters fill the model's first
 * parameter slots.  One process-wide instance; fdm_compat_release frees it. */
int fdm_compat_configure(int model, int n_fibers, int n_instances_per_fiber, int n_parameters_per_instance,
                         int firing_rows, int firing_cols, int n_jitter_per_fiber, int n_algebraics_for_transfer,
                         int n_states_for_transfer, int diffusion_scheme, int approximate_exponential_function,
                         int reaction_precision, int method);
/* The CellmlAdapter's generic right-hand side (the non-fast nested solver path), structure of arrays
 * var[index * n_instances + i] as the reference's generated "gpu" source (04_generator_gpu.cpp:13-113):
 * states[n_states * n], parameters[n_parameters * n] (the variant's parameter slots) in; rates[n_states * n]
 * and algebraics[n_algebraics * n] (may be NULL) out.  Device pointers, on stream (a cudaStream_t, NULL:
 * the legacy default stream). */
int fdm_cellml_rhs_device(int model, int approximate_exponential_function, int64_t n_instances, double t,
                          const double *states, const double *parameters, double *rates, double *algebraics,
                          void *stream);
/* "initializeStatesToEquilibrium" of the CellmlAdapter (03_cellml_adapter.tpp:445-515): classical RK4 steps of one
 * instance with the given parameters, from states (in/out, host) until no state increment exceeds 1e-5, dt halved
 * and the search restarted from the initial values whenever one exceeds 1e4, at most 1e7 steps; computed on the
 * device.  *iterations, *max_increment and *dt_final (each may be null) report the search; the result is FDM_OK
 * also when it did not converge (the reference then logs an error and keeps the last values). */
int fdm_model_equilibrium(int model, int device, int approximate_exponential_function, const double *parameters,
                          double dt, double *states, int64_t *iterations, double *max_increment, double *dt_final);
/* the reference's generated entry point with its signature (04_generator_gpu.cpp:25-26), host arrays, sized by a
 * preceding fdm_cellml_rhs_configure (the reference bakes n_instances into the source); process-wide */
int fdm_cellml_rhs_configure(int model, int64_t n_instances, int approximate_exponential_function, int device);
void computeCellMLRightHandSide(void *context, double t, double *states, double *rates, double *algebraics,
                                double *parameters);
/* fast_monodomain_solver_gpu.tpp:361-365 */
void initializeArrays(const double *statesOneInstance, const int *algebraicsForTransferIndices,
                      const int *statesForTransferIndices, const char *firingEvents,
                      const double *setSpecificStatesFrequencyJitter, const int *motorUnitNo,
                      const int *fiberStimulationPointIndex, const double *lastStimulationCheckTime,
                      const double *setSpecificStatesCallFrequency, const double *setSpecificStatesRepeatAfterFirstCall,
                      const double *setSpecificStatesCallEnableBegin);
/* fast_monodomain_solver_gpu.tpp:478-481 */
void computeMonodomain(const float *parameters, double *algebraicsForTransfer, double *statesForTransfer,
                       const float *elementLengths, double startTime, double timeStepWidthSplitting,
                       int nTimeStepsSplitting, double dt0D, int nTimeSteps0D, double dt1D, int nTimeSteps1D,
                       double prefactor, double valueForStimulatedPoint);
int fdm_compat_release(void);

#ifdef __cplusplus
}
#endif
#endif /* FDM_B200_H */
