// Internal launch interface between the host solver (fdm_host.cu) and the kernel translation units.
// Every launcher is a plain C++ function taking device pointers and a stream.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "fdm_kernels.cuh"
#include "fdm_equilibrium.cuh"

namespace fdm {

// records msg as the message fdm_last_error(NULL) returns on this thread; returns code
int fdm_report_error(int code, const std::string& msg);

enum MathKind { MATH_EXACT = 0, MATH_APPROX = 1 };
enum RealKind { REAL_F64 = 0, REAL_F32 = 1 };

struct ModelDesc {
  const char* name;
  int n_states, n_algebraics, n_parameters;
  const double* states_initial;
  const double* parameter_defaults;
  bool fused_supported;
};

// model table (fdm_kernels_split.cu): the built-in models, then the registered run-time model modules
int n_models();
const ModelDesc* model_desc(int model);

// A run-time model module: a shared library built from a generated translation unit (fdm_model_module.cuh)
// that holds the kernels of one further CellML model or parameter variant.  Its entry point
// fdm_model_module_v1 fills this table; abi must equal FDM_MODEL_MODULE_ABI of the library that loads it (the
// argument structures the two pass between them must have the same layout).
struct ModelModule {
  int abi;
  ModelDesc desc;
  cudaError_t (*reaction)(RealKind rk, MathKind mk, const ReactionArgs& a, cudaStream_t s);
  cudaError_t (*cellml_rhs)(MathKind mk, int64_t n, double t, const double* states, const double* params,
                            double* rates, double* algebraics, cudaStream_t s);
  cudaError_t (*equilibrium_search)(MathKind mk, double* u, const double* u0, const double* params,
                                    EquilibriumSearch* es, int64_t max_iterations, cudaStream_t s);
  cudaError_t (*reaction_eq)(RealKind rk, MathKind mk, const ReactionArgs& a, const EqLayout& L, const EqSpec& e,
                             cudaStream_t s);
  cudaError_t (*adjoint_half)(MathKind mk, const AdjointArgs& a, cudaStream_t s);
};
#define FDM_MODEL_MODULE_ABI                                                                                     \
  (int)(1000000 + 97 * sizeof(fdm::ReactionArgs) + 89 * sizeof(fdm::AdjointArgs) + 83 * sizeof(fdm::EqLayout) +   \
        79 * sizeof(fdm::EqSpec) + 73 * sizeof(fdm::ModelDesc) + 71 * sizeof(fdm::EquilibriumSearch) +            \
        67 * sizeof(fdm::SplitStep))
typedef int (*ModelModuleEntry)(ModelModule* out);
// registers a module's table; returns its model number (after the built-in ones) or -1
int register_model_module(const ModelModule& m);

// split path
cudaError_t launch_reaction(int model, RealKind rk, MathKind mk, const ReactionArgs& a, cudaStream_t s);
// at most max_iterations RK4 steps of the equilibrium search of one instance (u in/out, u0 the initial values)
cudaError_t launch_equilibrium_search(int model, MathKind mk, double* u, const double* u0, const double* params,
                               EquilibriumSearch* es, int64_t max_iterations, cudaStream_t s);
cudaError_t launch_schedule(const StimArgs& a, const SplitStep* steps, int n_steps, cudaStream_t s);
// FP64 states <-> FP32 (value, residual) pairs on the device: hi = (float)x, lo = (float)(x - hi); x = hi + lo
// (the same expressions as the host conversions of the staged transfers, so both give the same bits)
cudaError_t launch_states_to_pairs(const double* x, float* hi, float* lo, int64_t n, cudaStream_t s);
cudaError_t launch_pairs_to_states(const float* hi, const float* lo, double* x, int64_t n, cudaStream_t s);
cudaError_t launch_coefficients(int n_fibers, const int64_t* fiber_offsets, const double* element_lengths, const double* prefactor, double dt, int implicit_euler,
                                double* coef, int64_t stride, cudaStream_t s);
// one diffusion solve of every fiber in place on vm (scratch: one double per node): a warp per fiber, or a
// CTA per fiber when the fibers are few
cudaError_t launch_diffusion(int n_fibers, const int64_t* fiber_offsets, const double* coef, int64_t stride,
                             double* vm, double* scratch, cudaStream_t s, const int* eq_counter = nullptr,
                             const int* eq_nbuf = nullptr, int n_ranks = 1);
// one half step with the equilibrium skip (fdm_equilibrium.cuh): speculative reaction, equilibrium tests,
// scan of the buffers, commit (and the trace after half 1)
cudaError_t launch_equilibrium_half(int model, RealKind rk, MathKind mk, const ReactionArgs& a, const EqLayout& L,
                                    const EqSpec& e, uint8_t* info, uint8_t* prefix, uint8_t* block_agg, int n_states,
                                    bool trace, cudaStream_t s);
// adjoint (FP64)
cudaError_t launch_adjoint_half(int model, MathKind mk, const AdjointArgs& a, cudaStream_t s);
cudaError_t launch_adjoint_diffusion(int n_fibers, const int64_t* fiber_offsets, const double* element_lengths,
                                     const double* coef, int64_t stride, double* lam, const double* u, const double* x,
                                     int implicit_euler, double* grad_prefactor, double* scratch, double* mu,
                                     int64_t max_fiber_len, cudaStream_t s);
// the CellmlAdapter's generic right-hand side on device arrays (SoA, index * n + instance)
cudaError_t launch_cellml_rhs(int model, MathKind mk, int64_t n, double t, const double* states, const double* params,
                              double* rates, double* algebraics, cudaStream_t s);
// counts non-finite entries of x[0..n) into *count (device int, must be zeroed by the caller)
cudaError_t launch_count_nonfinite(const double* x, int64_t n, int* count, cudaStream_t s);

// fused path (fdm_fused_*.cu)
struct FusedShape {
  int threads, nodes_per_thread;
};
int fused_shapes(FusedShape* out, int capacity);
// cluster mode shapes (threads per CTA, nodes per thread); a fiber spans up to 8 CTAs of one cluster.  One node
// per thread gives the few-fiber case the most independent Heun chains per SM
#define FDM_CLUSTER_SHAPES(X) \
  X(128, 2)                   \
  X(256, 2)                   \
  X(512, 2)                   \
  X(256, 4)                   \
  X(192, 1)                   \
  X(256, 1)
constexpr int FDM_MAX_CLUSTER = 8;
int cluster_shapes(FusedShape* out, int capacity);
// one fiber per cluster of csize CTAs (FP32/FP64 reaction with exact exponentials, no onlyComputeIfHasBeenStimulated)
cudaError_t launch_fused_cluster(int model, RealKind rk, int shape, int csize, const FusedArgs& a, cudaStream_t s);
// shape index into fused_shapes(); returns cudaErrorInvalidValue if the combination is not built
cudaError_t launch_fused(int model, RealKind rk, MathKind mk, int shape, const FusedArgs& a, cudaStream_t s);

} // namespace fdm
