// Model-dependent kernel launchers: every kernel template that is instantiated per CellML model.  Included by
// the library's own translation units for its built-in models and by a run-time model module (a generated
// translation unit for one further model or parameter variant, fdm_model_module.cuh), so that both launch the
// same kernels the same way.
#pragma once
#include "fdm_internal.h"

namespace fdm {

template<class Model, class RR, class Math>
inline cudaError_t reaction_one(const ReactionArgs& a, cudaStream_t s)
{
  const int T = 128;
  const int64_t blocks = (a.n_nodes + T - 1) / T;
  if (blocks == 0)
    return cudaSuccess;
  reaction_kernel<Model, RR, Math><<<(unsigned)blocks, T, 0, s>>>(a);
  return cudaGetLastError();
}

// up to this many nodes the FP64 split path advances a node's states on separate warps (reaction_group_kernel):
// one thread per node would leave fewer than about 16 warps per SM
constexpr int64_t kGroupKernelMaxNodes = 65536;

template<class Model, class Math>
inline cudaError_t reaction_group_one(const ReactionArgs& a, cudaStream_t s)
{
  const dim3 block(32, Model::nGroups);
  reaction_group_kernel<Model, Math><<<(unsigned)((a.n_nodes + 31) / 32), block, 0, s>>>(a);
  return cudaGetLastError();
}

template<class Model>
inline cudaError_t reaction_model(RealKind rk, MathKind mk, const ReactionArgs& a, cudaStream_t s)
{
  if constexpr (Model::nGroups > 0) {
    // few nodes, nothing but the Heun substeps asked of the launch: a warp per state of 32 nodes
    if (rk == REAL_F64 && a.n_nodes > 0 && a.n_nodes <= kGroupKernelMaxNodes && !a.gate && !a.store_states &&
        !a.store_vm_out && !a.store_alg && !a.per_node)
      return mk == MATH_EXACT ? reaction_group_one<Model, fdm_math_exact>(a, s)
                              : reaction_group_one<Model, fdm_math_approx>(a, s);
  }
  if (rk == REAL_F64)
    return mk == MATH_EXACT ? reaction_one<Model, double, fdm_math_exact>(a, s)
                            : reaction_one<Model, double, fdm_math_approx>(a, s);
  return mk == MATH_EXACT ? reaction_one<Model, float, fdm_math_exact>(a, s)
                          : reaction_one<Model, float, fdm_math_approx>(a, s);
}

template<class Model>
inline cudaError_t cellml_rhs_model(MathKind mk, int64_t n, double t, const double* st, const double* p, double* r,
                                    double* alg, cudaStream_t s)
{
  const int T = 128;
  const unsigned blocks = (unsigned)((n + T - 1) / T);
  if (mk == MATH_EXACT)
    cellml_rhs_kernel<Model, fdm_math_exact><<<blocks, T, 0, s>>>(n, t, st, p, r, alg);
  else
    cellml_rhs_kernel<Model, fdm_math_approx><<<blocks, T, 0, s>>>(n, t, st, p, r, alg);
  return cudaGetLastError();
}

template<class Model>
inline cudaError_t equilibrium_search_model(MathKind mk, double* u, const double* u0, const double* P, EquilibriumSearch* es,
                                     int64_t n, cudaStream_t s)
{
  if (mk == MATH_EXACT)
    equilibrium_search_kernel<Model, fdm_math_exact><<<1, 1, 0, s>>>(u, u0, P, es, n);
  else
    equilibrium_search_kernel<Model, fdm_math_approx><<<1, 1, 0, s>>>(u, u0, P, es, n);
  return cudaGetLastError();
}

template<class Model, class RR, class Math>
inline cudaError_t reaction_eq_one(const ReactionArgs& a, const EqLayout& L, const EqSpec& e, cudaStream_t s)
{
  const int T = 128;
  const int64_t blocks = (e.nt + T - 1) / T;
  if (blocks == 0)
    return cudaSuccess;
  reaction_eq_kernel<Model, RR, Math><<<(unsigned)blocks, T, 0, s>>>(a, L, e);
  return cudaGetLastError();
}

template<class Model>
inline cudaError_t reaction_eq_model(RealKind rk, MathKind mk, const ReactionArgs& a, const EqLayout& L,
                                     const EqSpec& e, cudaStream_t s)
{
  if (rk == REAL_F64)
    return mk == MATH_EXACT ? reaction_eq_one<Model, double, fdm_math_exact>(a, L, e, s)
                            : reaction_eq_one<Model, double, fdm_math_approx>(a, L, e, s);
  return mk == MATH_EXACT ? reaction_eq_one<Model, float, fdm_math_exact>(a, L, e, s)
                          : reaction_eq_one<Model, float, fdm_math_approx>(a, L, e, s);
}

template<class Model>
inline cudaError_t adjoint_model(MathKind mk, const AdjointArgs& a, cudaStream_t s)
{
  const int T = 128;
  const int64_t blocks = (a.n_nodes + T - 1) / T;
  if (blocks == 0)
    return cudaSuccess;
  if (mk == MATH_EXACT)
    adjoint_half_kernel<Model, fdm_math_exact><<<(unsigned)blocks, T, 0, s>>>(a);
  else
    adjoint_half_kernel<Model, fdm_math_approx><<<(unsigned)blocks, T, 0, s>>>(a);
  return cudaGetLastError();
}

} // namespace fdm
