// A run-time model module: the kernels of one CellML model (or parameter variant) that is not built into
// libfdm_b200.so, compiled into a shared library of its own at run time.  A generated translation unit
// includes the generated model header and then this file with FDM_MODULE_MODEL naming the model's struct:
//
//   #include "<generated model>.cuh"
//   #define FDM_MODULE_MODEL fdm_model_<name>_<variant>
//   #include "fdm_model_module.cuh"
//
// The library loads it with fdm_register_model_library (dlopen), the way the reference loads the library it
// generated and compiled from the model file (fast_monodomain_solver_gpu.tpp:106-205, the libraryFilename
// option of CellmlAdapter).  The module's kernels are the library's own templates (fdm_model_launch.cuh).
#pragma once
#include "fdm_model_launch.cuh"

#ifndef FDM_MODULE_MODEL
#error "define FDM_MODULE_MODEL (the generated model struct) before including fdm_model_module.cuh"
#endif

namespace fdm_module {
using Model = FDM_MODULE_MODEL;

static cudaError_t reaction(fdm::RealKind rk, fdm::MathKind mk, const fdm::ReactionArgs& a, cudaStream_t s)
{
  return fdm::reaction_model<Model>(rk, mk, a, s);
}
static cudaError_t cellml_rhs(fdm::MathKind mk, int64_t n, double t, const double* st, const double* p, double* r,
                              double* alg, cudaStream_t s)
{
  return n == 0 ? cudaSuccess : fdm::cellml_rhs_model<Model>(mk, n, t, st, p, r, alg, s);
}
static cudaError_t equilibrium_search(fdm::MathKind mk, double* u, const double* u0, const double* p,
                                      fdm::EquilibriumSearch* es, int64_t n, cudaStream_t s)
{
  return fdm::equilibrium_search_model<Model>(mk, u, u0, p, es, n, s);
}
static cudaError_t reaction_eq(fdm::RealKind rk, fdm::MathKind mk, const fdm::ReactionArgs& a,
                               const fdm::EqLayout& L, const fdm::EqSpec& e, cudaStream_t s)
{
  return fdm::reaction_eq_model<Model>(rk, mk, a, L, e, s);
}
static cudaError_t adjoint_half(fdm::MathKind mk, const fdm::AdjointArgs& a, cudaStream_t s)
{
  return fdm::adjoint_model<Model>(mk, a, s);
}
} // namespace fdm_module

extern "C" __attribute__((visibility("default"))) int fdm_model_module_v1(fdm::ModelModule* out)
{
  using M = fdm_module::Model;
  if (!out)
    return 1;
  out->abi = FDM_MODEL_MODULE_ABI;
  out->desc = fdm::ModelDesc{M::name, M::nStates, M::nAlgebraics, M::nParameters, M::statesInitialValues,
                             M::parameterDefaults, false};
  out->reaction = fdm_module::reaction;
  out->cellml_rhs = fdm_module::cellml_rhs;
  out->equilibrium_search = fdm_module::equilibrium_search;
  out->reaction_eq = fdm_module::reaction_eq;
  out->adjoint_half = fdm_module::adjoint_half;
  return 0;
}
