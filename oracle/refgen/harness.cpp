// C entry point around the compute0DInstance that the reference's code generator emitted (compiled together
// with it).  TEST INFRASTRUCTURE ONLY.
//   refgen_heun_buffer: n_steps calls of compute0DInstance on one point buffer of Vc::double_v::size() lanes,
//   states[s * W + lane] in/out, params[q * W + lane]; step k at t0 + k * dt; the algebraics for transfer of
//   the last step go to alg_out[k * W + lane].
#include <vector>

#include <vc_or_std_simd.h>

extern "C" void compute0DInstance(Vc::double_v states[], std::vector<Vc::double_v>& parameters, double currentTime,
                                  double timeStepWidth, bool stimulate, bool storeAlgebraicsForTransfer,
                                  std::vector<Vc::double_v>& algebraicsForTransfer,
                                  const std::vector<int>& algebraicsForTransferIndices, double valueForStimulatedPoint);

extern "C" int refgen_lanes() { return (int)Vc::double_v::size(); }

extern "C" int refgen_heun_buffer(int n_states, int n_params, double* states, const double* params, double t0,
                                  double dt, int n_steps, int stimulate, double v_stim, int n_alg,
                                  const int* alg_indices, double* alg_out)
{
  const int W = (int)Vc::double_v::size();
  std::vector<Vc::double_v> y((size_t)n_states), p((size_t)(n_params > 0 ? n_params : 1)), alg((size_t)n_alg);
  for (int s = 0; s < n_states; s++)
    for (int l = 0; l < W; l++)
      y[(size_t)s][l] = states[s * W + l];
  for (int q = 0; q < n_params; q++)
    for (int l = 0; l < W; l++)
      p[(size_t)q][l] = params[q * W + l];
  const std::vector<int> idx(alg_indices, alg_indices + n_alg);
  for (int k = 0; k < n_steps; k++)
    compute0DInstance(y.data(), p, t0 + k * dt, dt, stimulate != 0, k == n_steps - 1 && n_alg > 0, alg, idx,
                      v_stim);
  for (int s = 0; s < n_states; s++)
    for (int l = 0; l < W; l++)
      states[s * W + l] = y[(size_t)s][l];
  for (int k = 0; k < n_alg; k++)
    for (int l = 0; l < W; l++)
      alg_out[k * W + l] = alg[(size_t)k][l];
  return 0;
}
