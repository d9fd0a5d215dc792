// Fibers -> 3D static bidomain (EMG): the caller downstream of the fiber solver in the reference's
// fibers_emg example (examples/electrophysiology/fibers/fibers_emg/src/fast_fibers_emg.cpp:17-63,
// Control::Coupling of the FastMonodomainSolver with TimeSteppingScheme::StaticBidomainSolver).
//
//  * mesh: structured hexahedral mesh (StructuredDeformableOfDimension<3>, linear Lagrange), nodes numbered
//    i + nx*(j + ny*k), element dofs a + 2b + 4c (the reference's dof order within an element);
//  * operators: stiffness matrices K(sigma) = int grad(phi_l) . sigma . grad(phi_m) stored as a 27-point
//    stencil per node (SoA: coef[q * N + node], q = (dx+1) + 3(dy+1) + 9(dz+1)), assembled per node in a fixed
//    order (deterministic) with Gauss-Legendre quadrature;
//  * potential flow (static_bidomain_solver.tpp:102-130): Laplace with Dirichlet values, the nodal gradient
//    averaged over the adjacent elements (08_field_variable_gradient.tpp:59-115), normalised to the fiber
//    direction (diffusion_tensor_directional.tpp:27-37);
//  * directional tensors (diffusion_tensor_directional.tpp:72-110, math_utility.tpp:587-655): the tensor
//    given in fiber coordinates, sigma_i or sigma_i + sigma_e, rotated onto the interpolated direction;
//  * transfer of Vm from the fibers (mapping_between_meshes 00_construct.tpp:90-160, 01_implementation.tpp:15-60,
//    03_manager_implementation.tpp:239-300): each fiber node adds phi_m(xi) * Vm to the 8 nodes of the element
//    it lies in, each 3D node divides by the sum of its factors (|sum| <= 1e-12: the default value);
//  * solve (static_bidomain_solver.tpp:37-55): K(sigma_i + sigma_e) phi_e = -K(sigma_i) Vm with the constant
//    functions as null space, by conjugate gradients with a Jacobi preconditioner, all on the device; the
//    result is the zero-mean solution.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fdm_b200.h"
#include "fdm_internal.h"

namespace {

constexpr int EMG_T = 256;          // threads per block of the vector kernels
constexpr int EMG_MAX_BLOCKS = 1184; // 148 SMs x 8 resident blocks: grid-stride loops, one partial per block
constexpr int EMG_MAX_GAUSS = 7;

template<class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t k)
  {
    if (k <= n && p)
      return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(k, 1) * sizeof(T));
    if (e == cudaSuccess)
      n = k;
    return e;
  }
  void release()
  {
    if (p)
      cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~Buf() { release(); }
};

struct Quad {
  int n;
  double x[EMG_MAX_GAUSS], w[EMG_MAX_GAUSS];
};

// Gauss-Legendre points and weights on [0, 1]: Newton's method on the Legendre polynomial P_n from the
// Chebyshev-node guesses, P_n and P_n' by the three-term recurrence.
Quad gauss_legendre(int n)
{
  Quad q{};
  q.n = n;
  for (int i = 0; i < n; i++) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) {
        p1 = z;
        p0 = 1.0;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16)
        break;
    }
    q.x[i] = 0.5 * (1.0 - z);
    q.w[i] = 1.0 / ((1.0 - z * z) * dp * dp); // 2/((1-z^2) P'^2) on [-1,1], halved on [0,1]
  }
  return q;
}

// ---- element geometry ------------------------------------------------------------------------------

struct Grid {
  int nx, ny, nz;
  __host__ __device__ int64_t n_nodes() const { return (int64_t)nx * ny * nz; }
  __host__ __device__ int64_t n_elements() const { return (int64_t)(nx - 1) * (ny - 1) * (nz - 1); }
  __host__ __device__ int64_t node(int i, int j, int k) const { return i + (int64_t)nx * (j + (int64_t)ny * k); }
  __host__ __device__ int64_t element(int i, int j, int k) const
  {
    return i + (int64_t)(nx - 1) * (j + (int64_t)(ny - 1) * k);
  }
};

// shape functions of the trilinear element and their derivatives at xi
__host__ __device__ inline void shape(const double xi[3], double phi[8], double dphi[8][3])
{
  for (int l = 0; l < 8; l++) {
    const int a = l & 1, b = (l >> 1) & 1, c = l >> 2;
    const double fx = a ? xi[0] : 1.0 - xi[0], fy = b ? xi[1] : 1.0 - xi[1], fz = c ? xi[2] : 1.0 - xi[2];
    const double gx = a ? 1.0 : -1.0, gy = b ? 1.0 : -1.0, gz = c ? 1.0 : -1.0;
    phi[l] = fx * fy * fz;
    dphi[l][0] = gx * fy * fz;
    dphi[l][1] = fx * gy * fz;
    dphi[l][2] = fx * fy * gz;
  }
}

// J[i][d] = d x_i / d xi_d; returns det J, writes the inverse
__host__ __device__ inline double jacobian(const double P[8][3], const double dphi[8][3], double inv[3][3])
{
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int l = 0; l < 8; l++)
    for (int i = 0; i < 3; i++)
      for (int d = 0; d < 3; d++)
        J[i][d] += P[l][i] * dphi[l][d];
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  inv[0][0] = c00 * id;
  inv[1][0] = c01 * id;
  inv[2][0] = c02 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return det;
}

// world-space gradient: grad_x phi = J^-T grad_xi phi  (inv = J^-1, inv[d][i] = d xi_d / d x_i)
__host__ __device__ inline void world_gradient(const double inv[3][3], const double g[3], double out[3])
{
  for (int i = 0; i < 3; i++)
    out[i] = inv[0][i] * g[0] + inv[1][i] * g[1] + inv[2][i] * g[2];
}

// the reference's rotation of a tensor given in fiber coordinates onto direction b (math_utility.tpp:587-655),
// its formulas kept as they are: for b along e_3 the basis is built from e_2, with its norm expression for
// the third basis vector (exact for |b| = 1, as nodal directions are)
__host__ __device__ inline void rotate_tensor(double S[3][3], const double b[3])
{
  const double b1 = b[0], b2 = b[1], b3 = b[2];
  const double bNorm = sqrt(b1 * b1 + b2 * b2 + b3 * b3);
  const double e3bNorm = sqrt(b1 * b1 + b2 * b2);
  const double be3bNorm = sqrt(b1 * b1 * b3 * b3 + b2 * b2 * b3 * b3 + (b1 * b1 + b2 * b2) * (b1 * b1 + b2 * b2));
  if (fabs(bNorm) < 1e-15)
    return;
  double B[3][3];
  if (fabs(e3bNorm) < 1e-15 || fabs(be3bNorm) < 1e-15) {
    const double e2bNorm = sqrt(b3 * b3 + b1 * b1);
    const double be2bNorm = sqrt(b1 * b1 * b2 * b2 + (b1 * b1 * b3 * b3) * (b1 * b1 * b3 * b3) + b2 * b2 + b3 * b3);
    if (fabs(e2bNorm) < 1e-15 || fabs(be2bNorm) < 1e-15)
      return;
    const double Bv[3][3] = {{b1 / bNorm, b3 / e2bNorm, -b1 * b2 / be2bNorm},
                             {b2 / bNorm, 0.0, (b1 * b1 + b3 * b3) / be2bNorm},
                             {b3 / bNorm, -b1 / e2bNorm, -b2 * b3 / be2bNorm}};
    memcpy(B, Bv, sizeof(B));
  } else {
    const double Bv[3][3] = {{b1 / bNorm, -b2 / e3bNorm, -b1 * b3 / be3bNorm},
                             {b2 / bNorm, b1 / e3bNorm, -b2 * b3 / be3bNorm},
                             {b3 / bNorm, 0.0, (b1 * b1 + b2 * b2) / be3bNorm}};
    memcpy(B, Bv, sizeof(B));
  }
  double T[3][3], R[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      T[i][j] = B[i][0] * S[0][j] + B[i][1] * S[1][j] + B[i][2] * S[2][j];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      R[i][j] = T[i][0] * B[j][0] + T[i][1] * B[j][1] + T[i][2] * B[j][2];
  memcpy(S, R, sizeof(R));
}

__device__ inline void element_nodes(const Grid& g, int ei, int ej, int ek, int64_t nodes[8])
{
  for (int l = 0; l < 8; l++)
    nodes[l] = g.node(ei + (l & 1), ej + ((l >> 1) & 1), ek + (l >> 2));
}

// ---- kernels -----------------------------------------------------------------------------------------

struct AssembleArgs {
  Grid g;
  const double* pos;       // [N][3]
  const double* dir;       // [N][3] normalised nodal directions, or null (tensor used as given)
  const double* tensor;    // 9 per element, or 9 for all (n_tensor == 1)
  const double* tensor2;   // added to tensor before the rotation (sigma_e), or null
  int64_t n_tensor, n_tensor2;
  double prefactor;
  Quad q;
  double* coef;            // [EMG_NC][N]: the centre and forward coefficients of each row
};

// row of node n of the assembled stiffness matrix: the sum over its adjacent elements (in element order) of the
// element matrix row, each integrated over the element's Gauss points in order
__global__ void __launch_bounds__(128) assemble_kernel(AssembleArgs a)
{
  const int64_t N = a.g.n_nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % a.g.nx), j = (int)((n / a.g.nx) % a.g.ny), k = (int)(n / ((int64_t)a.g.nx * a.g.ny));
    double row[27];
    for (int q = 0; q < 27; q++)
      row[q] = 0.0;
    for (int c = 1; c >= 0; c--)
      for (int b = 1; b >= 0; b--)
        for (int aa = 1; aa >= 0; aa--) {
          // element whose local node (aa, b, c) is this node
          const int ei = i - aa, ej = j - b, ek = k - c;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= a.g.nx - 1 || ej >= a.g.ny - 1 || ek >= a.g.nz - 1)
            continue;
          const int l = aa + 2 * b + 4 * c;
          int64_t nodes[8];
          element_nodes(a.g, ei, ej, ek, nodes);
          double P[8][3], D[8][3];
          for (int m = 0; m < 8; m++)
            for (int d = 0; d < 3; d++) {
              P[m][d] = a.pos[nodes[m] * 3 + d];
              D[m][d] = a.dir ? a.dir[nodes[m] * 3 + d] : 0.0;
            }
          const int64_t e = a.g.element(ei, ej, ek);
          const double* t1 = a.tensor + 9 * (a.n_tensor == 1 ? 0 : e);
          const double* t2 = a.tensor2 ? a.tensor2 + 9 * (a.n_tensor2 == 1 ? 0 : e) : nullptr;
          for (int qz = 0; qz < a.q.n; qz++)
            for (int qy = 0; qy < a.q.n; qy++)
              for (int qx = 0; qx < a.q.n; qx++) {
                const double xi[3] = {a.q.x[qx], a.q.x[qy], a.q.x[qz]};
                const double w = a.q.w[qx] * a.q.w[qy] * a.q.w[qz];
                double phi[8], dphi[8][3], inv[3][3];
                shape(xi, phi, dphi);
                const double det = jacobian(P, dphi, inv);
                double S[3][3];
                for (int r = 0; r < 3; r++)
                  for (int s = 0; s < 3; s++)
                    S[r][s] = t1[3 * r + s] + (t2 ? t2[3 * r + s] : 0.0);
                if (a.dir) {
                  double bvec[3] = {0.0, 0.0, 0.0};
                  for (int m = 0; m < 8; m++)
                    for (int d = 0; d < 3; d++)
                      bvec[d] += phi[m] * D[m][d];
                  if (!isfinite(bvec[0]) || !isfinite(bvec[1]) || !isfinite(bvec[2])) {
                    bvec[0] = 0.0;
                    bvec[1] = 0.0;
                    bvec[2] = 1.0;
                  }
                  rotate_tensor(S, bvec);
                }
                double gl[3], sg[3];
                world_gradient(inv, dphi[l], gl);
                for (int r = 0; r < 3; r++)
                  sg[r] = S[r][0] * gl[0] + S[r][1] * gl[1] + S[r][2] * gl[2];
                const double f = a.prefactor * w * fabs(det);
                for (int m = 0; m < 8; m++) {
                  double gm[3];
                  world_gradient(inv, dphi[m], gm);
                  const int dx = (m & 1) - aa, dy = ((m >> 1) & 1) - b, dz = (m >> 2) - c;
                  row[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] += f * (sg[0] * gm[0] + sg[1] * gm[1] + sg[2] * gm[2]);
                }
              }
        }
    // the centre and forward half (the backward half equals the neighbours' forward entries: K is symmetric)
    for (int q = 13; q < 27; q++)
      a.coef[(q - 13) * N + n] = row[q];
  }
}

// nodal gradient of u: per adjacent element the gradient at the node's corner, divided by the number of
// adjacent elements, summed; then normalised (a zero gradient gives a non-finite direction, which the
// assembly replaces by (0, 0, 1) as the reference does)
__global__ void gradient_direction_kernel(Grid g, const double* pos, const double* u, double* dir)
{
  const int64_t N = g.n_nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((int64_t)g.nx * g.ny));
    int n_adj = 0;
    for (int c = 0; c < 2; c++)
      for (int b = 0; b < 2; b++)
        for (int aa = 0; aa < 2; aa++) {
          const int ei = i - aa, ej = j - b, ek = k - c;
          n_adj += (ei >= 0 && ej >= 0 && ek >= 0 && ei < g.nx - 1 && ej < g.ny - 1 && ek < g.nz - 1) ? 1 : 0;
        }
    double grad[3] = {0.0, 0.0, 0.0};
    // elements in element order (the reference loops over elements and adds into the node)
    for (int c = 1; c >= 0; c--)
      for (int b = 1; b >= 0; b--)
        for (int aa = 1; aa >= 0; aa--) {
          const int ei = i - aa, ej = j - b, ek = k - c;
          if (ei < 0 || ej < 0 || ek < 0 || ei >= g.nx - 1 || ej >= g.ny - 1 || ek >= g.nz - 1)
            continue;
          int64_t nodes[8];
          element_nodes(g, ei, ej, ek, nodes);
          double P[8][3], uv[8];
          for (int m = 0; m < 8; m++) {
            for (int d = 0; d < 3; d++)
              P[m][d] = pos[nodes[m] * 3 + d];
            uv[m] = u[nodes[m]];
          }
          const double xi[3] = {(double)aa, (double)b, (double)c};
          double phi[8], dphi[8][3], inv[3][3];
          shape(xi, phi, dphi);
          jacobian(P, dphi, inv);
          double gxi[3] = {0.0, 0.0, 0.0};
          for (int m = 0; m < 8; m++)
            for (int d = 0; d < 3; d++)
              gxi[d] += uv[m] * dphi[m][d];
          double gw[3];
          world_gradient(inv, gxi, gw);
          for (int d = 0; d < 3; d++)
            grad[d] += gw[d] / n_adj;
        }
    const double nrm = sqrt(grad[0] * grad[0] + grad[1] * grad[1] + grad[2] * grad[2]);
    for (int d = 0; d < 3; d++)
      dir[n * 3 + d] = grad[d] / nrm;
  }
}

// ---- symmetric stencil storage and the conjugate-gradient kernels ----------------------------------------
// K is symmetric: only the centre and the 13 forward coefficients of each row are stored,
// U[k * N + n] = K[n][n + off(13 + k)] for stencil index q = 13 + k = (dx+1) + 3(dy+1) + 9(dz+1) >= 13; the
// backward entry K[n][n - off(q)] is the forward entry U[q - 13][n - off(q)] of the neighbour.
constexpr int EMG_NC = 14;

__host__ __device__ inline void stencil_offset(int q, int& dx, int& dy, int& dz)
{
  dx = q % 3 - 1;
  dy = (q / 3) % 3 - 1;
  dz = q / 9 - 1;
}

// Row n of K applied to the vector v(m).  The assembly leaves the coefficient of a neighbour outside the grid
// at exactly 0, and every forward offset is positive in the linear numbering, so no bounds test is needed on
// the coefficients: a forward coefficient towards a missing neighbour is 0, and the forward coefficient
// U[q][n - off] of a node whose forward neighbour is not n (a wrap-around in the numbering) is 0 too; only
// n - off < 0 is cut off.  The loads are then unconditional and issue together; v is read at clamped indices
// (its values there meet a 0 coefficient and must only be finite).
template<class V>
__device__ __forceinline__ double stencil_row(const Grid& g, const double* __restrict__ U, int64_t n, V v)
{
  const int64_t N = g.n_nodes();
  const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
  double s = U[n] * v(n);
#pragma unroll
  for (int q = 14; q < 27; q++) {
    int dx, dy, dz;
    stencil_offset(q, dx, dy, dz);
    const int64_t off = dx + dy * sy + dz * sz;
    const int64_t f = min(n + off, N - 1), b = n - off;
    const double cb = b >= 0 ? U[(q - 13) * N + b] : 0.0;
    s += U[(q - 13) * N + n] * v(f) + cb * v(max(b, (int64_t)0));
  }
  return s;
}

// Grid-wide sums of K values per thread: each block writes its partials, the block that finishes last sums
// all partials in block order (a fixed order: results do not depend on scheduling) and returns true in its
// thread 0 with the totals in tot; the counter is reset for the next launch.
template<int K>
__device__ bool grid_sum(double (&v)[K], double* partial, unsigned* counter, double (&tot)[K])
{
  __shared__ double red[K][EMG_T / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < K; c++) {
    double a = v[c];
    for (int o = 16; o > 0; o >>= 1)
      a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0)
      red[c][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int c = 0; c < K; c++) {
      double t = 0.0;
      for (int w = 0; w < EMG_T / 32; w++)
        t += red[c][w];
      partial[c * EMG_MAX_BLOCKS + blockIdx.x] = t;
    }
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return false;
  __threadfence();
#pragma unroll
  for (int c = 0; c < K; c++) {
    double a = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += EMG_T)
      a += __ldcg(&partial[c * EMG_MAX_BLOCKS + b]);
    for (int o = 16; o > 0; o >>= 1)
      a += __shfl_down_sync(0xffffffffu, a, o);
    __syncthreads();
    if (lane == 0)
      red[c][warp] = a;
  }
  __syncthreads();
  if (threadIdx.x != 0)
    return false;
#pragma unroll
  for (int c = 0; c < K; c++) {
    double t = 0.0;
    for (int w = 0; w < EMG_T / 32; w++)
      t += red[c][w];
    tot[c] = t;
  }
  *counter = 0u;
  return true;
}

// CG scalars in device memory: S[0] r.z, S[1] p.Ap, S[3] r.r, S[4] alpha, S[5] beta, S[6] sum, S[7] b.b
enum { CG_RZ = 0, CG_PQ = 1, CG_RR = 3, CG_ALPHA = 4, CG_BETA = 5, CG_SUM = 6, CG_BB = 7 };

// y = scale * K x
__global__ void __launch_bounds__(EMG_T) apply_kernel(Grid g, const double* __restrict__ U,
                                                      const double* __restrict__ x, double* __restrict__ y,
                                                      double scale)
{
  const int64_t N = g.n_nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
    y[n] = scale * stencil_row(g, U, n, [&](int64_t m) { return x[m]; });
}

// r = b - K x (rows in mask: r = 0), z = dinv r; S[RZ], S[RR]; beta = 0 for the first direction
__global__ void __launch_bounds__(EMG_T, 4) cg_init_kernel(Grid g, const double* __restrict__ U,
                                                        const unsigned char* __restrict__ mask,
                                                        const double* __restrict__ b, const double* __restrict__ x,
                                                        double* r, double* z, const double* __restrict__ dinv,
                                                        double* S, double* partial, unsigned* counter)
{
  const int64_t N = g.n_nodes();
  double acc[2] = {0.0, 0.0}, tot[2];
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    const bool fixed = mask && mask[n];
    const double rn = fixed ? 0.0 : b[n] - stencil_row(g, U, n, [&](int64_t m) { return x[m]; });
    const double zn = rn * dinv[n];
    r[n] = rn;
    z[n] = zn;
    acc[0] += rn * zn;
    acc[1] += rn * rn;
  }
  if (grid_sum<2>(acc, partial, counter, tot)) {
    S[CG_RZ] = tot[0];
    S[CG_RR] = tot[1];
    S[CG_BETA] = 0.0;
  }
}

// The nine rows (dy, dz in {-1, 0, 1}) of z around the block's EMG_T consecutive nodes [n0, n0 + EMG_T), one
// node of halo each side, staged in shared memory: neighbour (dx, dy, dz) of node n0 + t is
// sv[(dy+1) + 3(dz+1)][t + 1 + dx].  Every global load is a coalesced row segment.
__device__ __forceinline__ void stage_rows(const Grid& g, const double* __restrict__ z, int64_t n0,
                                           double (*sv)[EMG_T + 2])
{
  const int64_t N = g.n_nodes();
  for (int e = threadIdx.x; e < 9 * (EMG_T + 2); e += EMG_T) {
    const int r = e / (EMG_T + 2), t = e % (EMG_T + 2);
    const int dy = r % 3 - 1, dz = r / 3 - 1;
    const int64_t m = n0 + dy * (int64_t)g.nx + dz * (int64_t)g.nx * g.ny + t - 1;
    sv[r][t] = (m >= 0 && m < N) ? z[m] : 0.0;
  }
}

// stencil_row with the neighbours' values from the staged rows (the same zero-coefficient argument)
__device__ __forceinline__ double stencil_row_staged(const Grid& g, const double* __restrict__ U, int64_t n, int t,
                                                     const double (*sv)[EMG_T + 2])
{
  const int64_t N = g.n_nodes();
  const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
  double s = U[n] * sv[4][t + 1];
#pragma unroll
  for (int q = 14; q < 27; q++) {
    int dx, dy, dz;
    stencil_offset(q, dx, dy, dz);
    const int64_t b = n - (dx + dy * sy + dz * sz);
    const double cb = b >= 0 ? U[(q - 13) * N + b] : 0.0;
    s += U[(q - 13) * N + n] * sv[(dy + 1) + 3 * (dz + 1)][t + 1 + dx] + cb * sv[(1 - dy) + 3 * (1 - dz)][t + 1 - dx];
  }
  return s;
}

// Direction and product in one pass (the Chronopoulos-Gear arrangement of CG): w = K z, p = z + beta p,
// q = w + beta q (= K p), so that only z is read around each node; alpha = r.z / p.q.  p and q start at 0.
__global__ void __launch_bounds__(EMG_T, 4) cg_direction_kernel(Grid g, const double* __restrict__ U,
                                                                const unsigned char* __restrict__ mask,
                                                                const double* __restrict__ z, double* __restrict__ p,
                                                                double* __restrict__ q, double* S, double* partial,
                                                                unsigned* counter)
{
  __shared__ double sv[9][EMG_T + 2];
  const int64_t N = g.n_nodes();
  const double beta = S[CG_BETA];
  double acc[1] = {0.0}, tot[1];
  for (int64_t n0 = (int64_t)blockIdx.x * EMG_T; n0 < N; n0 += (int64_t)gridDim.x * EMG_T) {
    stage_rows(g, z, n0, sv);
    __syncthreads();
    const int64_t n = n0 + threadIdx.x;
    if (n < N) {
      const double w = (mask && mask[n]) ? 0.0 : stencil_row_staged(g, U, n, threadIdx.x, sv);
      const double pn = z[n] + beta * p[n];
      const double qn = w + beta * q[n];
      p[n] = pn;
      q[n] = qn;
      acc[0] += pn * qn;
    }
    __syncthreads();
  }
  if (grid_sum<1>(acc, partial, counter, tot)) {
    S[CG_PQ] = tot[0];
    S[CG_ALPHA] = tot[0] != 0.0 ? S[CG_RZ] / tot[0] : 0.0;
  }
}

// x += alpha p, r -= alpha q, z = dinv r; beta = r.z new / r.z
__global__ void __launch_bounds__(EMG_T) cg_update_kernel(int64_t N, double* __restrict__ x, double* __restrict__ r,
                                                          double* __restrict__ z, const double* __restrict__ p,
                                                          const double* __restrict__ q,
                                                          const double* __restrict__ dinv, double* S, double* partial,
                                                          unsigned* counter)
{
  const double alpha = S[CG_ALPHA];
  double acc[2] = {0.0, 0.0}, tot[2];
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    x[n] += alpha * p[n];
    const double rn = r[n] - alpha * q[n];
    const double zn = rn * dinv[n];
    r[n] = rn;
    z[n] = zn;
    acc[0] += rn * zn;
    acc[1] += rn * rn;
  }
  if (grid_sum<2>(acc, partial, counter, tot)) {
    S[CG_BETA] = S[CG_RZ] != 0.0 ? tot[0] / S[CG_RZ] : 0.0;
    S[CG_RZ] = tot[0];
    S[CG_RR] = tot[1];
  }
}

// S[SUM] = sum x, S[BB] = b.b (b may be null)
__global__ void __launch_bounds__(EMG_T) sum_kernel(int64_t N, const double* __restrict__ x,
                                                    const double* __restrict__ b, double* S, double* partial,
                                                    unsigned* counter)
{
  double acc[2] = {0.0, 0.0}, tot[2];
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    acc[0] += x[n];
    if (b)
      acc[1] += b[n] * b[n];
  }
  if (grid_sum<2>(acc, partial, counter, tot)) {
    S[CG_SUM] = tot[0];
    S[CG_BB] = tot[1];
  }
}

// y = x - mean(x) (x may equal y)
__global__ void subtract_mean_kernel(int64_t N, const double* x, double* y, const double* S)
{
  const double m = S[CG_SUM] / (double)N;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
    y[n] = x[n] - m;
}

__global__ void inverse_diag_kernel(int64_t N, const double* diag /* the centre coefficients */,
                                    const unsigned char* mask, double* dinv)
{
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
    dinv[n] = (mask && mask[n]) ? 0.0 : (diag[n] != 0.0 ? 1.0 / diag[n] : 1.0);
}

// ---- geometric multigrid preconditioner (bidomain solve) ----------------------------------------------
// Coarsening per direction: coarse nodes at the fine indices 0, 2, 4, ... and the last one; interpolation
// linear in the index between neighbouring coarse nodes (P); coarse operators P^T A P (Galerkin);
// l1-Jacobi smoothing (x += (b - A x) / sum_m |a_nm|: convergent for symmetric positive semidefinite A
// without a damping estimate -- Baker, Falgout, Kolev, Yang, "Multigrid smoothers for ultraparallel
// computing", SIAM J. Sci. Comput. 33 (2011)), two sweeps before and after; on the coarsest grid the same
// sweeps in one block.  Pre- and post-smoothing by the same symmetric smoother make the V-cycle a symmetric
// positive semidefinite preconditioner.
constexpr int MG_MAX_LEVELS = 12;
constexpr int MG_COARSEST = 1024;   // nodes of the grid solved by sweeps in one block
constexpr int MG_COARSEST_SWEEPS = 30;

struct MgMap {
  Grid fine, coarse;
  const int* lo[3];      // per fine index: the coarse node at or below it
  const double* w[3];    // per fine index: weight of coarse node lo + 1 (that of lo is 1 - w)
  const int* rlo[3];     // per coarse index: the fine range of its interpolation support
  const int* rhi[3];
};

__device__ __forceinline__ double mg_weight(const MgMap& M, int d, int i, int c)
{
  const int l = M.lo[d][i];
  const double w = M.w[d][i];
  return c == l ? 1.0 - w : (c == l + 1 ? w : 0.0);
}

// one row of P^T A P: coarse node I against its 27 coarse neighbours, the centre and forward half stored
__global__ void mg_galerkin_kernel(MgMap M, const double* __restrict__ Uf, double* __restrict__ Uc)
{
  const int64_t Nc = M.coarse.n_nodes(), Nf = M.fine.n_nodes();
  const int64_t sy = M.fine.nx, sz = (int64_t)M.fine.nx * M.fine.ny;
  for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < Nc; I += (int64_t)gridDim.x * blockDim.x) {
    const int ci = (int)(I % M.coarse.nx), cj = (int)((I / M.coarse.nx) % M.coarse.ny),
              ck = (int)(I / ((int64_t)M.coarse.nx * M.coarse.ny));
    double row[27];
    for (int q = 0; q < 27; q++)
      row[q] = 0.0;
    for (int fk = M.rlo[2][ck]; fk <= M.rhi[2][ck]; fk++)
      for (int fj = M.rlo[1][cj]; fj <= M.rhi[1][cj]; fj++)
        for (int fi = M.rlo[0][ci]; fi <= M.rhi[0][ci]; fi++) {
          const double wI = mg_weight(M, 0, fi, ci) * mg_weight(M, 1, fj, cj) * mg_weight(M, 2, fk, ck);
          if (wI == 0.0)
            continue;
          const int64_t n = M.fine.node(fi, fj, fk);
          for (int q = 0; q < 27; q++) {
            int dx, dy, dz;
            stencil_offset(q, dx, dy, dz);
            const int mi = fi + dx, mj = fj + dy, mk = fk + dz;
            if (mi < 0 || mj < 0 || mk < 0 || mi >= M.fine.nx || mj >= M.fine.ny || mk >= M.fine.nz)
              continue;
            const int64_t mn = n + dx + dy * sy + dz * sz;
            const double a = q >= 13 ? Uf[(q - 13) * Nf + n] : Uf[(13 - q) * Nf + mn];
            if (a == 0.0)
              continue;
            const int lx = M.lo[0][mi], ly = M.lo[1][mj], lz = M.lo[2][mk];
            for (int c = 0; c < 8; c++) {
              const int Jx = lx + (c & 1), Jy = ly + ((c >> 1) & 1), Jz = lz + (c >> 2);
              if (Jx >= M.coarse.nx || Jy >= M.coarse.ny || Jz >= M.coarse.nz)
                continue;
              const double wJ = mg_weight(M, 0, mi, Jx) * mg_weight(M, 1, mj, Jy) * mg_weight(M, 2, mk, Jz);
              // a nonzero weight puts J next to I (the fine neighbour lies between the coarse neighbours of I)
              if (wJ == 0.0 || abs(Jx - ci) > 1 || abs(Jy - cj) > 1 || abs(Jz - ck) > 1)
                continue;
              row[(Jx - ci + 1) + 3 * (Jy - cj + 1) + 9 * (Jz - ck + 1)] += wI * a * wJ;
            }
          }
        }
    for (int q = 13; q < 27; q++)
      Uc[(q - 13) * Nc + I] = row[q];
  }
}

// b_c = P^T r
__global__ void mg_restrict_kernel(MgMap M, const double* __restrict__ r, double* __restrict__ bc)
{
  const int64_t Nc = M.coarse.n_nodes();
  for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < Nc; I += (int64_t)gridDim.x * blockDim.x) {
    const int ci = (int)(I % M.coarse.nx), cj = (int)((I / M.coarse.nx) % M.coarse.ny),
              ck = (int)(I / ((int64_t)M.coarse.nx * M.coarse.ny));
    double s = 0.0;
    for (int fk = M.rlo[2][ck]; fk <= M.rhi[2][ck]; fk++) {
      const double wz = mg_weight(M, 2, fk, ck);
      for (int fj = M.rlo[1][cj]; fj <= M.rhi[1][cj]; fj++) {
        const double wyz = wz * mg_weight(M, 1, fj, cj);
        for (int fi = M.rlo[0][ci]; fi <= M.rhi[0][ci]; fi++)
          s += wyz * mg_weight(M, 0, fi, ci) * r[M.fine.node(fi, fj, fk)];
      }
    }
    bc[I] = s;
  }
}

// x += P e_c
__global__ void mg_prolong_add_kernel(MgMap M, const double* __restrict__ ec, double* __restrict__ x)
{
  const int64_t Nf = M.fine.n_nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < Nf; n += (int64_t)gridDim.x * blockDim.x) {
    const int fi = (int)(n % M.fine.nx), fj = (int)((n / M.fine.nx) % M.fine.ny),
              fk = (int)(n / ((int64_t)M.fine.nx * M.fine.ny));
    const int lx = M.lo[0][fi], ly = M.lo[1][fj], lz = M.lo[2][fk];
    double s = 0.0;
    for (int c = 0; c < 8; c++) {
      const int Jx = lx + (c & 1), Jy = ly + ((c >> 1) & 1), Jz = lz + (c >> 2);
      if (Jx >= M.coarse.nx || Jy >= M.coarse.ny || Jz >= M.coarse.nz)
        continue;
      const double w = mg_weight(M, 0, fi, Jx) * mg_weight(M, 1, fj, Jy) * mg_weight(M, 2, fk, Jz);
      if (w != 0.0)
        s += w * ec[M.coarse.node(Jx, Jy, Jz)];
    }
    x[n] += s;
  }
}

// 1 / sum_m |a_nm| of each row (the l1-Jacobi scaling)
__global__ void mg_l1_kernel(Grid g, const double* __restrict__ U, double* __restrict__ dl1)
{
  const int64_t N = g.n_nodes();
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    // the centre, the forward entries, and the backward entries (the neighbours' forward ones; zero where
    // the neighbour does not exist, as in stencil_row)
    const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
    double sum = fabs(U[n]);
    for (int q = 14; q < 27; q++) {
      int dx, dy, dz;
      stencil_offset(q, dx, dy, dz);
      const int64_t bk = n - (dx + dy * sy + dz * sz);
      sum += fabs(U[(q - 13) * N + n]) + (bk >= 0 ? fabs(U[(q - 13) * N + bk]) : 0.0);
    }
    dl1[n] = sum > 0.0 ? 1.0 / sum : 0.0;
  }
}

// l1-Jacobi sweep: xo = x + dl1 (b - A x) (x's rows staged in shared memory); from zero (x null): xo = dl1 b
__global__ void __launch_bounds__(EMG_T, 4) mg_jacobi_kernel(Grid g, const double* __restrict__ U,
                                                             const double* __restrict__ dl1,
                                                             const double* __restrict__ b,
                                                             const double* __restrict__ x, double* __restrict__ xo)
{
  __shared__ double sv[9][EMG_T + 2];
  const int64_t N = g.n_nodes();
  if (!x) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
      xo[n] = dl1[n] * b[n];
    return;
  }
  for (int64_t n0 = (int64_t)blockIdx.x * EMG_T; n0 < N; n0 += (int64_t)gridDim.x * EMG_T) {
    stage_rows(g, x, n0, sv);
    __syncthreads();
    const int64_t n = n0 + threadIdx.x;
    if (n < N)
      xo[n] = sv[4][threadIdx.x + 1] + dl1[n] * (b[n] - stencil_row_staged(g, U, n, threadIdx.x, sv));
    __syncthreads();
  }
}

// r = b - A x (x's rows staged in shared memory)
__global__ void __launch_bounds__(EMG_T, 4) mg_residual_kernel(Grid g, const double* __restrict__ U,
                                                               const double* __restrict__ b,
                                                               const double* __restrict__ x, double* __restrict__ r)
{
  __shared__ double sv[9][EMG_T + 2];
  const int64_t N = g.n_nodes();
  for (int64_t n0 = (int64_t)blockIdx.x * EMG_T; n0 < N; n0 += (int64_t)gridDim.x * EMG_T) {
    stage_rows(g, x, n0, sv);
    __syncthreads();
    const int64_t n = n0 + threadIdx.x;
    if (n < N)
      r[n] = b[n] - stencil_row_staged(g, U, n, threadIdx.x, sv);
    __syncthreads();
  }
}

// coarsest grid: `sweeps` l1-Jacobi sweeps from zero in one block (x and t ping-pong; x holds the result)
__global__ void __launch_bounds__(1024) mg_coarsest_kernel(Grid g, const double* __restrict__ U,
                                                           const double* __restrict__ dl1,
                                                           const double* __restrict__ b, double* x, double* t,
                                                           int sweeps)
{
  const int64_t N = g.n_nodes();
  for (int64_t n = threadIdx.x; n < N; n += blockDim.x)
    x[n] = dl1[n] * b[n];
  __syncthreads();
  double* cur = x;
  double* oth = t;
  for (int s = 1; s < sweeps; s++) {
    for (int64_t n = threadIdx.x; n < N; n += blockDim.x) {
      const double ax = stencil_row(g, U, n, [&](int64_t m) { return cur[m]; });
      oth[n] = cur[n] + dl1[n] * (b[n] - ax);
    }
    __syncthreads();
    double* sw = cur;
    cur = oth;
    oth = sw;
  }
  if (cur != x) {
    for (int64_t n = threadIdx.x; n < N; n += blockDim.x)
      x[n] = cur[n];
  }
}

// x = z after the update: partial r.z -> beta = r.z new / r.z, r.z (preconditioner applied outside)
__global__ void __launch_bounds__(EMG_T) cg_rz_kernel(int64_t N, const double* __restrict__ r,
                                                      const double* __restrict__ z, double* S, double* partial,
                                                      unsigned* counter, int first)
{
  double acc[1] = {0.0}, tot[1];
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x)
    acc[0] += r[n] * z[n];
  if (grid_sum<1>(acc, partial, counter, tot)) {
    S[CG_BETA] = (!first && S[CG_RZ] != 0.0) ? tot[0] / S[CG_RZ] : 0.0;
    S[CG_RZ] = tot[0];
  }
}

// the update without a preconditioner: x += alpha p, r -= alpha q; r.r
__global__ void __launch_bounds__(EMG_T) cg_update_plain_kernel(int64_t N, double* __restrict__ x,
                                                                double* __restrict__ r, const double* __restrict__ p,
                                                                const double* __restrict__ q, double* S,
                                                                double* partial, unsigned* counter)
{
  const double alpha = S[CG_ALPHA];
  double acc[1] = {0.0}, tot[1];
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    x[n] += alpha * p[n];
    const double rn = r[n] - alpha * q[n];
    r[n] = rn;
    acc[0] += rn * rn;
  }
  if (grid_sum<1>(acc, partial, counter, tot))
    S[CG_RR] = tot[0];
}

// 3D node n: sum over its contributions (fiber node, factor) in fiber-node order, divided by the factor sum
__global__ void map_kernel(int64_t N, const int64_t* ptr, const int64_t* src, const double* w, const double* fsum,
                           const double* vm, double default_value, double* out)
{
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int64_t e = ptr[n]; e < ptr[n + 1]; e++)
      v += w[e] * vm[src[e]];
    out[n] = fabs(fsum[n]) > 1e-12 ? v / fsum[n] : default_value;
  }
}

int blocks_for(int64_t n)
{
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + EMG_T - 1) / EMG_T, EMG_MAX_BLOCKS));
}

// ---- host: trilinear inversion and element search ------------------------------------------------------

struct HostMesh {
  Grid g;
  std::vector<double> pos; // [N][3]
  void element_points(int64_t e, double P[8][3]) const
  {
    const int ex = (int)(e % (g.nx - 1)), ey = (int)((e / (g.nx - 1)) % (g.ny - 1)),
              ez = (int)(e / ((int64_t)(g.nx - 1) * (g.ny - 1)));
    for (int l = 0; l < 8; l++) {
      const int64_t n = g.node(ex + (l & 1), ey + ((l >> 1) & 1), ez + (l >> 2));
      for (int d = 0; d < 3; d++)
        P[l][d] = pos[n * 3 + d];
    }
  }
  // xi of point x in element e by Newton's method on the trilinear map; returns the largest distance of xi
  // outside [0, 1] (0 inside)
  double locate(int64_t e, const double x[3], double xi[3]) const
  {
    double P[8][3];
    element_points(e, P);
    xi[0] = xi[1] = xi[2] = 0.5;
    for (int it = 0; it < 50; it++) {
      double phi[8], dphi[8][3], inv[3][3];
      shape(xi, phi, dphi);
      jacobian(P, dphi, inv);
      double r[3] = {-x[0], -x[1], -x[2]};
      for (int l = 0; l < 8; l++)
        for (int d = 0; d < 3; d++)
          r[d] += phi[l] * P[l][d];
      double dmax = 0.0;
      for (int d = 0; d < 3; d++) {
        const double dx = inv[d][0] * r[0] + inv[d][1] * r[1] + inv[d][2] * r[2];
        xi[d] -= dx;
        dmax = std::max(dmax, std::fabs(dx));
      }
      if (!(dmax > 1e-15) || !std::isfinite(dmax))
        break;
    }
    double out = 0.0;
    for (int d = 0; d < 3; d++)
      out = std::max(out, std::max(-xi[d], xi[d] - 1.0));
    return std::isfinite(out) ? out : 1e300;
  }
};

} // namespace

// ---- the solver object -----------------------------------------------------------------------------------

// one level of the multigrid hierarchy (level 0: the fine grid, whose operator and vectors belong to the CG)
struct MgLevel {
  Grid g{};
  Buf<double> U, dinv, b, x, t, r;      // operator, l1 scaling and vectors (level 0: the operator and b, x are
                                        // the CG's)
  Buf<int> lo, rlo, rhi;                // map to the next coarser level, three directions concatenated
  Buf<double> w;
  MgMap map{};
};

struct fdm_emg {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  HostMesh hm;
  int64_t N = 0;
  // stencils U (EMG_NC coefficients per node): K(sigma_i), K(sigma_i + sigma_e), the potential flow's Laplacian
  Buf<double> pos, dir, flow, coef_i, coef_ie, coef_lap, dinv, vm, rhs, phi, r, z, p0, q, partial,
      scal, tensor_i, tensor_e, tmp;
  Buf<unsigned char> mask;
  Buf<unsigned> counter;                       // last-block counter of the grid reductions
  cudaGraphExec_t graphs[1] = {nullptr};       // CG chunk of the bidomain solve
  int precond = FDM_EMG_PRECOND_MULTIGRID;     // of the bidomain solve
  std::vector<MgLevel*> mg;                    // multigrid hierarchy of K(sigma_i + sigma_e), built on first use
  bool have_dir = false, have_ops = false, have_map = false;
  int64_t n_tensor_i = 0, n_tensor_e = 0;
  // fiber -> mesh transfer (CSR over 3D nodes)
  Buf<int64_t> map_ptr, map_src;
  Buf<double> map_w, map_fsum;
  int64_t n_source = 0, n_mapped = 0;
  double default_value = 0.0;
  int last_iterations = 0;
  double last_residual = 0.0;
  float last_solve_ms = 0.f;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

int emg_fail(fdm_emg* m, int code, const std::string& msg)
{
  if (m)
    m->err = msg;
  else
    fdm::fdm_report_error(code, msg);
  return code;
}

#define EMG_CUDA(m, call)                                                                                   \
  do {                                                                                                      \
    cudaError_t e_ = (call);                                                                                \
    if (e_ != cudaSuccess)                                                                                  \
      return emg_fail(m, FDM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

#define EMG_BIND(m) EMG_CUDA(m, cudaSetDevice((m)->device))

// conjugate gradients on A x = b with A the symmetric stencil U (Dirichlet rows in mask: x keeps its value
// there and p, r vanish), Jacobi preconditioner dinv; nullspace: b's and x's means removed (constant null
// space).  Two kernels per iteration (direction + product, update), their reductions finished by the last
// block; chunks of 8 iterations run as one CUDA graph (captured on the first use for this right-hand side and
// solution vector).  Convergence: ||r||_2 <= max(rtol ||b||_2, atol) (unpreconditioned residual, from the
// recurrence), checked after every chunk.
// One V-cycle x = M^-1 b on level l (b, x, t, r: the level's right-hand side, result and two work vectors).
void vcycle(fdm_emg* m, size_t l, const double* U, const double* dinv, const double* b, double* x, double* t,
            double* r)
{
  cudaStream_t s = m->stream;
  const Grid g = m->mg[l]->g;
  const int64_t N = g.n_nodes();
  const int nb = blocks_for(N);
  if (l + 1 == m->mg.size()) {
    mg_coarsest_kernel<<<1, 1024, 0, s>>>(g, U, dinv, b, x, t, MG_COARSEST_SWEEPS);
    return;
  }
  MgLevel* c = m->mg[l + 1];
  mg_jacobi_kernel<<<nb, EMG_T, 0, s>>>(g, U, dinv, b, nullptr, t);
  mg_jacobi_kernel<<<nb, EMG_T, 0, s>>>(g, U, dinv, b, t, x);
  mg_residual_kernel<<<nb, EMG_T, 0, s>>>(g, U, b, x, r);
  mg_restrict_kernel<<<blocks_for(c->g.n_nodes()), EMG_T, 0, s>>>(m->mg[l]->map, r, c->b.p);
  vcycle(m, l + 1, c->U.p, c->dinv.p, c->b.p, c->x.p, c->t.p, c->r.p);
  mg_prolong_add_kernel<<<nb, EMG_T, 0, s>>>(m->mg[l]->map, c->x.p, x);
  mg_jacobi_kernel<<<nb, EMG_T, 0, s>>>(g, U, dinv, b, x, t);
  mg_jacobi_kernel<<<nb, EMG_T, 0, s>>>(g, U, dinv, b, t, x);
}

void mg_release(fdm_emg* m)
{
  for (MgLevel* L : m->mg)
    delete L;
  m->mg.clear();
}

// coarse nodes along one direction of n fine nodes: fine indices 0, 2, 4, ... and n - 1 (none coarsened
// below 3 nodes)
std::vector<int> coarse_indices(int n)
{
  std::vector<int> F;
  if (n <= 2) {
    for (int i = 0; i < n; i++)
      F.push_back(i);
    return F;
  }
  for (int i = 0; i < n; i += 2)
    F.push_back(i);
  if (F.back() != n - 1)
    F.push_back(n - 1);
  return F;
}

// the hierarchy of K(sigma_i + sigma_e): coarsen until at most MG_COARSEST nodes (or nothing coarsens)
int mg_build(fdm_emg* m)
{
  mg_release(m);
  MgLevel* L0 = new MgLevel();
  L0->g = m->hm.g;
  m->mg.push_back(L0);
  EMG_CUDA(m, L0->t.alloc(m->N));
  EMG_CUDA(m, L0->r.alloc(m->N));
  EMG_CUDA(m, L0->dinv.alloc(m->N));     // level 0: the l1 scaling of the fine operator
  mg_l1_kernel<<<blocks_for(m->N), EMG_T, 0, m->stream>>>(m->hm.g, m->coef_ie.p, L0->dinv.p);
  const double* Uf = m->coef_ie.p;
  while ((int)m->mg.size() < MG_MAX_LEVELS) {
    MgLevel* F = m->mg.back();
    if (F->g.n_nodes() <= MG_COARSEST)
      break;
    const int nf[3] = {F->g.nx, F->g.ny, F->g.nz};
    std::vector<int> Fi[3];
    bool coarsened = false;
    for (int d = 0; d < 3; d++) {
      Fi[d] = coarse_indices(nf[d]);
      coarsened = coarsened || (int)Fi[d].size() < nf[d];
    }
    if (!coarsened)
      break;
    std::vector<int> lo, rlo, rhi;
    std::vector<double> w;
    int off_lo[3], off_r[3];
    for (int d = 0; d < 3; d++) {
      const std::vector<int>& C = Fi[d];
      const int nc = (int)C.size();
      off_lo[d] = (int)lo.size();
      off_r[d] = (int)rlo.size();
      for (int i = 0, c = 0; i < nf[d]; i++) {
        while (c + 1 < nc && C[c + 1] <= i)
          c++;
        lo.push_back(c);
        w.push_back(c + 1 < nc ? double(i - C[c]) / double(C[c + 1] - C[c]) : 0.0);
      }
      for (int c = 0; c < nc; c++) {
        rlo.push_back(c == 0 ? 0 : C[c - 1] + 1);
        rhi.push_back(c == nc - 1 ? nf[d] - 1 : C[c + 1] - 1);
      }
    }
    MgLevel* Cl = new MgLevel();
    m->mg.push_back(Cl);
    Cl->g = Grid{(int)Fi[0].size(), (int)Fi[1].size(), (int)Fi[2].size()};
    const int64_t Nc = Cl->g.n_nodes();
    EMG_CUDA(m, F->lo.alloc(lo.size()));
    EMG_CUDA(m, F->w.alloc(w.size()));
    EMG_CUDA(m, F->rlo.alloc(rlo.size()));
    EMG_CUDA(m, F->rhi.alloc(rhi.size()));
    EMG_CUDA(m, cudaMemcpyAsync(F->lo.p, lo.data(), sizeof(int) * lo.size(), cudaMemcpyHostToDevice, m->stream));
    EMG_CUDA(m, cudaMemcpyAsync(F->w.p, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, m->stream));
    EMG_CUDA(m, cudaMemcpyAsync(F->rlo.p, rlo.data(), sizeof(int) * rlo.size(), cudaMemcpyHostToDevice, m->stream));
    EMG_CUDA(m, cudaMemcpyAsync(F->rhi.p, rhi.data(), sizeof(int) * rhi.size(), cudaMemcpyHostToDevice, m->stream));
    F->map.fine = F->g;
    F->map.coarse = Cl->g;
    for (int d = 0; d < 3; d++) {
      F->map.lo[d] = F->lo.p + off_lo[d];
      F->map.w[d] = F->w.p + off_lo[d];
      F->map.rlo[d] = F->rlo.p + off_r[d];
      F->map.rhi[d] = F->rhi.p + off_r[d];
    }
    for (auto* b : {&Cl->dinv, &Cl->b, &Cl->x, &Cl->t, &Cl->r})
      EMG_CUDA(m, b->alloc(Nc));
    EMG_CUDA(m, Cl->U.alloc(EMG_NC * Nc));
    mg_galerkin_kernel<<<blocks_for(Nc), EMG_T, 0, m->stream>>>(F->map, Uf, Cl->U.p);
    mg_l1_kernel<<<blocks_for(Nc), EMG_T, 0, m->stream>>>(Cl->g, Cl->U.p, Cl->dinv.p);
    EMG_CUDA(m, cudaGetLastError());
    Uf = Cl->U.p;
  }
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  return FDM_OK;
}

// after the operator or the preconditioner changes: the captured CG chunk and the hierarchy are rebuilt
void emg_invalidate(fdm_emg* m)
{
  for (auto& ge : m->graphs)
    if (ge) {
      cudaGraphExecDestroy(ge);
      ge = nullptr;
    }
  mg_release(m);
}

int cg_solve(fdm_emg* m, const double* U, const unsigned char* mask, bool nullspace, const double* b, double* x,
             double rtol, double atol, int max_it, int* iterations, double* residual, int graph_slot)
{
  // the multigrid preconditioner (bidomain operator only; the V-cycle replaces z = D^-1 r)
  const bool use_mg = graph_slot == 0 && m->precond == FDM_EMG_PRECOND_MULTIGRID && m->mg.size() > 1;
  const int64_t N = m->N;
  const Grid g = m->hm.g;
  const int nb = blocks_for(N);
  cudaStream_t s = m->stream;
  double* S = m->scal.p;
  double* P = m->partial.p;
  unsigned* C = m->counter.p;
  const double* bb = b;
  if (nullspace) {
    // b <- b - mean(b) (consistency of the singular system), into tmp
    sum_kernel<<<nb, EMG_T, 0, s>>>(N, b, nullptr, S, P, C);
    subtract_mean_kernel<<<nb, EMG_T, 0, s>>>(N, b, m->tmp.p, S);
    bb = m->tmp.p;
  }
  sum_kernel<<<nb, EMG_T, 0, s>>>(N, bb, bb, S, P, C);
  EMG_CUDA(m, cudaMemsetAsync(m->p0.p, 0, sizeof(double) * N, s));
  EMG_CUDA(m, cudaMemsetAsync(m->q.p, 0, sizeof(double) * N, s));
  cg_init_kernel<<<nb, EMG_T, 0, s>>>(g, U, mask, bb, x, m->r.p, m->z.p, m->dinv.p, S, P, C);
  if (use_mg) {
    vcycle(m, 0, U, m->mg[0]->dinv.p, m->r.p, m->z.p, m->mg[0]->t.p, m->mg[0]->r.p);
    cg_rz_kernel<<<nb, EMG_T, 0, s>>>(N, m->r.p, m->z.p, S, P, C, 1);
  }
  double hs[8];
  EMG_CUDA(m, cudaMemcpyAsync(hs, S, sizeof(hs), cudaMemcpyDeviceToHost, s));
  EMG_CUDA(m, cudaStreamSynchronize(s));
  // relative to ||b|| (to the initial residual where b vanishes: the Dirichlet problem, whose right-hand side
  // -K_fd u_d sits in the initial residual)
  const double bnorm = hs[CG_BB] > 0 ? std::sqrt(hs[CG_BB]) : std::sqrt(hs[CG_RR]);
  const double target = std::max(rtol * bnorm, atol);
  double rn = std::sqrt(hs[CG_RR]);
  // one iteration: direction and product, then the update
  auto iteration = [&]() {
    cg_direction_kernel<<<nb, EMG_T, 0, s>>>(g, U, mask, m->z.p, m->p0.p, m->q.p, S, P, C);
    if (use_mg) {
      cg_update_plain_kernel<<<nb, EMG_T, 0, s>>>(N, x, m->r.p, m->p0.p, m->q.p, S, P, C);
      vcycle(m, 0, U, m->mg[0]->dinv.p, m->r.p, m->z.p, m->mg[0]->t.p, m->mg[0]->r.p);
      cg_rz_kernel<<<nb, EMG_T, 0, s>>>(N, m->r.p, m->z.p, S, P, C, 0);
    } else {
      cg_update_kernel<<<nb, EMG_T, 0, s>>>(N, x, m->r.p, m->z.p, m->p0.p, m->q.p, m->dinv.p, S, P, C);
    }
  };
  // iterations per graph launch and convergence check: a multigrid iteration is long and few are needed
  const int CHUNK = use_mg ? 2 : 8;
  cudaGraphExec_t no_graph = nullptr;
  cudaGraphExec_t& ge = graph_slot >= 0 ? m->graphs[graph_slot] : no_graph;
  if (!ge && graph_slot >= 0) {
    cudaGraph_t gr = nullptr;
    EMG_CUDA(m, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int c = 0; c < CHUNK; c++)
      iteration();
    cudaError_t e = cudaStreamEndCapture(s, &gr);
    if (e == cudaSuccess)
      e = cudaGraphInstantiate(&ge, gr, 0);
    if (gr)
      cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
      ge = nullptr;
      return emg_fail(m, FDM_ERR_CUDA, std::string("conjugate gradients: graph capture: ") + cudaGetErrorString(e));
    }
  }
  int it = 0;
  while (rn > target && it < max_it) {
    if (ge && max_it - it >= CHUNK) {
      EMG_CUDA(m, cudaGraphLaunch(ge, s));
      it += CHUNK;
    } else {
      const int chunk = std::min(CHUNK, max_it - it);
      for (int c = 0; c < chunk; c++)
        iteration();
      it += chunk;
    }
    EMG_CUDA(m, cudaGetLastError());
    EMG_CUDA(m, cudaMemcpyAsync(hs, S, sizeof(hs), cudaMemcpyDeviceToHost, s));
    EMG_CUDA(m, cudaStreamSynchronize(s));
    rn = std::sqrt(hs[CG_RR]);
    if (!std::isfinite(rn))
      return emg_fail(m, FDM_ERR_NAN, "conjugate gradients: non-finite residual");
  }
  if (nullspace) {
    sum_kernel<<<nb, EMG_T, 0, s>>>(N, x, nullptr, S, P, C);
    subtract_mean_kernel<<<nb, EMG_T, 0, s>>>(N, x, x, S);
  }
  EMG_CUDA(m, cudaGetLastError());
  EMG_CUDA(m, cudaStreamSynchronize(s));
  if (iterations)
    *iterations = it;
  if (residual)
    *residual = rn;
  return FDM_OK;
}

int assemble(fdm_emg* m, const double* tensor, int64_t nt, const double* tensor2, int64_t nt2, double prefactor,
             int gauss, bool directional, double* coef)
{
  AssembleArgs a{};
  a.g = m->hm.g;
  a.pos = m->pos.p;
  a.dir = directional ? m->dir.p : nullptr;
  a.tensor = tensor;
  a.tensor2 = tensor2;
  a.n_tensor = nt;
  a.n_tensor2 = nt2;
  a.prefactor = prefactor;
  a.q = gauss_legendre(gauss);
  a.coef = coef;
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((m->N + 127) / 128, 148 * 16));
  assemble_kernel<<<nb, 128, 0, m->stream>>>(a);
  EMG_CUDA(m, cudaGetLastError());
  return FDM_OK;
}

} // namespace

namespace fdm {
// the fiber solver's Vm on the device, its node count and stream (fdm_host.cu)
int solver_vm_device(fdm_solver* s, const double** vm, int64_t* n_nodes, cudaStream_t* stream, int* device);
} // namespace fdm

extern "C" int fdm_emg_create(int nx, int ny, int nz, const double* node_positions, int device, fdm_emg** out)
{
  if (!out || !node_positions || nx < 2 || ny < 2 || nz < 2)
    return emg_fail(nullptr, FDM_ERR_ARG, "fdm_emg_create: at least 2 nodes per direction and node positions needed");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return emg_fail(nullptr, FDM_ERR_NO_DEVICE, "fdm_emg_create: no CUDA device");
  if (device < 0 || device >= ndev)
    return emg_fail(nullptr, FDM_ERR_ARG, "fdm_emg_create: device ordinal out of range");
  if (cudaSetDevice(device) != cudaSuccess)
    return emg_fail(nullptr, FDM_ERR_CUDA, "fdm_emg_create: cudaSetDevice failed");
  fdm_emg* m = new fdm_emg();
  m->device = device;
  m->hm.g = Grid{nx, ny, nz};
  m->N = m->hm.g.n_nodes();
  m->hm.pos.assign(node_positions, node_positions + 3 * m->N);
  // every element must have a positive Jacobian determinant at its corners
  for (int64_t e = 0; e < m->hm.g.n_elements(); e++) {
    double P[8][3];
    m->hm.element_points(e, P);
    for (int l = 0; l < 8; l++) {
      const double xi[3] = {(double)(l & 1), (double)((l >> 1) & 1), (double)(l >> 2)};
      double phi[8], dphi[8][3], inv[3][3];
      shape(xi, phi, dphi);
      const double det = jacobian(P, dphi, inv);
      if (!(det > 0) || !std::isfinite(det)) {
        delete m;
        return emg_fail(nullptr, FDM_ERR_ARG, "fdm_emg_create: element " + std::to_string(e) +
                                                  " is degenerate or inverted (node order: x fastest, then y, z)");
      }
    }
  }
  const int64_t N = m->N;
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = cudaEventCreate(&m->ev0);
  if (e == cudaSuccess)
    e = cudaEventCreate(&m->ev1);
  for (auto* b : {&m->pos, &m->dir})
    if (e == cudaSuccess)
      e = b->alloc(3 * N);
  for (auto* b : {&m->coef_i, &m->coef_ie})
    if (e == cudaSuccess)
      e = b->alloc(EMG_NC * N);
  for (auto* b : {&m->flow, &m->dinv, &m->vm, &m->rhs, &m->phi, &m->r, &m->z, &m->p0, &m->q, &m->tmp})
    if (e == cudaSuccess)
      e = b->alloc(N);
  if (e == cudaSuccess)
    e = m->partial.alloc(2 * EMG_MAX_BLOCKS);
  if (e == cudaSuccess)
    e = m->scal.alloc(8);
  if (e == cudaSuccess)
    e = m->counter.alloc(1);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(m->counter.p, 0, sizeof(unsigned), m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->pos.p, node_positions, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(m->vm.p, 0, sizeof(double) * N, m->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(m->phi.p, 0, sizeof(double) * N, m->stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(m->scal.p, 0, sizeof(double) * 8, m->stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) {
    std::string msg = std::string("fdm_emg_create: ") + cudaGetErrorString(e);
    fdm_emg_destroy(m);
    return emg_fail(nullptr, FDM_ERR_CUDA, msg);
  }
  *out = m;
  return FDM_OK;
}

extern "C" int fdm_emg_destroy(fdm_emg* m)
{
  if (!m)
    return FDM_OK;
  cudaSetDevice(m->device);
  if (m->stream)
    cudaStreamSynchronize(m->stream);
  for (auto* b : {&m->pos, &m->dir, &m->flow, &m->coef_i, &m->coef_ie, &m->coef_lap, &m->dinv, &m->vm, &m->rhs,
                  &m->phi, &m->r, &m->z, &m->p0, &m->q, &m->partial, &m->scal, &m->tensor_i, &m->tensor_e,
                  &m->tmp, &m->map_w, &m->map_fsum})
    b->release();
  for (auto& ge : m->graphs)
    if (ge)
      cudaGraphExecDestroy(ge);
  mg_release(m);
  m->mask.release();
  m->counter.release();
  m->map_ptr.release();
  m->map_src.release();
  if (m->ev0)
    cudaEventDestroy(m->ev0);
  if (m->ev1)
    cudaEventDestroy(m->ev1);
  if (m->stream)
    cudaStreamDestroy(m->stream);
  delete m;
  return FDM_OK;
}

extern "C" const char* fdm_emg_last_error(const fdm_emg* m)
{
  return m ? m->err.c_str() : fdm_last_error(nullptr);
}

extern "C" int fdm_emg_potential_flow(fdm_emg* m, int64_t n_dirichlet, const int64_t* nodes, const double* values,
                                      int gauss_points, double rtol, double atol, int max_iterations,
                                      int* iterations)
{
  if (!m || n_dirichlet < 1 || !nodes || !values || gauss_points < 1 || gauss_points > EMG_MAX_GAUSS ||
      max_iterations < 1)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_potential_flow: Dirichlet nodes and values, 1..7 Gauss points needed");
  EMG_BIND(m);
  const int64_t N = m->N;
  std::vector<unsigned char> mk(N, 0);
  std::vector<double> x0(N, 0.0);
  for (int64_t d = 0; d < n_dirichlet; d++) {
    if (nodes[d] < 0 || nodes[d] >= N)
      return emg_fail(m, FDM_ERR_ARG, "fdm_emg_potential_flow: Dirichlet node out of range");
    mk[nodes[d]] = 1;
    x0[nodes[d]] = values[d];
  }
  EMG_CUDA(m, m->coef_lap.alloc(EMG_NC * N));
  EMG_CUDA(m, m->mask.alloc(N));
  EMG_CUDA(m, m->tensor_i.alloc(9));
  const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  EMG_CUDA(m, cudaMemcpyAsync(m->tensor_i.p, eye, sizeof(eye), cudaMemcpyHostToDevice, m->stream));
  EMG_CUDA(m, cudaMemcpyAsync(m->mask.p, mk.data(), N, cudaMemcpyHostToDevice, m->stream));
  EMG_CUDA(m, cudaMemcpyAsync(m->flow.p, x0.data(), sizeof(double) * N, cudaMemcpyHostToDevice, m->stream));
  int rc = assemble(m, m->tensor_i.p, 1, nullptr, 0, 1.0, gauss_points, false, m->coef_lap.p);
  if (rc)
    return rc;
  const int nb = blocks_for(N);
  inverse_diag_kernel<<<nb, EMG_T, 0, m->stream>>>(N, m->coef_lap.p, m->mask.p, m->dinv.p);
  // free rows: K_ff u_f = -K_fd u_d (b = 0, x0 holding the Dirichlet values; Dirichlet rows masked)
  EMG_CUDA(m, cudaMemsetAsync(m->rhs.p, 0, sizeof(double) * N, m->stream));
  int its = 0;
  double res = 0.0;
  rc = cg_solve(m, m->coef_lap.p, m->mask.p, false, m->rhs.p, m->flow.p, rtol, atol, max_iterations, &its, &res, -1);
  if (rc)
    return rc;
  gradient_direction_kernel<<<nb, EMG_T, 0, m->stream>>>(m->hm.g, m->pos.p, m->flow.p, m->dir.p);
  EMG_CUDA(m, cudaGetLastError());
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  m->coef_lap.release();
  m->have_dir = true;
  m->have_ops = false;
  if (iterations)
    *iterations = its;
  return FDM_OK;
}

extern "C" int fdm_emg_set_direction(fdm_emg* m, const double* direction)
{
  if (!m || !direction)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_direction: bad argument");
  EMG_BIND(m);
  EMG_CUDA(m, cudaMemcpyAsync(m->dir.p, direction, sizeof(double) * 3 * m->N, cudaMemcpyHostToDevice, m->stream));
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  m->have_dir = true;
  m->have_ops = false;
  return FDM_OK;
}

extern "C" int fdm_emg_set_conductivity(fdm_emg* m, int64_t n_sigma_i, const double* sigma_i, int64_t n_sigma_e,
                                        const double* sigma_e, int gauss_points)
{
  if (!m || !sigma_i || !sigma_e || gauss_points < 1 || gauss_points > EMG_MAX_GAUSS)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_conductivity: bad argument");
  const int64_t ne = m->hm.g.n_elements();
  if ((n_sigma_i != 1 && n_sigma_i != ne) || (n_sigma_e != 1 && n_sigma_e != ne))
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_conductivity: one tensor for all elements or one per element");
  if (!m->have_dir)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_conductivity: call fdm_emg_potential_flow or fdm_emg_set_direction "
                                    "first");
  EMG_BIND(m);
  EMG_CUDA(m, m->tensor_i.alloc(9 * n_sigma_i));
  EMG_CUDA(m, m->tensor_e.alloc(9 * n_sigma_e));
  EMG_CUDA(m, cudaMemcpyAsync(m->tensor_i.p, sigma_i, sizeof(double) * 9 * n_sigma_i, cudaMemcpyHostToDevice,
                              m->stream));
  EMG_CUDA(m, cudaMemcpyAsync(m->tensor_e.p, sigma_e, sizeof(double) * 9 * n_sigma_e, cudaMemcpyHostToDevice,
                              m->stream));
  int rc = assemble(m, m->tensor_i.p, n_sigma_i, nullptr, 0, 1.0, gauss_points, true, m->coef_i.p);
  if (!rc)
    rc = assemble(m, m->tensor_i.p, n_sigma_i, m->tensor_e.p, n_sigma_e, 1.0, gauss_points, true, m->coef_ie.p);
  if (rc)
    return rc;
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  m->n_tensor_i = n_sigma_i;
  m->n_tensor_e = n_sigma_e;
  m->have_ops = true;
  emg_invalidate(m);
  return FDM_OK;
}

extern "C" int fdm_emg_set_fiber_mapping(fdm_emg* m, int64_t n_source, const double* positions, double xi_tolerance,
                                         double default_value, int64_t* n_mapped)
{
  if (!m || n_source < 0 || (n_source > 0 && !positions))
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_fiber_mapping: bad argument");
  EMG_BIND(m);
  if (xi_tolerance <= 0)
    xi_tolerance = 1e-1; // 00_construct.tpp:78-79
  const Grid g = m->hm.g;
  const int64_t ne = g.n_elements();
  // CSR over 3D nodes of (fiber node, factor), fiber nodes in increasing order per 3D node
  std::vector<std::vector<std::pair<int64_t, double>>> lists(m->N);
  int64_t mapped = 0, guess = 0;
  for (int64_t s = 0; s < n_source; s++) {
    const double* x = positions + 3 * s;
    double xi[3];
    // walk from the previous element towards the point, then fall back to all elements
    int64_t e = guess;
    double out = m->hm.locate(e, x, xi);
    for (int step = 0; step < g.nx + g.ny + g.nz && out > 1e-12; step++) {
      int ex = (int)(e % (g.nx - 1)), ey = (int)((e / (g.nx - 1)) % (g.ny - 1)),
          ez = (int)(e / ((int64_t)(g.nx - 1) * (g.ny - 1)));
      const int ox = ex, oy = ey, oz = ez;
      ex = std::min(std::max(ex + (xi[0] < 0 ? -1 : xi[0] > 1 ? 1 : 0), 0), g.nx - 2);
      ey = std::min(std::max(ey + (xi[1] < 0 ? -1 : xi[1] > 1 ? 1 : 0), 0), g.ny - 2);
      ez = std::min(std::max(ez + (xi[2] < 0 ? -1 : xi[2] > 1 ? 1 : 0), 0), g.nz - 2);
      if (ex == ox && ey == oy && ez == oz)
        break;
      e = g.element(ex, ey, ez);
      out = m->hm.locate(e, x, xi);
    }
    if (out > 1e-12) {
      double best = 1e300;
      int64_t be = 0;
      for (int64_t c = 0; c < ne; c++) {
        double t[3];
        const double o = m->hm.locate(c, x, t);
        if (o < best - 1e-15) {
          best = o;
          be = c;
          if (o <= 1e-12)
            break;
        }
      }
      e = be;
      out = m->hm.locate(e, x, xi);
    }
    if (out <= 1e-12) {
      // the lowest-numbered element containing the point (points on shared faces and edges)
      const int ex = (int)(e % (g.nx - 1)), ey = (int)((e / (g.nx - 1)) % (g.ny - 1)),
                ez = (int)(e / ((int64_t)(g.nx - 1) * (g.ny - 1)));
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            const int cx = ex + dx, cy = ey + dy, cz = ez + dz;
            if (cx < 0 || cy < 0 || cz < 0 || cx > g.nx - 2 || cy > g.ny - 2 || cz > g.nz - 2)
              continue;
            const int64_t c = g.element(cx, cy, cz);
            if (c >= e)
              continue;
            double t[3];
            if (m->hm.locate(c, x, t) <= 1e-12)
              e = c;
          }
      out = m->hm.locate(e, x, xi);
    }
    guess = e;
    if (out > xi_tolerance)
      continue; // outside the mesh: this fiber node maps nowhere
    mapped++;
    double phi[8], dphi[8][3];
    shape(xi, phi, dphi);
    const int ex = (int)(e % (g.nx - 1)), ey = (int)((e / (g.nx - 1)) % (g.ny - 1)),
              ez = (int)(e / ((int64_t)(g.nx - 1) * (g.ny - 1)));
    for (int l = 0; l < 8; l++) {
      double f = phi[l];
      if (std::fabs(f) < 1e-14)
        f = f >= 0 ? 1e-14 : -1e-14; // 00_construct.tpp:127-137
      lists[g.node(ex + (l & 1), ey + ((l >> 1) & 1), ez + (l >> 2))].push_back({s, f});
    }
  }
  std::vector<int64_t> ptr(m->N + 1, 0), src;
  std::vector<double> w, fsum(m->N, 0.0);
  for (int64_t n = 0; n < m->N; n++) {
    ptr[n + 1] = ptr[n] + (int64_t)lists[n].size();
    for (auto& pr : lists[n]) {
      src.push_back(pr.first);
      w.push_back(pr.second);
      fsum[n] += pr.second;
    }
  }
  EMG_CUDA(m, m->map_ptr.alloc(m->N + 1));
  EMG_CUDA(m, m->map_src.alloc(std::max<size_t>(src.size(), 1)));
  EMG_CUDA(m, m->map_w.alloc(std::max<size_t>(w.size(), 1)));
  EMG_CUDA(m, m->map_fsum.alloc(m->N));
  EMG_CUDA(m, cudaMemcpyAsync(m->map_ptr.p, ptr.data(), sizeof(int64_t) * (m->N + 1), cudaMemcpyHostToDevice,
                              m->stream));
  if (!src.empty()) {
    EMG_CUDA(m, cudaMemcpyAsync(m->map_src.p, src.data(), sizeof(int64_t) * src.size(), cudaMemcpyHostToDevice,
                                m->stream));
    EMG_CUDA(m, cudaMemcpyAsync(m->map_w.p, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, m->stream));
  }
  EMG_CUDA(m, cudaMemcpyAsync(m->map_fsum.p, fsum.data(), sizeof(double) * m->N, cudaMemcpyHostToDevice, m->stream));
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  m->n_source = n_source;
  m->n_mapped = mapped;
  m->default_value = default_value;
  m->have_map = true;
  if (n_mapped)
    *n_mapped = mapped;
  return FDM_OK;
}

extern "C" int fdm_emg_map_fibers(fdm_emg* m, fdm_solver* s)
{
  if (!m || !s || !m->have_map)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_map_fibers: call fdm_emg_set_fiber_mapping first");
  const double* vm = nullptr;
  int64_t n = 0;
  cudaStream_t ss = nullptr;
  int dev = 0;
  int rc = fdm::solver_vm_device(s, &vm, &n, &ss, &dev);
  if (rc)
    return emg_fail(m, rc, "fdm_emg_map_fibers: the fiber solver has no state");
  if (dev != m->device || n != m->n_source)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_map_fibers: the fiber solver's device or node count differs from the "
                                    "mapping's");
  EMG_BIND(m);
  // order after the fiber solver's work
  EMG_CUDA(m, cudaEventRecord(m->ev0, ss));
  EMG_CUDA(m, cudaStreamWaitEvent(m->stream, m->ev0, 0));
  map_kernel<<<blocks_for(m->N), EMG_T, 0, m->stream>>>(m->N, m->map_ptr.p, m->map_src.p, m->map_w.p, m->map_fsum.p, vm,
                                                         m->default_value, m->vm.p);
  EMG_CUDA(m, cudaGetLastError());
  // the fiber solver may overwrite Vm only after the transfer
  EMG_CUDA(m, cudaEventRecord(m->ev1, m->stream));
  EMG_CUDA(m, cudaStreamWaitEvent(ss, m->ev1, 0));
  return FDM_OK;
}

extern "C" int fdm_emg_map_values(fdm_emg* m, const double* fiber_values)
{
  if (!m || !m->have_map || (m->n_source > 0 && !fiber_values))
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_map_values: call fdm_emg_set_fiber_mapping first");
  EMG_BIND(m);
  Buf<double> src;
  EMG_CUDA(m, src.alloc(std::max<int64_t>(m->n_source, 1)));
  if (m->n_source > 0)
    EMG_CUDA(m, cudaMemcpyAsync(src.p, fiber_values, sizeof(double) * m->n_source, cudaMemcpyHostToDevice,
                                m->stream));
  map_kernel<<<blocks_for(m->N), EMG_T, 0, m->stream>>>(m->N, m->map_ptr.p, m->map_src.p, m->map_w.p, m->map_fsum.p,
                                                         src.p, m->default_value, m->vm.p);
  EMG_CUDA(m, cudaGetLastError());
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  return FDM_OK;
}

extern "C" int fdm_emg_set_vm(fdm_emg* m, const double* vm)
{
  if (!m || !vm)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_vm: bad argument");
  EMG_BIND(m);
  EMG_CUDA(m, cudaMemcpyAsync(m->vm.p, vm, sizeof(double) * m->N, cudaMemcpyHostToDevice, m->stream));
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  return FDM_OK;
}

extern "C" int fdm_emg_solve(fdm_emg* m, double rtol, double atol, int max_iterations, int initial_guess_nonzero,
                             int* iterations, double* residual)
{
  if (!m || !m->have_ops || max_iterations < 1)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_solve: call fdm_emg_set_conductivity first; max_iterations >= 1");
  EMG_BIND(m);
  const int64_t N = m->N;
  const int nb = blocks_for(N);
  if (m->precond == FDM_EMG_PRECOND_MULTIGRID && m->mg.empty()) {
    const int rb = mg_build(m);
    if (rb)
      return rb;
  }
  EMG_CUDA(m, cudaEventRecord(m->ev0, m->stream));
  // rhs = -K(sigma_i) Vm
  apply_kernel<<<nb, EMG_T, 0, m->stream>>>(m->hm.g, m->coef_i.p, m->vm.p, m->rhs.p, -1.0);
  inverse_diag_kernel<<<nb, EMG_T, 0, m->stream>>>(N, m->coef_ie.p, nullptr, m->dinv.p);
  if (!initial_guess_nonzero)
    EMG_CUDA(m, cudaMemsetAsync(m->phi.p, 0, sizeof(double) * N, m->stream));
  int its = 0;
  double res = 0.0;
  int rc = cg_solve(m, m->coef_ie.p, nullptr, true, m->rhs.p, m->phi.p, rtol, atol, max_iterations, &its, &res, 0);
  if (rc)
    return rc;
  EMG_CUDA(m, cudaEventRecord(m->ev1, m->stream));
  EMG_CUDA(m, cudaEventSynchronize(m->ev1));
  EMG_CUDA(m, cudaEventElapsedTime(&m->last_solve_ms, m->ev0, m->ev1));
  m->last_iterations = its;
  m->last_residual = res;
  if (iterations)
    *iterations = its;
  if (residual)
    *residual = res;
  return FDM_OK;
}

extern "C" int fdm_emg_set_preconditioner(fdm_emg* m, int type, int* levels)
{
  if (!m || (type != FDM_EMG_PRECOND_JACOBI && type != FDM_EMG_PRECOND_MULTIGRID))
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_set_preconditioner: FDM_EMG_PRECOND_JACOBI or FDM_EMG_PRECOND_MULTIGRID");
  EMG_BIND(m);
  if (type != m->precond)
    emg_invalidate(m);
  m->precond = type;
  if (type == FDM_EMG_PRECOND_MULTIGRID && m->have_ops && m->mg.empty()) {
    const int rc = mg_build(m);
    if (rc)
      return rc;
  }
  if (levels)
    *levels = type == FDM_EMG_PRECOND_MULTIGRID ? (int)m->mg.size() : 1;
  return FDM_OK;
}

extern "C" int fdm_emg_get(fdm_emg* m, int field, double* out)
{
  if (!m || !out)
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_get: bad argument");
  EMG_BIND(m);
  const double* src = nullptr;
  int64_t n = m->N;
  switch (field) {
  case FDM_EMG_PHI_E: src = m->phi.p; break;
  case FDM_EMG_VM: src = m->vm.p; break;
  case FDM_EMG_RHS: src = m->rhs.p; break;
  case FDM_EMG_FLOW_POTENTIAL: src = m->flow.p; break;
  case FDM_EMG_DIRECTION: src = m->dir.p; n = 3 * m->N; break;
  default: return emg_fail(m, FDM_ERR_ARG, "fdm_emg_get: unknown field");
  }
  EMG_CUDA(m, cudaMemcpyAsync(out, src, sizeof(double) * n, cudaMemcpyDeviceToHost, m->stream));
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  return FDM_OK;
}

extern "C" int fdm_emg_get_stencil(fdm_emg* m, int which, double* out)
{
  if (!m || !out || !m->have_ops || (which != 0 && which != 1))
    return emg_fail(m, FDM_ERR_ARG, "fdm_emg_get_stencil: operators not assembled or bad argument");
  EMG_BIND(m);
  const int64_t N = m->N;
  std::vector<double> U(EMG_NC * N);
  EMG_CUDA(m, cudaMemcpyAsync(U.data(), which == 0 ? m->coef_i.p : m->coef_ie.p, sizeof(double) * EMG_NC * N,
                              cudaMemcpyDeviceToHost, m->stream));
  EMG_CUDA(m, cudaStreamSynchronize(m->stream));
  // the full 27-point rows: the forward half as stored, the backward half from the neighbours' forward entries
  const Grid g = m->hm.g;
  for (int64_t n = 0; n < N; n++) {
    const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((int64_t)g.nx * g.ny));
    for (int q = 0; q < 27; q++) {
      int dx, dy, dz;
      stencil_offset(q, dx, dy, dz);
      double v = 0.0;
      if (i + dx >= 0 && i + dx < g.nx && j + dy >= 0 && j + dy < g.ny && k + dz >= 0 && k + dz < g.nz) {
        if (q >= 13)
          v = U[(q - 13) * N + n];
        else
          v = U[(13 - q) * N + n + dx + (int64_t)g.nx * (dy + (int64_t)g.ny * dz)];
      }
      out[q * N + n] = v;
    }
  }
  return FDM_OK;
}

extern "C" int fdm_emg_timing(const fdm_emg* m, double* last_solve_ms, int* last_iterations, double* last_residual)
{
  if (!m)
    return FDM_ERR_ARG;
  if (last_solve_ms)
    *last_solve_ms = m->last_solve_ms;
  if (last_iterations)
    *last_iterations = m->last_iterations;
  if (last_residual)
    *last_residual = m->last_residual;
  return FDM_OK;
}
