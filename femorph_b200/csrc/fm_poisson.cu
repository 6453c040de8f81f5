// Poisson solver: femPoissonSolver::solve (femSolver.cpp:409-654), the
// implicit neighbour of the explicit element loops.
//
// Host: the element matrices and source vectors of the reference's
// irSecondOrder Gauss loops (femElement::formPoissonMatrix /
// formPoissonSource, femElement.cpp:903-981) in parallel over elements, then
// the assembled matrix in CSR form with every entry summed in element order
// (the order of the reference's assembly loop, femSolver.cpp:446-459), the
// right-hand side (sources in ELSOURCE row order, then the face Neumann
// values, femSolver.cpp:478-558) and the Dirichlet rows.
// Device: conjugate gradients with a Jacobi preconditioner.  Per iteration
// three kernels: q = K p with the partial sums of p.q, the updates of x, r, z
// with the partial sums of r.z and r.r, and p = z + beta p; the last block of
// the first two (ticket counter, no waiting) sums the block partials in block
// order and forms alpha / beta, so every reduction has a fixed order and the
// iterates do not change from run to run.  Blocks of FM_CG_GRAPH iterations
// are replayed from one captured CUDA graph; the device counts the
// iterations and raises a done flag that makes the remaining launches of a
// block return at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "fm_internal.hpp"

namespace fm {
int fail(int code, const std::string& msg);
}

using fm::fail;

namespace {

constexpr int kThreads = 256;
// lanes summing one matrix row (a tet4 row has ~15 entries, a hexa8 row
// ~27); measured on the 96^3 Kuhn-tet cube: 8 lanes 0.128 ms an iteration,
// 4 lanes 0.088 ms, 2 lanes 0.086 ms
constexpr int kRowLanes = 4;
constexpr int FM_CG_GRAPH = 16;

// ---- element kinematics on the host (reference Gauss loops) ----
// irSecondOrder (femIntegrationRule.cpp): tet4 4 points, weight (1/6)(1/4);
// hexa8 2x2x2 points at +-1/sqrt(3) in the reference's order, weight 1.
struct Rule {
  int ngp;
  double q[8][3];
  double w[8];
};
void make_rule(int npe, Rule& r) {
  if (npe == 4) {
    const double a = 0.58541020, b = 0.13819660;
    const double t[4][3] = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    r.ngp = 4;
    for (int g = 0; g < 4; ++g) {
      for (int k = 0; k < 3; ++k) r.q[g][k] = t[g][k];
      r.w[g] = (1.0 / 6.0) * (1.0 / 4.0);
    }
  } else {
    const double s = 1.0 / std::sqrt(3.0);
    const double t[8][3] = {{-s, -s, s}, {s, -s, s}, {s, s, s}, {-s, s, s},
                            {-s, -s, -s}, {s, -s, -s}, {s, s, -s}, {-s, s, -s}};
    r.ngp = 8;
    for (int g = 0; g < 8; ++g) {
      for (int k = 0; k < 3; ++k) r.q[g][k] = t[g][k];
      r.w[g] = 8.0 * (1.0 / 8.0);
    }
  }
}
// hexa8 corner signs (femHexa8.cpp:13-42, VTK node order): x -++- -++-,
// y --++ --++, z ---- ++++
__host__ __device__ inline double hx(int a) { return ((a & 3) == 1 || (a & 3) == 2) ? 1.0 : -1.0; }
__host__ __device__ inline double hy(int a) { return (a & 2) ? 1.0 : -1.0; }
__host__ __device__ inline double hz(int a) { return (a & 4) ? 1.0 : -1.0; }

// Shape values (femTetra4.cpp:295-301, femHexa8.cpp:13-26).
__host__ __device__ inline void shape_values(int npe, const double q[3], double N[8]) {
  if (npe == 4) {
    N[0] = q[0];
    N[1] = q[1];
    N[2] = q[2];
    N[3] = 1.0 - q[0] - q[1] - q[2];
  } else {
    for (int a = 0; a < 8; ++a)
      N[a] = (1.0 / 8.0) * (1.0 + q[0] * hx(a)) * (1.0 + q[1] * hy(a)) * (1.0 + q[2] * hz(a));
  }
}
// Local derivatives (femTetra4.cpp:304-330, femHexa8.cpp:28-42).
__host__ __device__ inline void shape_derivs(int npe, const double q[3], double dN[8][3]) {
  if (npe == 4) {
    for (int a = 0; a < 4; ++a)
      for (int k = 0; k < 3; ++k) dN[a][k] = (a == k) ? 1.0 : (a == 3 ? -1.0 : 0.0);
  } else {
    for (int a = 0; a < 8; ++a) {
      dN[a][0] = (1.0 / 8.0) * hx(a) * (1.0 + q[1] * hy(a)) * (1.0 + q[2] * hz(a));
      dN[a][1] = (1.0 / 8.0) * hy(a) * (1.0 + q[0] * hx(a)) * (1.0 + q[2] * hz(a));
      dN[a][2] = (1.0 / 8.0) * hz(a) * (1.0 + q[0] * hx(a)) * (1.0 + q[1] * hy(a));
    }
  }
}
// Jacobian J[a][b] = sum_n dN[n][a] x[n][b] (femElement.cpp:104-127) from
// the local derivatives dN at the point.
__host__ __device__ inline void jacobian(int npe, const double xe[8][3], const double dN[8][3], double J[3][3]) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = 0.0;
      for (int n = 0; n < npe; ++n) t += dN[n][a] * xe[n][b];
      J[a][b] = t;
    }
}
// Its determinant by the cofactors of the first row (femUtils.cpp:729-731).
__host__ __device__ inline double det3(const double J[3][3]) {
  const double c00 = J[1][1] * J[2][2] - J[2][1] * J[1][2];
  const double c01 = J[1][0] * J[2][2] - J[1][2] * J[2][0];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  return J[0][0] * c00 - J[0][1] * c01 + J[0][2] * c02;
}
// detJ at local point q alone (femElement::evalJacobian, femElement.cpp:149-186).
__host__ __device__ inline double jacobian_det(int npe, const double xe[8][3], const double q[3]) {
  double dN[8][3], J[3][3];
  shape_derivs(npe, q, dN);
  jacobian(npe, xe, dN, J);
  return det3(J);
}
// The Jacobian, its cofactor inverse and determinant (femUtils.cpp:716-770),
// global derivatives gd[n][b] = sum_c inv[b][c] dN[n][c] (femElement.cpp:
// 345-352).
__host__ __device__ inline double global_derivs(int npe, const double xe[8][3], const double q[3], double gd[8][3]) {
  double dN[8][3], J[3][3];
  shape_derivs(npe, q, dN);
  jacobian(npe, xe, dN, J);
  const double c00 = J[1][1] * J[2][2] - J[2][1] * J[1][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = det3(J);
  const double id = 1.0 / det;
  double inv[3][3];
  inv[0][0] = c00 * id;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  inv[1][2] = (J[1][0] * J[0][2] - J[0][0] * J[1][2]) * id;
  inv[2][0] = c02 * id;
  inv[2][1] = (J[2][0] * J[0][1] - J[0][0] * J[2][1]) * id;
  inv[2][2] = (J[0][0] * J[1][1] - J[1][0] * J[0][1]) * id;
  for (int n = 0; n < npe; ++n)
    for (int b = 0; b < 3; ++b) {
      double t = 0.0;
      for (int c = 0; c < 3; ++c) t += inv[b][c] * dN[n][c];
      gd[n][b] = t;
    }
  return det;
}

// Element matrix of femElement::formPoissonMatrix (femElement.cpp:903-944).
// A tet4's local derivatives do not depend on the point, so its derivatives,
// determinant and products are the same at every Gauss point: they are
// formed once and added once a point, which gives the reference loop's sums.
void element_matrix(int npe, const Rule& r, const double xe[8][3], const double diff[3], double K[8][8]) {
  for (int a = 0; a < npe; ++a)
    for (int b = 0; b < npe; ++b) K[a][b] = 0.0;
  double gd[8][3], detJ = 0.0, S[8][8];
  for (int g = 0; g < r.ngp; ++g) {
    if (g == 0 || npe == 8) {
      detJ = global_derivs(npe, xe, r.q[g], gd);
      for (int a = 0; a < npe; ++a)
        for (int b = 0; b < npe; ++b) {
          double s = 0.0;
          for (int d = 0; d < 3; ++d) s += diff[d] * gd[a][d] * gd[b][d];
          S[a][b] = s;
        }
    }
    for (int a = 0; a < npe; ++a)
      for (int b = 0; b < npe; ++b) K[a][b] += S[a][b] * detJ * r.w[g];
  }
}
// Element source of femElement::formPoissonSource (femElement.cpp:949-981)
// (a tet4's determinant formed once, as above).
void element_source(int npe, const Rule& r, const double xe[8][3], double value, double f[8]) {
  for (int a = 0; a < npe; ++a) f[a] = 0.0;
  double detJ = 0.0;
  for (int g = 0; g < r.ngp; ++g) {
    double N[8];
    shape_values(npe, r.q[g], N);
    if (g == 0 || npe == 8) detJ = jacobian_det(npe, xe, r.q[g]);
    for (int a = 0; a < npe; ++a) f[a] += N[a] * value * detJ * r.w[g];
  }
}

// ---- device kernels ----
// scal: [0] r.z  [1] p.q  [2] alpha  [3] beta  [4] r.r  [5] b.b  [6] tol^2 b.b  [7] average
// ctl:  [0] done  [1] iterations  [2] error  [3] max iterations  [4] ticket
struct Cg {
  const int32_t* rowp;
  const int32_t* col;
  const double* val;
  const double* dinv;
  const double* b;      // right-hand side with the Dirichlet rows set to 0 (their residual at x0)
  const double* xinit;  // x0: the Dirichlet values on their rows, 0 elsewhere
  double *x, *r, *z, *p, *q;
  double* part;  // 2 x blocks partial sums
  double* scal;
  int32_t* ctl;
  int64_t n;
};

// Block sum in a fixed tree order (lane order within a warp, then warp
// order); the result is valid in thread 0.
__device__ inline double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = l < (int)(blockDim.x >> 5) ? sh[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// Stores this block's two partials; returns true in every thread of the
// block that arrives last (fence, ticket, no waiting), after which that
// block's thread 0 sums all blocks' partials in block order into s0 / s1.
__device__ inline bool last_block_sums(const Cg& c, double v0, double v1, double* s0, double* s1) {
  __shared__ double sh[32];
  __shared__ bool last;
  v0 = block_sum(v0, sh);
  v1 = block_sum(v1, sh);
  if (threadIdx.x == 0) {
    c.part[2 * blockIdx.x] = v0;
    c.part[2 * blockIdx.x + 1] = v1;
    __threadfence();
    const unsigned t = atomicAdd(reinterpret_cast<unsigned*>(c.ctl + 4), 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // every thread of the last block sums a fixed strided subset of the block
  // partials, then the block sum (fixed order throughout)
  double a = 0.0, b = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
    a += c.part[2 * k];
    b += c.part[2 * k + 1];
  }
  a = block_sum(a, sh);
  b = block_sum(b, sh);
  if (threadIdx.x == 0) {
    *s0 = a;
    *s1 = b;
    c.ctl[4] = 0;
  }
  return true;
}

// x = x0 (the Dirichlet values on their rows: those rows are identity rows
// whose columns the other rows have moved to the right-hand side, so their
// residual is 0 from the start and they keep their exact values), r = b - K x0
// = b with the Dirichlet rows at 0, z = D^-1 r, p = z.
__global__ void __launch_bounds__(kThreads) cg_init_kernel(Cg c) {
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < c.n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = c.b[i], zi = c.dinv[i] * ri;
    c.x[i] = c.xinit[i];
    c.r[i] = ri;
    c.z[i] = zi;
    c.p[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  double s0, s1;
  if (last_block_sums(c, rz, rr, &s0, &s1) && threadIdx.x == 0) {
    c.scal[0] = s0;
    c.scal[4] = s1;
    c.ctl[1] = 0;
    c.ctl[2] = 0;
    c.ctl[0] = (s1 <= c.scal[6] || c.ctl[3] <= 0) ? 1 : 0;  // x0 meets the tolerance, or no iterations asked
  }
}

// q = K p (kRowLanes lanes a row, their sums added in a fixed shuffle order)
// and p.q; the last block forms alpha = r.z / p.q.
__global__ void __launch_bounds__(kThreads) cg_spmv_kernel(Cg c) {
  if (c.ctl[0]) return;
  // each warp takes 32 / kRowLanes consecutive rows a pass; the pass loop
  // is warp-uniform, so every lane reaches the shuffles
  const int lane = threadIdx.x % kRowLanes;
  constexpr int kRowsPerWarp = 32 / kRowLanes;
  const int64_t warp = blockIdx.x * (int64_t)(blockDim.x / 32) + threadIdx.x / 32;
  const int64_t stride = (int64_t)gridDim.x * (blockDim.x / 32) * kRowsPerWarp;
  double pq = 0.0;
  for (int64_t base = warp * kRowsPerWarp; base < c.n; base += stride) {
    const int64_t i = base + (threadIdx.x % 32) / kRowLanes;
    double s = 0.0;
    if (i < c.n) {
      // a lane's entries k0 + lane, + kRowLanes, ... in order, four a pass:
      // the column ids, then the values and gathers of the pass are loaded
      // together (one round trip each instead of one an entry)
      const int32_t k0 = c.rowp[i], k1 = c.rowp[i + 1];
      for (int32_t kb = k0 + lane; kb < k1; kb += 4 * kRowLanes) {
        int32_t cj[4];
        double vj[4], pj[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int32_t k = kb + u * kRowLanes;
          cj[u] = k < k1 ? c.col[k] : 0;
          vj[u] = k < k1 ? c.val[k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) pj[u] = c.p[cj[u]];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (kb + u * kRowLanes < k1) s += vj[u] * pj[u];
      }
    }
#pragma unroll
    for (int o = kRowLanes / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, kRowLanes);
    if (lane == 0 && i < c.n) {
      c.q[i] = s;
      pq += c.p[i] * s;
    }
  }
  double s0, s1;
  if (last_block_sums(c, pq, 0.0, &s0, &s1) && threadIdx.x == 0) {
    c.scal[1] = s0;
    if (!(s0 > 0.0) || !isfinite(s0)) {
      c.ctl[2] = 1;  // breakdown: K not positive definite on p, or a NaN
      c.ctl[0] = 1;
    } else {
      c.scal[2] = c.scal[0] / s0;
    }
  }
}

// x += alpha p, r -= alpha q, z = D^-1 r, with r.z and r.r; the last block
// counts the iteration, tests convergence and forms beta.
__global__ void __launch_bounds__(kThreads) cg_update_kernel(Cg c) {
  if (c.ctl[0]) return;
  const double alpha = c.scal[2];
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < c.n; i += (int64_t)gridDim.x * blockDim.x) {
    c.x[i] += alpha * c.p[i];
    const double ri = c.r[i] - alpha * c.q[i];
    const double zi = c.dinv[i] * ri;
    c.r[i] = ri;
    c.z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  double s0, s1;
  if (last_block_sums(c, rz, rr, &s0, &s1) && threadIdx.x == 0) {
    const int it = c.ctl[1] + 1;
    c.ctl[1] = it;
    c.scal[4] = s1;
    if (!isfinite(s1)) {
      c.ctl[2] = 1;
      c.ctl[0] = 1;
    } else if (s1 <= c.scal[6] || it >= c.ctl[3]) {
      c.ctl[0] = 1;
    } else {
      c.scal[3] = s0 / c.scal[0];
      c.scal[0] = s0;
    }
  }
}

__global__ void __launch_bounds__(kThreads) cg_direction_kernel(Cg c) {
  if (c.ctl[0]) return;
  const double beta = c.scal[3];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < c.n; i += (int64_t)gridDim.x * blockDim.x)
    c.p[i] = c.z[i] + beta * c.p[i];
}

// Average of x in fixed order (FM_POISSON_PPE subtracts it).
__global__ void __launch_bounds__(kThreads) avg_kernel(Cg c) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < c.n; i += (int64_t)gridDim.x * blockDim.x)
    s += c.x[i];
  double s0, s1;
  if (last_block_sums(c, s, 0.0, &s0, &s1) && threadIdx.x == 0) c.scal[7] = s0 / (double)c.n;
}
// out = x - shift (shift = the average for FM_POISSON_PPE, else 0).
__global__ void __launch_bounds__(kThreads) shift_kernel(const double* x, const double* scal, int ppe, int64_t n,
                                                         double* out) {
  const double a = ppe ? scal[7] : 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = x[i] - a;
}

// Element wall distance of evalDistanceFromPoissonSolution
// (femSolver.cpp:366-403): the solution and its gradient at local
// coordinates (0, 0, 0) (a vertex of the tet4 reference element, the centre
// of the hexa8 one), d = -|grad| + sqrt(|grad|^2 + 2 phi).
__global__ void __launch_bounds__(kThreads) distance_kernel(const double* coords, const int32_t* conn, int npe,
                                                            int64_t ne, const double* x, double* dist) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    double xe[8][3], u[8];
    for (int a = 0; a < npe; ++a) {
      const int32_t v = conn[e * npe + a];
      xe[a][0] = coords[3 * (int64_t)v];
      xe[a][1] = coords[3 * (int64_t)v + 1];
      xe[a][2] = coords[3 * (int64_t)v + 2];
      u[a] = x[v];
    }
    const double q0[3] = {0.0, 0.0, 0.0};
    double N[8], gd[8][3];
    shape_values(npe, q0, N);
    global_derivs(npe, xe, q0, gd);
    double phi = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int a = 0; a < npe; ++a) {
      phi += N[a] * u[a];
      g0 += gd[a][0] * u[a];
      g1 += gd[a][1] * u[a];
      g2 += gd[a][2] * u[a];
    }
    const double g2n = g0 * g0 + g1 * g1 + g2 * g2;
    dist[e] = -sqrt(g2n) + sqrt(g2n + 2.0 * phi);
  }
}

struct DeviceRestore {
  int prev = -1;
  DeviceRestore() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceRestore() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

struct fm_poisson {
  int32_t device = 0, npe = 4, problem = 0;
  int64_t N = 0, E = 0, nnz = 0;
  int blocks = 1;   // grid of the CG kernels (rows)
  int eblocks = 1;  // grid of the element kernel (wall distance)
  bool has_result = false;
  // device arrays (one allocation)
  void* block = nullptr;
  Cg c{};
  double* coords = nullptr;
  int32_t* conn = nullptr;
  double* out = nullptr;   // x with the PPE average removed
  double* dist = nullptr;  // FM_POISSON_DISTANCE element distances
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int32_t* h_ctl = nullptr;  // pinned copy of the control words
  double* h_scal = nullptr;
  double bb = 0.0;           // |b|^2 of the whole right-hand side
  // host copies for the VTK writer (fm_poisson_write_vtk): the model's
  // coordinates, the fixed connectivity, the diffusivity rows and the source,
  // Neumann and Dirichlet markers of femModel::ExportToVTKLegacy
  fm::PoissonHostView view{};
  std::vector<double> h_coords, h_diff, h_src, h_neu, h_dir;
  std::vector<int32_t> h_conn;
};

#define PCK(x)                                                                                         \
  do {                                                                                                 \
    cudaError_t _e = (x);                                                                              \
    if (_e != cudaSuccess) return fail(FM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); \
  } while (0)

extern "C" {

FM_API int fm_poisson_destroy(fm_poisson* s) {
  if (!s) return FM_OK;
  DeviceRestore restore;
  cudaSetDevice(s->device);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->block) cudaFree(s->block);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_scal) cudaFreeHost(s->h_scal);
  delete s;
  return FM_OK;
}

static int poisson_create(const fm_poisson_desc* d, int32_t device, fm_poisson** out) {
  if (!d || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  const int npe = d->elem_type;
  if (npe != 4 && npe != 8) return fail(FM_ERR_INVALID, "elem_type must be FM_TET4 or FM_HEXA8");
  if (d->problem < FM_POISSON_CLASSIC || d->problem > FM_POISSON_DISTANCE) return fail(FM_ERR_INVALID, "bad problem type");
  const int64_t N = d->n_nodes, E = d->n_elems;
  if (N <= 0 || E <= 0 || !d->coords || !d->conn || !d->diffusivity) return fail(FM_ERR_INVALID, "empty mesh");
  if (N >= INT32_MAX || E * npe >= INT32_MAX) return fail(FM_ERR_INVALID, "mesh too large for 32-bit indices");
  for (int64_t i = 0; i < E * npe; ++i)
    if (d->conn[i] < 0 || d->conn[i] >= N) return fail(FM_ERR_INVALID, "connectivity out of range");
  if ((d->n_sources > 0 && (!d->source_elem || !d->source_value)) ||
      (d->n_neumann > 0 && (!d->neumann_off || !d->neumann_nodes || !d->neumann_value)) ||
      (d->n_dirichlet > 0 && (!d->dir_node || !d->dir_value)))
    return fail(FM_ERR_INVALID, "null boundary / source array");
  for (int64_t k = 0; k < d->n_sources; ++k)
    if (d->source_elem[k] < 0 || d->source_elem[k] >= E) return fail(FM_ERR_INVALID, "ELSOURCE element out of range");
  if (d->n_neumann < 0 || d->n_sources < 0 || d->n_dirichlet < 0) return fail(FM_ERR_INVALID, "negative count");
  if (d->n_neumann > 0 && d->neumann_off[0] < 0) return fail(FM_ERR_INVALID, "FACENEUMANN offsets must start at >= 0");
  for (int64_t k = 0; k < d->n_neumann; ++k) {
    if (d->neumann_off[k + 1] <= d->neumann_off[k]) return fail(FM_ERR_INVALID, "FACENEUMANN row without nodes");
    for (int32_t j = d->neumann_off[k]; j < d->neumann_off[k + 1]; ++j)
      if (d->neumann_nodes[j] < 0 || d->neumann_nodes[j] >= N) return fail(FM_ERR_INVALID, "FACENEUMANN node out of range");
  }
  for (int64_t k = 0; k < d->n_dirichlet; ++k)
    if (d->dir_node[k] < 0 || d->dir_node[k] >= N) return fail(FM_ERR_INVALID, "NODEDIRBC node out of range");

  // femModel::FixedElementConnectivities (femModel.cpp:3554-3569), which the
  // reference's Poisson driver runs after reading the model (main.cpp:491):
  // an element whose smallest Jacobian determinant over the irSecondOrder
  // points is <= 0 gets one swap, tet4 nodes 0 / 1 (femTetra4.cpp:160-170),
  // hexa8 nodes 2 / 3 and 6 / 7 (femHexa8.cpp:93-103)
  Rule rule;
  make_rule(npe, rule);
  fm::hvec<int32_t> cfix((size_t)(E * npe));
  fm::parallel_blocks(E, [&](int64_t eb, int64_t ee, int) {
    for (int64_t e = eb; e < ee; ++e) {
      for (int a = 0; a < npe; ++a) cfix[e * npe + a] = d->conn[e * npe + a];
      double xe[8][3], mn = 1e308;
      for (int a = 0; a < npe; ++a)
        for (int k = 0; k < 3; ++k) xe[a][k] = d->coords[3 * (int64_t)cfix[e * npe + a] + k];
      // a tet4's Jacobian is the same at every point
      for (int g = 0; g < (npe == 4 ? 1 : rule.ngp); ++g) mn = std::min(mn, jacobian_det(npe, xe, rule.q[g]));
      if (mn <= 0.0) {
        int32_t* c = &cfix[e * npe];
        if (npe == 4) {
          std::swap(c[0], c[1]);
        } else {
          std::swap(c[2], c[3]);
          std::swap(c[6], c[7]);
        }
      }
    }
  }, 4096);
  const int32_t* conn = cfix.data();
  // element matrices, in parallel over elements
  const int m2 = npe * npe;
  fm::hvec<double> Ke((size_t)E * m2);
  fm::parallel_blocks(E, [&](int64_t eb, int64_t ee, int) {
    for (int64_t e = eb; e < ee; ++e) {
      double xe[8][3], K[8][8];
      for (int a = 0; a < npe; ++a)
        for (int k = 0; k < 3; ++k) xe[a][k] = d->coords[3 * (int64_t)conn[e * npe + a] + k];
      element_matrix(npe, rule, xe, d->diffusivity + 3 * e, K);
      for (int a = 0; a < npe; ++a)
        for (int b = 0; b < npe; ++b) Ke[(size_t)e * m2 + a * npe + b] = K[a][b];
    }
  }, 1024);
  // node -> incident (element, corner) in element order: counts per
  // contiguous element range, each range's entries of a node placed after
  // those of the ranges before it, the ranges filled on the host threads
  const int64_t hwt = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  std::vector<int32_t> ioff(N + 1, 0);
  std::vector<int32_t> inc(E * npe);
  {
    const int64_t nr = std::min<int64_t>(hwt, std::max<int64_t>(1, E / 65536));
    std::vector<std::vector<int32_t>> at(nr);
    auto ranges = [&](auto&& f) {
      std::vector<std::thread> th;
      for (int64_t r = 0; r < nr; ++r) th.emplace_back([&, r] { f(r, E * r / nr * npe, E * (r + 1) / nr * npe); });
      for (auto& x : th) x.join();
    };
    ranges([&](int64_t r, int64_t i0, int64_t i1) {
      at[r].assign(N, 0);
      for (int64_t i = i0; i < i1; ++i) at[r][conn[i]]++;
    });
    fm::parallel_blocks(N, [&](int64_t vb, int64_t ve, int) {
      for (int64_t v = vb; v < ve; ++v) {
        int32_t c = 0;
        for (int64_t r = 0; r < nr; ++r) c += at[r][v];
        ioff[v + 1] = c;
      }
    }, 1 << 14);
    for (int64_t v = 0; v < N; ++v) ioff[v + 1] += ioff[v];
    fm::parallel_blocks(N, [&](int64_t vb, int64_t ve, int) {
      for (int64_t v = vb; v < ve; ++v) {
        int32_t pos = ioff[v];
        for (int64_t r = 0; r < nr; ++r) {
          const int32_t c = at[r][v];
          at[r][v] = pos;
          pos += c;
        }
      }
    }, 1 << 14);
    ranges([&](int64_t r, int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i) inc[at[r][conn[i]]++] = (int32_t)i;
    });
  }
  // Dirichlet rows (a later row of the same node wins, as ReplaceGlobalValue)
  std::vector<int32_t> dir_of(N, -1);
  for (int64_t k = 0; k < d->n_dirichlet; ++k) dir_of[d->dir_node[k]] = (int32_t)k;
  // right-hand side: sources in row order, then the Neumann vector (its own
  // sums in row order) added node by node (femSolver.cpp:478-558)
  std::vector<double> rhs(N, 0.0);
  {
    // element vectors in parallel, added in row order
    fm::hvec<double> fs((size_t)d->n_sources * npe);
    fm::parallel_blocks(d->n_sources, [&](int64_t kb, int64_t ke, int) {
      for (int64_t k = kb; k < ke; ++k) {
        const int64_t e = d->source_elem[k];
        double xe[8][3];
        for (int a = 0; a < npe; ++a)
          for (int q = 0; q < 3; ++q) xe[a][q] = d->coords[3 * (int64_t)conn[e * npe + a] + q];
        element_source(npe, rule, xe, d->source_value[k], &fs[(size_t)k * npe]);
      }
    }, 4096);
    for (int64_t k = 0; k < d->n_sources; ++k) {
      const int64_t e = d->source_elem[k];
      for (int a = 0; a < npe; ++a) rhs[conn[e * npe + a]] += fs[(size_t)k * npe + a];
    }
  }
  {
    std::vector<double> nv(N, 0.0);
    for (int64_t k = 0; k < d->n_neumann; ++k) {
      const int32_t j0 = d->neumann_off[k], j1 = d->neumann_off[k + 1];
      for (int32_t j = j0; j < j1; ++j) nv[d->neumann_nodes[j]] += d->neumann_value[k] / (double)(j1 - j0);
    }
    for (int64_t v = 0; v < N; ++v) rhs[v] += nv[v];
  }
  // CSR rows (columns sorted), each entry summed over the incident elements
  // in element order; Dirichlet rows become identity rows with the value on
  // the right-hand side, and their columns move to the right-hand side of
  // the other rows (same solution, symmetric matrix)
  // One pass over contiguous row blocks on the host threads: each block
  // forms its rows' sorted columns and summed values into its own arrays,
  // which are then placed at the block's offset.
  std::vector<int32_t> rowp(N + 1, 0);
  fm::hvec<int32_t> rowlen(N);
  std::vector<double> bvec(N), dinv(N);
  const int64_t nblk = std::min<int64_t>(hwt, std::max<int64_t>(1, N / 2048));
  std::vector<std::vector<int32_t>> bcol(nblk);
  std::vector<std::vector<double>> bval(nblk);
  auto rows = [&](int64_t kb) {
    std::vector<int32_t>& lc = bcol[kb];
    std::vector<double>& lv = bval[kb];
    std::vector<int32_t> cl;
    // the row's distinct columns (open addressing, at most half full) with
    // their positions in the sorted row
    std::vector<int32_t> hkey(64, -1), hval(64), hused;
    uint32_t hmask = 63;
    auto hslot = [&](int32_t w) {
      uint32_t h = ((uint32_t)w * 2654435761u) & hmask;
      while (hkey[h] != w && hkey[h] >= 0) h = (h + 1) & hmask;
      return h;
    };
    for (int64_t v = N * kb / nblk; v < N * (kb + 1) / nblk; ++v) {
      if (dir_of[v] >= 0) {
        lc.push_back((int32_t)v);
        lv.push_back(1.0);
        rowlen[v] = 1;
        bvec[v] = d->dir_value[dir_of[v]];
        dinv[v] = 1.0;
        continue;
      }
      const uint32_t raw = (uint32_t)(ioff[v + 1] - ioff[v]) * (uint32_t)npe;
      if (2 * raw + 2 > hmask + 1) {
        uint32_t cap = hmask + 1;
        while (cap < 2 * raw + 2) cap <<= 1;
        hkey.assign(cap, -1);
        hval.resize(cap);
        hmask = cap - 1;
      }
      cl.clear();
      for (int32_t k = ioff[v]; k < ioff[v + 1]; ++k) {
        const int64_t e = inc[k] / npe;
        for (int b = 0; b < npe; ++b) {
          const int32_t w = conn[e * npe + b];
          if (dir_of[w] >= 0) continue;
          const uint32_t h = hslot(w);
          if (hkey[h] < 0) {
            hkey[h] = w;
            hused.push_back((int32_t)h);
            cl.push_back(w);
          }
        }
      }
      std::sort(cl.begin(), cl.end());
      for (size_t j = 0; j < cl.size(); ++j) hval[hslot(cl[j])] = (int32_t)j;
      if (cl.empty()) {  // a node of no element (and not Dirichlet): identity row, value 0
        lc.push_back((int32_t)v);
        lv.push_back(1.0);
        rowlen[v] = 1;
        bvec[v] = 0.0;
        dinv[v] = 1.0;
        continue;
      }
      const size_t r0 = lv.size();
      lc.insert(lc.end(), cl.begin(), cl.end());
      lv.resize(r0 + cl.size(), 0.0);
      double bv = rhs[v], diag = 0.0;
      for (int32_t k = ioff[v]; k < ioff[v + 1]; ++k) {
        const int64_t e = inc[k] / npe;
        const int a = inc[k] % npe;
        for (int b = 0; b < npe; ++b) {
          const int32_t w = conn[e * npe + b];
          const double kv = Ke[(size_t)e * m2 + a * npe + b];
          if (dir_of[w] >= 0) {
            bv -= kv * d->dir_value[dir_of[w]];
          } else {
            lv[r0 + (size_t)hval[hslot(w)]] += kv;
          }
        }
      }
      for (int32_t h : hused) hkey[h] = -1;
      hused.clear();
      for (size_t j = 0; j < cl.size(); ++j)
        if (cl[j] == v) diag = lv[r0 + j];
      rowlen[v] = (int32_t)cl.size();
      bvec[v] = bv;
      dinv[v] = diag != 0.0 ? 1.0 / diag : 1.0;
    }
  };
  {
    std::vector<std::thread> th;
    for (int64_t kb = 0; kb < nblk; ++kb) th.emplace_back(rows, kb);
    for (auto& x : th) x.join();
  }
  int64_t nnz = 0;
  for (int64_t v = 0; v < N; ++v) {
    nnz += rowlen[v];
    if (nnz >= INT32_MAX) return fail(FM_ERR_INVALID, "matrix too large for 32-bit row offsets");
    rowp[v + 1] = (int32_t)nnz;
  }
  fm::hvec<int32_t> col(nnz);
  fm::hvec<double> val(nnz);
  {
    std::vector<std::thread> th;
    for (int64_t kb = 0; kb < nblk; ++kb)
      th.emplace_back([&, kb] {
        const int64_t r0 = rowp[N * kb / nblk];
        std::copy(bcol[kb].begin(), bcol[kb].end(), col.begin() + r0);
        std::copy(bval[kb].begin(), bval[kb].end(), val.begin() + r0);
        std::vector<int32_t>().swap(bcol[kb]);
        std::vector<double>().swap(bval[kb]);
      });
    for (auto& x : th) x.join();
  }
  // no Dirichlet row: K is singular (constants), so the right-hand side is
  // projected onto its range (zero sum) to make the system consistent
  if (d->n_dirichlet == 0) {
    double s = 0.0;
    for (int64_t v = 0; v < N; ++v) s += bvec[v];
    const double m = s / (double)N;
    for (int64_t v = 0; v < N; ++v) bvec[v] -= m;
  }
  // x0 holds the Dirichlet values, the right-hand side uploaded is the
  // residual at x0 (Dirichlet rows 0); the stopping test is relative to the
  // whole right-hand side b (Dirichlet values included)
  std::vector<double> xinit(N, 0.0);
  double bb = 0.0;
  for (int64_t v = 0; v < N; ++v) bb += bvec[v] * bvec[v];
  for (int64_t v = 0; v < N; ++v)
    if (dir_of[v] >= 0) {
      xinit[v] = bvec[v];
      bvec[v] = 0.0;
    }

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FM_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(FM_ERR_INVALID, "bad device ordinal");
  DeviceRestore restore;
  PCK(cudaSetDevice(device));
  fm_poisson* s = new fm_poisson();
  s->device = device;
  s->npe = npe;
  s->problem = d->problem;
  s->N = N;
  s->E = E;
  s->nnz = nnz;
  s->bb = bb;
  // the exporter's fields (femModel.cpp:1400-1500): Dirichlet nodes 1,
  // Neumann face nodes their row's value, source elements their value (a
  // later row wins in each)
  s->h_coords.assign(d->coords, d->coords + N * 3);
  s->h_conn.assign(cfix.begin(), cfix.end());
  s->h_diff.assign(d->diffusivity, d->diffusivity + E * 3);
  s->h_src.assign(E, 0.0);
  for (int64_t k = 0; k < d->n_sources; ++k) s->h_src[d->source_elem[k]] = d->source_value[k];
  s->h_neu.assign(N, 0.0);
  for (int64_t k = 0; k < d->n_neumann; ++k)
    for (int32_t j = d->neumann_off[k]; j < d->neumann_off[k + 1]; ++j) s->h_neu[d->neumann_nodes[j]] = d->neumann_value[k];
  s->h_dir.assign(N, 0.0);
  for (int64_t k = 0; k < d->n_dirichlet; ++k) s->h_dir[d->dir_node[k]] = 1.0;
  s->view = fm::PoissonHostView{N, E, npe, d->problem, s->h_coords.data(), s->h_conn.data(), s->h_diff.data(),
                                s->h_src.data(), s->h_neu.data(), s->h_dir.data()};
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  s->blocks = (int)std::max<int64_t>(1, std::min<int64_t>((N + kThreads - 1) / kThreads, (int64_t)sms * 8));
  s->eblocks = (int)std::max<int64_t>(1, std::min<int64_t>((E + kThreads - 1) / kThreads, (int64_t)sms * 8));
  // one device allocation carved into the arrays (256-byte aligned)
  size_t total = 0;
  auto take = [&](size_t bytes) {
    const size_t off = (total + 255) & ~(size_t)255;
    total = off + std::max<size_t>(bytes, 16);
    return off;
  };
  const size_t o_rowp = take((N + 1) * 4), o_col = take(nnz * 4), o_val = take(nnz * 8), o_dinv = take(N * 8),
               o_b = take(N * 8), o_xi = take(N * 8), o_x = take(N * 8), o_r = take(N * 8), o_z = take(N * 8), o_p = take(N * 8),
               o_q = take(N * 8), o_part = take((size_t)2 * s->blocks * 8), o_scal = take(8 * 8), o_ctl = take(8 * 4),
               o_out = take(N * 8), o_coords = take(N * 3 * 8), o_conn = take(E * npe * 4),
               o_dist = take(d->problem == FM_POISSON_DISTANCE ? E * 8 : 16);
  if (cudaMalloc(&s->block, total) != cudaSuccess) {
    cudaGetLastError();
    fm_poisson_destroy(s);
    return fail(FM_ERR_OOM, "device allocation of the Poisson system failed");
  }
  char* base = static_cast<char*>(s->block);
  Cg& c = s->c;
  c.rowp = reinterpret_cast<int32_t*>(base + o_rowp);
  c.col = reinterpret_cast<int32_t*>(base + o_col);
  c.val = reinterpret_cast<double*>(base + o_val);
  c.dinv = reinterpret_cast<double*>(base + o_dinv);
  c.b = reinterpret_cast<double*>(base + o_b);
  c.xinit = reinterpret_cast<double*>(base + o_xi);
  c.x = reinterpret_cast<double*>(base + o_x);
  c.r = reinterpret_cast<double*>(base + o_r);
  c.z = reinterpret_cast<double*>(base + o_z);
  c.p = reinterpret_cast<double*>(base + o_p);
  c.q = reinterpret_cast<double*>(base + o_q);
  c.part = reinterpret_cast<double*>(base + o_part);
  c.scal = reinterpret_cast<double*>(base + o_scal);
  c.ctl = reinterpret_cast<int32_t*>(base + o_ctl);
  c.n = N;
  s->out = reinterpret_cast<double*>(base + o_out);
  s->coords = reinterpret_cast<double*>(base + o_coords);
  s->conn = reinterpret_cast<int32_t*>(base + o_conn);
  s->dist = reinterpret_cast<double*>(base + o_dist);
  auto fail_free = [&](const char* what, cudaError_t e) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    fm_poisson_destroy(s);
    return fail(FM_ERR_CUDA, m);
  };
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_ctl, 8 * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_scal, 8 * sizeof(double));
  if (e != cudaSuccess) return fail_free("stream / event / pinned buffer", e);
  const cudaStream_t st = s->stream;
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
  };
  if (e == cudaSuccess) e = up((void*)c.rowp, rowp.data(), (N + 1) * 4);
  if (e == cudaSuccess) e = up((void*)c.col, col.data(), nnz * 4);
  if (e == cudaSuccess) e = up((void*)c.val, val.data(), nnz * 8);
  if (e == cudaSuccess) e = up((void*)c.dinv, dinv.data(), N * 8);
  if (e == cudaSuccess) e = up((void*)c.b, bvec.data(), N * 8);
  if (e == cudaSuccess) e = up((void*)c.xinit, xinit.data(), N * 8);
  if (e == cudaSuccess) e = up(s->coords, d->coords, N * 3 * 8);
  if (e == cudaSuccess) e = up(s->conn, conn, E * npe * 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(c.ctl, 0, 8 * sizeof(int32_t), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host vectors go out of scope
  if (e != cudaSuccess) return fail_free("upload of the Poisson system", e);
  *out = s;
  return FM_OK;
}

FM_API int fm_poisson_create(const fm_poisson_desc* d, int32_t device, fm_poisson** out) {
  fm::NvtxRange nv("fm_poisson_create");
  try {
    return poisson_create(d, device, out);
  } catch (const std::bad_alloc&) {
    return fail(FM_ERR_OOM, "host allocation failed while assembling the Poisson system");
  }
}

FM_API int fm_poisson_info(const fm_poisson* s, int64_t* rows, int64_t* nonzeros) {
  if (!s) return fail(FM_ERR_INVALID, "null solver");
  if (rows) *rows = s->N;
  if (nonzeros) *nonzeros = s->nnz;
  return FM_OK;
}

FM_API int fm_poisson_model(const fm_poisson* s, int64_t* n_nodes, int64_t* n_elems, int32_t* elem_type,
                            int32_t* problem) {
  if (!s) return fail(FM_ERR_INVALID, "null solver");
  if (n_nodes) *n_nodes = s->N;
  if (n_elems) *n_elems = s->E;
  if (elem_type) *elem_type = s->npe;
  if (problem) *problem = s->problem;
  return FM_OK;
}

FM_API int fm_poisson_solve(fm_poisson* s, double rel_tol, int32_t max_iter, int32_t* iterations,
                            double* rel_residual, double* device_ms) {
  fm::NvtxRange nv("fm_poisson_solve");
  if (!s) return fail(FM_ERR_INVALID, "null solver");
  if (!(rel_tol >= 0.0) || max_iter < 0) return fail(FM_ERR_INVALID, "bad tolerance or iteration limit");
  DeviceRestore restore;
  PCK(cudaSetDevice(s->device));
  const cudaStream_t st = s->stream;
  const Cg& c = s->c;
  const int G = s->blocks;
  // stopping test r.r <= tol^2 b.b (scal[5] = b.b, scal[6] = the threshold)
  const int32_t ctl_init[8] = {0, 0, 0, max_iter, 0, 0, 0, 0};
  const double sc[2] = {s->bb, rel_tol * rel_tol * s->bb};
  PCK(cudaMemcpyAsync(c.ctl, ctl_init, sizeof(ctl_init), cudaMemcpyHostToDevice, st));
  PCK(cudaMemcpyAsync(c.scal + 5, sc, sizeof(sc), cudaMemcpyHostToDevice, st));
  PCK(cudaEventRecord(s->ev0, st));
  cg_init_kernel<<<G, kThreads, 0, st>>>(c);
  PCK(cudaGetLastError());
  if (!s->graph) {
    cudaGraph_t g = nullptr;
    PCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < FM_CG_GRAPH; ++i) {
      cg_spmv_kernel<<<G, kThreads, 0, st>>>(c);
      cg_update_kernel<<<G, kThreads, 0, st>>>(c);
      cg_direction_kernel<<<G, kThreads, 0, st>>>(c);
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (ce != cudaSuccess) return fail(FM_ERR_CUDA, std::string("CG graph capture: ") + cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      s->graph = nullptr;
      return fail(FM_ERR_CUDA, std::string("CG graph instantiate: ") + cudaGetErrorString(ie));
    }
  }
  // replay blocks of iterations until the device raises its done flag
  for (int64_t launched = 0;; launched += FM_CG_GRAPH) {
    PCK(cudaMemcpyAsync(s->h_ctl, c.ctl, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    PCK(cudaStreamSynchronize(st));
    if (s->h_ctl[0] || launched > (int64_t)max_iter + FM_CG_GRAPH) break;
    PCK(cudaGraphLaunch(s->graph, st));
  }
  PCK(cudaEventRecord(s->ev1, st));
  avg_kernel<<<G, kThreads, 0, st>>>(c);
  shift_kernel<<<G, kThreads, 0, st>>>(c.x, c.scal, s->problem == FM_POISSON_PPE, s->N, s->out);
  if (s->problem == FM_POISSON_DISTANCE)
    distance_kernel<<<s->eblocks, kThreads, 0, st>>>(s->coords, s->conn, s->npe, s->E, s->out, s->dist);
  PCK(cudaGetLastError());
  PCK(cudaMemcpyAsync(s->h_ctl, c.ctl, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  PCK(cudaMemcpyAsync(s->h_scal, c.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  PCK(cudaStreamSynchronize(st));
  float ms = 0.0f;
  PCK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
  if (device_ms) *device_ms = ms;
  if (iterations) *iterations = s->h_ctl[1];
  const double bb = s->bb;
  if (rel_residual) *rel_residual = bb > 0.0 ? std::sqrt(s->h_scal[4] / bb) : 0.0;
  s->has_result = true;
  if (s->h_ctl[2]) return fail(FM_ERR_DIVERGED, "CG breakdown (matrix not positive definite on the search direction, or NaN)");
  return FM_OK;
}

FM_API int fm_poisson_get_solution(fm_poisson* s, double* x, double* cell_distance) {
  if (!s) return fail(FM_ERR_INVALID, "null solver");
  if (!s->has_result) return fail(FM_ERR_INVALID, "fm_poisson_solve has not run");
  if (cell_distance && s->problem != FM_POISSON_DISTANCE)
    return fail(FM_ERR_INVALID, "cell distances exist for FM_POISSON_DISTANCE only");
  DeviceRestore restore;
  PCK(cudaSetDevice(s->device));
  if (x) PCK(cudaMemcpyAsync(x, s->out, s->N * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  if (cell_distance) PCK(cudaMemcpyAsync(cell_distance, s->dist, s->E * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  PCK(cudaStreamSynchronize(s->stream));
  return FM_OK;
}

}  // extern "C"

namespace fm {
const PoissonHostView* poisson_host_view(const fm_poisson* s) { return s ? &s->view : nullptr; }
}  // namespace fm
