// FE load mapping (PREPOST/map_forces_to_nodes.jl): net triangle forces to
// the nearest structural nodes with force and moment equilibrium.
//
// The reference is a serial host script: for every triangle a brute-force
// search of its object's nodes, a 6 x 3k pseudo-inverse (LAPACK SVD) and a
// running sum per node.  Here every triangle is one GPU thread:
//   k_fe_distribute  nearest k <= 3 nodes of the object (squared FP64
//                    distances, ties to the earlier node, as a stable
//                    partial sort), then f = pinv(A) b by a one-sided Jacobi
//                    SVD of A^T (9 x 6, zero rows when k = 2), singular values
//                    <= 6 eps sigma_max dropped (LinearAlgebra.pinv's default
//                    for a 6 x 3k matrix);
//   k_fe_accumulate  each contribution added to its node in fixed point,
//                    scaled to the node's largest contribution (2^40 units of
//                    it), with 64-bit integer atomics: exact, so the sum does
//                    not depend on the order the threads arrive in;
//   k_fe_finish      back to FP64.
// Node coordinates are read by all threads of a warp at the same index
// (triangles of one object are contiguous), i.e. broadcast loads.
#include <cfloat>
#include <climits>
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace ol {
namespace {

constexpr int kFeThreads = 128;
constexpr int kFeFracBits = 40;           // fixed-point bits below a node's top exponent
constexpr int kFeMaxContrib = 1 << 21;    // per node: 2^(40 + 1 + 21) < 2^63
constexpr int kFeNoExp = INT_MIN;
constexpr int kFeMaxSweeps = 40;

struct FeScratch {
  int32_t *exp;                 // [n] largest ilogb of a contribution component
  int32_t *cnt;                 // [n] contributions
  unsigned long long *acc;      // [3 n] fixed-point sums
  int32_t *flags;               // [2] unconverged triangles, overflow
};

__host__ __device__ inline size_t fe_align(size_t x) { return (x + 255) & ~(size_t)255; }

FeScratch fe_scratch(void *base, int n) {
  char *p = (char *)base;
  FeScratch s;
  s.exp = (int32_t *)p;
  p += fe_align(sizeof(int32_t) * (size_t)n);
  s.cnt = (int32_t *)p;
  p += fe_align(sizeof(int32_t) * (size_t)n);
  s.acc = (unsigned long long *)p;
  p += fe_align(sizeof(unsigned long long) * 3 * (size_t)n);
  s.flags = (int32_t *)p;
  return s;
}

size_t fe_scratch_bytes(int n) {
  return fe_align(sizeof(int32_t) * (size_t)n) * 2 +
         fe_align(sizeof(unsigned long long) * 3 * (size_t)n) + fe_align(2 * sizeof(int32_t));
}

__global__ void k_fe_clear(FeScratch s, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    s.exp[i] = kFeNoExp;
    s.cnt[i] = 0;
    s.acc[i] = 0ull;
    s.acc[i + n] = 0ull;
    s.acc[i + 2 * n] = 0ull;
  }
  if (i < 2) s.flags[i] = 0;
}

// Object of triangle t: the last o with tri_begin[o] <= t.
__device__ int fe_object_of(const int32_t *begin, int n_obj, int t) {
  int lo = 0, hi = n_obj;  // begin[lo] <= t < begin[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(begin + mid) <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// f = pinv(A) b for the 6 x 3k equilibrium matrix A (k = 2 or 3) of node
// offsets r[i] = p_i - c and b = (F, 0, 0, 0).  B = A^T is 9 x 6 (rows 3k..8
// zero when k = 2).  One-sided Jacobi: rotate column pairs of B (and of V)
// until all are orthogonal, B V = U S; then A = V S U^T and
// pinv(A) b = sum_j B_j (v_j . b) / s_j^2 over s_j > 6 eps s_max.
// Returns false when the sweep limit was reached.
__device__ bool fe_distribute(int k, const double (&r)[3][3], const double (&F)[3],
                              double (&out)[3][3]) {
  double B[9][6], V[6][6];
#pragma unroll
  for (int i = 0; i < 9; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) B[i][j] = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) V[i][j] = i == j ? 1.0 : 0.0;
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    if (n >= k) break;
    const double rx = r[n][0], ry = r[n][1], rz = r[n][2];
    // force rows: A[a][3n + a] = 1; moment rows: A[3 + a][3n + b] = skew(r)[a][b]
    // skew(r) = [0 -rz ry; rz 0 -rx; -ry rx 0]
#pragma unroll
    for (int a = 0; a < 3; ++a) B[3 * n + a][a] = 1.0;
    B[3 * n + 0][3] = 0.0;  B[3 * n + 1][3] = -rz;  B[3 * n + 2][3] = ry;
    B[3 * n + 0][4] = rz;   B[3 * n + 1][4] = 0.0;  B[3 * n + 2][4] = -rx;
    B[3 * n + 0][5] = -ry;  B[3 * n + 1][5] = rx;   B[3 * n + 2][5] = 0.0;
  }
  bool converged = false;
  for (int sweep = 0; sweep < kFeMaxSweeps && !converged; ++sweep) {
    converged = true;
#pragma unroll
    for (int p = 0; p < 5; ++p)
#pragma unroll
      for (int q = p + 1; q < 6; ++q) {
        double alpha = 0.0, beta = 0.0, gamma = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          alpha += B[i][p] * B[i][p];
          beta += B[i][q] * B[i][q];
          gamma += B[i][p] * B[i][q];
        }
        if (gamma == 0.0 || fabs(gamma) <= 1e-15 * sqrt(alpha * beta)) continue;
        converged = false;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = fabs(zeta) > 1e150 ? 0.5 / zeta
                                            : copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          const double bp = B[i][p], bq = B[i][q];
          B[i][p] = c * bp - s * bq;
          B[i][q] = s * bp + c * bq;
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          const double vp = V[i][p], vq = V[i][q];
          V[i][p] = c * vp - s * vq;
          V[i][q] = s * vp + c * vq;
        }
      }
  }
  double s2[6], smax = 0.0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double a = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) a += B[i][j] * B[i][j];
    s2[j] = a;
    smax = fmax(smax, sqrt(a));
  }
  const double tol = 6.0 * DBL_EPSILON * smax;
  double f[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) f[i] = 0.0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    if (!(sqrt(s2[j]) > tol)) continue;
    const double vb = V[0][j] * F[0] + V[1][j] * F[1] + V[2][j] * F[2];   // b = (F, 0, 0, 0)
    const double w = vb / s2[j];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] += B[i][j] * w;
  }
#pragma unroll
  for (int n = 0; n < 3; ++n)
#pragma unroll
    for (int a = 0; a < 3; ++a) out[n][a] = f[3 * n + a];
  return converged;
}

__global__ void __launch_bounds__(kFeThreads) k_fe_distribute(const ol_fe_map_view v, FeScratch s) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= v.n_tris) return;
  const int T = v.n_tris, N = v.n_nodes;
  const int o = fe_object_of(v.tri_begin, v.n_objects, t);
  const int n0 = __ldg(v.node_begin + o), n1 = __ldg(v.node_begin + o + 1);
  const int k = min(3, n1 - n0);
  const double c[3] = {v.tri_xyz[t], v.tri_xyz[t + T], v.tri_xyz[t + 2 * T]};
  const double F[3] = {v.tri_force[t], v.tri_force[t + T], v.tri_force[t + 2 * T]};
  // k nearest: insertion into a sorted list of k, strict comparison (the
  // earlier node stays first on a tie)
  double bd[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  int bi[3] = {-1, -1, -1};
  for (int i = n0; i < n1; ++i) {
    const double dx = __dsub_rn(__ldg(v.node_xyz + i), c[0]);
    const double dy = __dsub_rn(__ldg(v.node_xyz + i + N), c[1]);
    const double dz = __dsub_rn(__ldg(v.node_xyz + i + 2 * N), c[2]);
    const double d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    if (k > 0 && (bi[k - 1] < 0 || d < bd[k - 1])) {
      int p = k - 1;
      while (p > 0 && (bi[p - 1] < 0 || d < bd[p - 1])) {
        bd[p] = bd[p - 1];
        bi[p] = bi[p - 1];
        --p;
      }
      bd[p] = d;
      bi[p] = i;
    }
  }
  double out[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  if (k == 1) {
    out[0][0] = F[0]; out[0][1] = F[1]; out[0][2] = F[2];
  } else if (k > 1) {
    double r[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int n = 0; n < k; ++n) {
      const int i = bi[n];
      r[n][0] = __ldg(v.node_xyz + i) - c[0];
      r[n][1] = __ldg(v.node_xyz + i + N) - c[1];
      r[n][2] = __ldg(v.node_xyz + i + 2 * N) - c[2];
    }
    if (!fe_distribute(k, r, F, out)) atomicAdd(s.flags, 1);
  }
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const int i = n < k ? bi[n] : -1;
    v.tri_nodes[n * T + t] = i;
#pragma unroll
    for (int a = 0; a < 3; ++a) v.tri_node_force[(3 * n + a) * T + t] = out[n][a];
    if (i >= 0) {
      atomicAdd(s.cnt + i, 1);
      const double m = fmax(fabs(out[n][0]), fmax(fabs(out[n][1]), fabs(out[n][2])));
      if (m > 0.0) atomicMax(s.exp + i, ilogb(m));
    }
  }
}

__global__ void __launch_bounds__(kFeThreads) k_fe_accumulate(const ol_fe_map_view v, FeScratch s) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= v.n_tris) return;
  const int T = v.n_tris, N = v.n_nodes;
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const int i = v.tri_nodes[n * T + t];
    if (i < 0) continue;
    const int e = s.exp[i];
    if (e == kFeNoExp) continue;   // every contribution to this node is zero
    if (s.cnt[i] > kFeMaxContrib) {
      atomicOr(s.flags + 1, 1);
      continue;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const long long q = __double2ll_rn(ldexp(v.tri_node_force[(3 * n + a) * T + t], kFeFracBits - e));
      atomicAdd(s.acc + a * N + i, (unsigned long long)q);
    }
  }
}

__global__ void k_fe_finish(const ol_fe_map_view v, FeScratch s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_nodes) return;
  const int N = v.n_nodes, e = s.exp[i];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    v.nodal_force[a * N + i] =
        e == kFeNoExp ? 0.0 : ldexp((double)(long long)s.acc[a * N + i], e - kFeFracBits);
}

}  // namespace
}  // namespace ol

using namespace ol;

extern "C" size_t ol_fe_map_scratch_bytes(int32_t n_nodes) {
  return n_nodes < 0 ? 0 : fe_scratch_bytes(n_nodes);
}

extern "C" int ol_fe_map_forces(const ol_fe_map_view *v, int32_t *n_unconverged, void *stream) {
  if (!v || !n_unconverged) return set_error(OL_ERR_ARG, "ol_fe_map_forces: null argument");
  if (v->n_nodes < 0 || v->n_tris < 0 || v->n_objects < 1)
    return set_error(OL_ERR_ARG, "ol_fe_map_forces: bad sizes (%d nodes, %d triangles, %d objects)",
                     v->n_nodes, v->n_tris, v->n_objects);
  if ((v->n_tris && (!v->tri_xyz || !v->tri_force || !v->tri_nodes || !v->tri_node_force)) ||
      (v->n_nodes && (!v->node_xyz || !v->nodal_force)) || !v->node_begin || !v->tri_begin ||
      !v->scratch)
    return set_error(OL_ERR_ARG, "ol_fe_map_forces: null array");
  cudaStream_t s = (cudaStream_t)stream;
  // the object ranges must cover exactly [0, n) in order
  std::vector<int32_t> nb(v->n_objects + 1), tb(v->n_objects + 1);
  cudaError_t e = cudaMemcpyAsync(nb.data(), v->node_begin, sizeof(int32_t) * nb.size(),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(tb.data(), v->tri_begin, sizeof(int32_t) * tb.size(),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "ol_fe_map_forces: object ranges");
  if (nb[0] != 0 || tb[0] != 0 || nb.back() != v->n_nodes || tb.back() != v->n_tris)
    return set_error(OL_ERR_ARG, "ol_fe_map_forces: object ranges do not cover the arrays");
  for (int o = 0; o < v->n_objects; ++o)
    if (nb[o + 1] < nb[o] || tb[o + 1] < tb[o])
      return set_error(OL_ERR_ARG, "ol_fe_map_forces: object ranges not ascending at %d", o);
  FeScratch sc = fe_scratch(v->scratch, v->n_nodes);
  const int g_nodes = std::max(1, (v->n_nodes + kFeThreads - 1) / kFeThreads);
  const int g_tris = (v->n_tris + kFeThreads - 1) / kFeThreads;
  k_fe_clear<<<g_nodes, kFeThreads, 0, s>>>(sc, v->n_nodes);
  if (g_tris) {
    k_fe_distribute<<<g_tris, kFeThreads, 0, s>>>(*v, sc);
    k_fe_accumulate<<<g_tris, kFeThreads, 0, s>>>(*v, sc);
  }
  if (v->n_nodes) k_fe_finish<<<g_nodes, kFeThreads, 0, s>>>(*v, sc);
  int32_t flags[2] = {0, 0};
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(flags, sc.flags, sizeof(flags), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "ol_fe_map_forces");
  *n_unconverged = flags[0];
  if (flags[1])
    return set_error(OL_ERR_ARG, "ol_fe_map_forces: more than %d contributions to one node",
                     kFeMaxContrib);
  return OL_OK;
}
