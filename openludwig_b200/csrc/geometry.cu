// Domain preprocessing on the device: cell voxelisation of the body
// (domain_generation.jl:10-32, :74-112) and the Bouzidi wall distances q
// (bouzidi_setup.jl:64-166, bouzidi_math.jl:9-101).  Both are FP64 and give
// the same bits as the host build (openludwig_b200/domain.py): every product,
// sum and difference is rounded on its own (__dmul_rn / __dadd_rn /
// __dsub_rn, never fused), in the host's operation order; division and
// square root are IEEE.  One CTA per 8^3 block, one thread per cell; the
// triangles a block can touch come as a CSR list (ascending triangle ids,
// built on the host from the triangles' bounding boxes), staged through
// shared memory in chunks.
#include <cuda_fp16.h>
#include <math_constants.h>

#include "common.cuh"

namespace ol {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
// (a0*b0 + a1*b1) + a2*b2
__device__ __forceinline__ double dot3(double a0, double a1, double a2, double b0, double b1,
                                       double b2) {
  return add(add(mul(a0, b0), mul(a1, b1)), mul(a2, b2));
}

struct GeoArgs {
  const int32_t *coords;  // [n_blocks][3] 1-based block coordinates (x, y, z)
  int32_t n_blocks;
  const double *tris;     // [n_tris][3 vertices][3]
  const int32_t *tri_off; // [n_blocks + 1] CSR offsets into tri_list
  const int32_t *tri_list;
  double dx, off[3];
};

// Cell centre ((b - 1) * 8 + l - 1/2) * dx, l = 1..8 (domain.py _cell_centers).
__device__ __forceinline__ void cell_centre(const GeoArgs &g, int b, int t, double c[3]) {
  const int l[3] = {(t & 7) + 1, ((t >> 3) & 7) + 1, (t >> 6) + 1};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int64_t gi = ((int64_t)g.coords[3 * b + a] - 1) * 8 + l[a];
    c[a] = mul(sub((double)gi, 0.5), g.dx);
  }
}

constexpr int kGeoThreads = 512;
constexpr int kVoxChunk = 256;  // triangles staged per round (9 doubles each)

// ---------------------------------------------------------------------------
// Voxelisation: a cell is solid when some triangle overlaps its box of half
// size 0.75 dx * 1.001 (separating-axis test, domain_generation.jl:10-32).
// ---------------------------------------------------------------------------
__device__ bool tri_box_overlap(const double t1[3], const double t2[3], const double t3[3],
                                double h) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double mn = fmin(fmin(t1[a], t2[a]), t3[a]);
    const double mx = fmax(fmax(t1[a], t2[a]), t3[a]);
    if (mn > h || mx < -h) return false;
  }
  double f[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    f[0][a] = sub(t2[a], t1[a]);
    f[1][a] = sub(t3[a], t2[a]);
    f[2][a] = sub(t1[a], t3[a]);
  }
#pragma unroll
  for (int ui = 0; ui < 3; ++ui) {
    const double u0 = ui == 0 ? 1.0 : 0.0, u1 = ui == 1 ? 1.0 : 0.0, u2 = ui == 2 ? 1.0 : 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double ax = sub(mul(u1, f[j][2]), mul(u2, f[j][1]));
      const double ay = sub(mul(u2, f[j][0]), mul(u0, f[j][2]));
      const double az = sub(mul(u0, f[j][1]), mul(u1, f[j][0]));
      if (add(add(mul(ax, ax), mul(ay, ay)), mul(az, az)) < 1e-10) continue;
      const double p1 = dot3(t1[0], t1[1], t1[2], ax, ay, az);
      const double p2 = dot3(t2[0], t2[1], t2[2], ax, ay, az);
      const double p3 = dot3(t3[0], t3[1], t3[2], ax, ay, az);
      const double r = add(add(mul(h, fabs(ax)), mul(h, fabs(ay))), mul(h, fabs(az)));
      if (fmin(p1, fmin(p2, p3)) > r || fmax(p1, fmax(p2, p3)) < -r) return false;
    }
  }
  return true;
}

__global__ void __launch_bounds__(kGeoThreads) k_voxelize(const GeoArgs g, uint8_t *obst) {
  __shared__ double sv[kVoxChunk][9];
  const int b = blockIdx.x, t = threadIdx.x;
  const int t0 = g.tri_off[b], t1e = g.tri_off[b + 1];
  if (t0 >= t1e) return;
  double c[3];
  cell_centre(g, b, t, c);
  const double h = mul(mul(0.75, g.dx), 1.001);
  bool hit = false;
  for (int base = t0; base < t1e; base += kVoxChunk) {
    const int m = min(kVoxChunk, t1e - base);
    __syncthreads();
    for (int i = t; i < m * 9; i += kGeoThreads) {
      const int tri = g.tri_list[base + i / 9], e = i % 9;
      sv[i / 9][e] = add(g.tris[9 * (int64_t)tri + e], g.off[e % 3]);
    }
    __syncthreads();
    for (int j = 0; j < m && !hit; ++j) {
      double p1[3], p2[3], p3[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        p1[a] = sub(sv[j][a], c[a]);
        p2[a] = sub(sv[j][3 + a], c[a]);
        p3[a] = sub(sv[j][6 + a], c[a]);
      }
      hit = tri_box_overlap(p1, p2, p3, h);
    }
  }
  obst[(int64_t)b * 512 + t] = hit ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Bouzidi q: for every cell and link k != rest, the nearest Moller-Trumbore
// hit (eps 1e-9) along the unit link direction d_k among the block's
// triangles (the first one in triangle order on ties); q = t / (dx |c_k|),
// kept when 0 < q <= 1, stored as binary16 (round to nearest even) with the
// 1-based triangle id.  The links are done in two passes of 13 so that the
// running minima of a pass stay in registers.
// ---------------------------------------------------------------------------
constexpr int kQChunk = 16;  // triangles staged per round
constexpr double kEps = 1e-9;

__device__ __forceinline__ int link_k(int pass, int i) {  // i = 0..12 -> k != 13
  const int k = pass * 13 + i;
  return k < 13 ? k : k + 1;
}

template <int PASS>
__device__ void qmap_pass(const GeoArgs &g, int b, int t, const double c[3], int64_t S,
                          uint16_t *q16, int32_t *trim, bool &has,
                          double (*tv)[9], double (*th)[13][4], bool (*tvalid)[13]) {
  double best[13];
  int bj[13];
#pragma unroll
  for (int i = 0; i < 13; ++i) { best[i] = CUDART_INF; bj[i] = -1; }
  const int t0 = g.tri_off[b], t1e = g.tri_off[b + 1];
  for (int base = t0; base < t1e; base += kQChunk) {
    const int m = min(kQChunk, t1e - base);
    __syncthreads();
    // triangle vertices (offset added), edges e1 = v2 - v1, e2 = v3 - v1
    if (t < m) {
      const int64_t tri = g.tri_list[base + t];
      double v[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) v[e] = add(g.tris[9 * tri + e], g.off[e % 3]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        tv[t][a] = v[a];
        tv[t][3 + a] = sub(v[3 + a], v[a]);
        tv[t][6 + a] = sub(v[6 + a], v[a]);
      }
    }
    __syncthreads();
    // per (triangle, link): h = d x e2, a = e1 . h, f = 1 / a
    if (t < m * 13) {
      const int j = t / 13, i = t % 13, k = link_k(PASS, i);
      const int cx = k % 3 - 1, cy = (k / 3) % 3 - 1, cz = k / 9 - 1;
      const double nrm = sqrt((double)(cx * cx) + (double)(cy * cy) + (double)(cz * cz));
      const double d0 = (double)cx / nrm, d1 = (double)cy / nrm, d2 = (double)cz / nrm;
      const double *e1 = tv[j] + 3, *e2 = tv[j] + 6;
      const double hx = sub(mul(d1, e2[2]), mul(d2, e2[1]));
      const double hy = sub(mul(d2, e2[0]), mul(d0, e2[2]));
      const double hz = sub(mul(d0, e2[1]), mul(d1, e2[0]));
      const double a = dot3(e1[0], e1[1], e1[2], hx, hy, hz);
      th[j][i][0] = hx; th[j][i][1] = hy; th[j][i][2] = hz;
      th[j][i][3] = 1.0 / a;
      tvalid[j][i] = !(fabs(a) < kEps);
    }
    __syncthreads();
    for (int j = 0; j < m; ++j) {
      const double s0 = sub(c[0], tv[j][0]), s1 = sub(c[1], tv[j][1]), s2 = sub(c[2], tv[j][2]);
      const double *e1 = tv[j] + 3, *e2 = tv[j] + 6;
      const double q0 = sub(mul(s1, e1[2]), mul(s2, e1[1]));
      const double q1 = sub(mul(s2, e1[0]), mul(s0, e1[2]));
      const double q2 = sub(mul(s0, e1[1]), mul(s1, e1[0]));
      const double tq = dot3(e2[0], e2[1], e2[2], q0, q1, q2);
#pragma unroll
      for (int i = 0; i < 13; ++i) {
        const int k = link_k(PASS, i);
        const int cx = k % 3 - 1, cy = (k / 3) % 3 - 1, cz = k / 9 - 1;
        const double nrm = sqrt((double)(cx * cx) + (double)(cy * cy) + (double)(cz * cz));
        const double d0 = (double)cx / nrm, d1 = (double)cy / nrm, d2 = (double)cz / nrm;
        const double f = th[j][i][3];
        const double u = mul(f, dot3(s0, s1, s2, th[j][i][0], th[j][i][1], th[j][i][2]));
        const double v = mul(f, dot3(d0, d1, d2, q0, q1, q2));
        const double tt = mul(f, tq);
        const bool hit = tvalid[j][i] && !(u < 0.0 || u > 1.0) && !(v < 0.0 || add(u, v) > 1.0) &&
                         tt > kEps;
        if (hit && tt < best[i]) { best[i] = tt; bj[i] = base + j; }
      }
    }
  }
  const int64_t cell = (int64_t)b * 512 + t;
#pragma unroll
  for (int i = 0; i < 13; ++i) {
    if (bj[i] < 0) continue;
    const int k = link_k(PASS, i);
    const int cx = k % 3 - 1, cy = (k / 3) % 3 - 1, cz = k / 9 - 1;
    const double nrm = sqrt((double)(cx * cx) + (double)(cy * cy) + (double)(cz * cz));
    const double q = best[i] / mul(g.dx, nrm);
    if (q > 0.0 && q <= 1.0) {
      q16[cell + k * S] = __half_as_ushort(__double2half(q));
      trim[cell + k * S] = g.tri_list[bj[i]] + 1;
      has = true;
    }
  }
}

__global__ void __launch_bounds__(kGeoThreads) k_bouzidi_qmap(const GeoArgs g, uint16_t *q16,
                                                               int32_t *trim, uint8_t *has_link) {
  __shared__ double tv[kQChunk][9];
  __shared__ double th[kQChunk][13][4];
  __shared__ bool tvalid[kQChunk][13];
  const int b = blockIdx.x, t = threadIdx.x;
  if (g.tri_off[b] >= g.tri_off[b + 1]) return;
  double c[3];
  cell_centre(g, b, t, c);
  const int64_t S = (int64_t)g.n_blocks * 512;
  bool has = false;
  qmap_pass<0>(g, b, t, c, S, q16, trim, has, tv, th, tvalid);
  qmap_pass<1>(g, b, t, c, S, q16, trim, has, tv, th, tvalid);
  has_link[(int64_t)b * 512 + t] = has ? 1 : 0;
}

}  // namespace
}  // namespace ol

using namespace ol;

static int geo_args(GeoArgs &g, const int32_t *coords, int32_t n_blocks, const double *tris,
                    int32_t n_tris, const int32_t *tri_off, const int32_t *tri_list, double dx,
                    const double *offset, const char *who) {
  OL_CHECK_ARG(n_blocks >= 0 && n_tris >= 0, "%s: negative size", who);
  OL_CHECK_ARG(n_blocks == 0 || (coords && tri_off), "%s: null block arrays", who);
  OL_CHECK_ARG(n_tris == 0 || tris, "%s: null triangles", who);
  OL_CHECK_ARG(offset && dx > 0.0, "%s: bad dx or offset", who);
  OL_CHECK_ARG((int64_t)n_blocks * 512 * 27 < (1LL << 62), "%s: level too large", who);
  g.coords = coords; g.n_blocks = n_blocks; g.tris = tris; g.tri_off = tri_off;
  g.tri_list = tri_list; g.dx = dx;
  g.off[0] = offset[0]; g.off[1] = offset[1]; g.off[2] = offset[2];
  return OL_OK;
}

extern "C" int ol_voxelize(const int32_t *coords, int32_t n_blocks, const double *tris,
                           int32_t n_tris, const int32_t *tri_off, const int32_t *tri_list,
                           double dx, const double offset[3], uint8_t *obstacle, void *stream) {
  GeoArgs g;
  int rc = geo_args(g, coords, n_blocks, tris, n_tris, tri_off, tri_list, dx, offset,
                    "ol_voxelize");
  if (rc) return rc;
  if (n_blocks == 0) return OL_OK;
  OL_CHECK_ARG(obstacle, "ol_voxelize: null output");
  const cudaStream_t s = (cudaStream_t)stream;
  OL_CUDA(cudaMemsetAsync(obstacle, 0, (size_t)n_blocks * 512, s));
  k_voxelize<<<n_blocks, kGeoThreads, 0, s>>>(g, obstacle);
  OL_LAUNCHED("ol_voxelize");
  return OL_OK;
}

extern "C" int ol_bouzidi_qmap(const int32_t *coords, int32_t n_blocks, const double *tris,
                               int32_t n_tris, const int32_t *tri_off, const int32_t *tri_list,
                               double dx, const double offset[3], uint16_t *q_map,
                               int32_t *tri_map, uint8_t *has_link, void *stream) {
  GeoArgs g;
  int rc = geo_args(g, coords, n_blocks, tris, n_tris, tri_off, tri_list, dx, offset,
                    "ol_bouzidi_qmap");
  if (rc) return rc;
  if (n_blocks == 0) return OL_OK;
  OL_CHECK_ARG(q_map && tri_map && has_link, "ol_bouzidi_qmap: null output");
  const cudaStream_t s = (cudaStream_t)stream;
  const size_t S = (size_t)n_blocks * 512;
  OL_CUDA(cudaMemsetAsync(q_map, 0, S * 27 * sizeof(uint16_t), s));
  OL_CUDA(cudaMemsetAsync(tri_map, 0, S * 27 * sizeof(int32_t), s));
  OL_CUDA(cudaMemsetAsync(has_link, 0, S, s));
  k_bouzidi_qmap<<<n_blocks, kGeoThreads, 0, s>>>(g, q_map, tri_map, has_link);
  OL_LAUNCHED("ol_bouzidi_qmap");
  return OL_OK;
}
