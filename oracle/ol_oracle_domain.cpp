/*
 * ol_oracle_domain.cpp -- CPU restatement of the reference's host-side domain
 * build: level block sets, neighbour tables, SAT surface voxelization, flood
 * fill, sponge, wall distance and the Bouzidi q-map.
 *
 * TEST INFRASTRUCTURE (see ol_oracle_kernels.cpp).  FP64 geometry is written
 * in the reference's expression order and compiled without contraction, so
 * integer outputs (block sets, tables, masks, Float16 q values, triangle ids)
 * are comparable bit for bit with the product's preprocessing.  Triangles come
 * in as a flat double array [ntri][3 vertices][xyz] in the unrotated-offset
 * (mesh) frame; `off` is mesh_offset.
 */
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <set>
#include <tuple>
#include <vector>

namespace orcd {

constexpr int BS = 8;
using B3 = std::array<int, 3>;

struct V3 { double x, y, z; };
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

inline V3 vert(const double *tris, int t, int v) {
  const double *p = tris + (size_t)t * 9 + v * 3;
  return {p[0], p[1], p[2]};
}
inline long ifloor(double v) { return (long)std::floor(v); }

// domain_topology.jl:9-52
static std::set<B3> active_blocks(const double *tris, int ntri, double dx, const double *off, int bxm,
                                  int bym, int bzm) {
  std::set<B3> s;
  const double margin = dx * 0.01;
  const double inv = 1.0 / (BS * dx);
  for (int t = 0; t < ntri; ++t) {
    V3 o{off[0], off[1], off[2]};
    V3 mn = add(vert(tris, t, 0), o), mx = mn;
    for (int v = 0; v < 3; ++v) {
      V3 p = add(vert(tris, t, v), o);
      mn = {std::min(mn.x, p.x), std::min(mn.y, p.y), std::min(mn.z, p.z)};
      mx = {std::max(mx.x, p.x), std::max(mx.y, p.y), std::max(mx.z, p.z)};
    }
    long x0 = ifloor((mn.x - margin) * inv) + 1, y0 = ifloor((mn.y - margin) * inv) + 1,
         z0 = ifloor((mn.z - margin) * inv) + 1;
    long x1 = ifloor((mx.x + margin) * inv) + 1, y1 = ifloor((mx.y + margin) * inv) + 1,
         z1 = ifloor((mx.z + margin) * inv) + 1;
    x0 = std::max(1L, x0); x1 = std::min(x1, (long)bxm);
    y0 = std::max(1L, y0); y1 = std::min(y1, (long)bym);
    z0 = std::max(1L, z0); z1 = std::min(z1, (long)bzm);
    for (long bz = z0; bz <= z1; ++bz)
      for (long by = y0; by <= y1; ++by)
        for (long bx = x0; bx <= x1; ++bx) s.insert({(int)bx, (int)by, (int)bz});
  }
  return s;
}

inline bool in_dims(int x, int y, int z, int bxm, int bym, int bzm) {
  return x >= 1 && x <= bxm && y >= 1 && y <= bym && z >= 1 && z <= bzm;
}
inline int jdiv2(int v) { return (v + 1) / 2; }  // (b + 1) ÷ 2 for b >= 1

// domain_topology.jl:54-99
static void add_halo(std::set<B3> &s, int layers, int bxm, int bym, int bzm) {
  for (int l = 0; l < layers; ++l) {
    std::set<B3> nb;
    for (const B3 &b : s)
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            if (!dx && !dy && !dz) continue;
            B3 n{b[0] + dx, b[1] + dy, b[2] + dz};
            if (in_dims(n[0], n[1], n[2], bxm, bym, bzm) && !s.count(n)) nb.insert(n);
          }
    std::set<B3> sib;
    for (const B3 &b : nb) {
      int px = jdiv2(b[0]), py = jdiv2(b[1]), pz = jdiv2(b[2]);
      for (int dz = 0; dz <= 1; ++dz)
        for (int dy = 0; dy <= 1; ++dy)
          for (int dx = 0; dx <= 1; ++dx) {
            B3 c{2 * px - 1 + dx, 2 * py - 1 + dy, 2 * pz - 1 + dz};
            if (in_dims(c[0], c[1], c[2], bxm, bym, bzm) && !s.count(c) && !nb.count(c)) sib.insert(c);
          }
    }
    s.insert(nb.begin(), nb.end());
    s.insert(sib.begin(), sib.end());
  }
}

// domain_topology.jl:101-133
static void parent_coverage(std::set<B3> &s, int bxm, int bym, int bzm) {
  bool added = true;
  int it = 0;
  while (added && it < 10) {
    added = false;
    ++it;
    std::set<B3> add_s;
    for (const B3 &b : s) {
      int px = jdiv2(b[0]), py = jdiv2(b[1]), pz = jdiv2(b[2]);
      for (int dz = 0; dz <= 1; ++dz)
        for (int dy = 0; dy <= 1; ++dy)
          for (int dx = 0; dx <= 1; ++dx) {
            B3 c{2 * px - 1 + dx, 2 * py - 1 + dy, 2 * pz - 1 + dz};
            if (in_dims(c[0], c[1], c[2], bxm, bym, bzm) && !s.count(c)) {
              add_s.insert(c);
              added = true;
            }
          }
    }
    s.insert(add_s.begin(), add_s.end());
  }
}

// geometry_blocks_tris: margin m, "(min - m) / (bs*dx)" form (domain_generation.jl:34-72
// with m = 2 dx; bouzidi_setup.jl:12-54 with m = 2.5 dx)
static std::vector<std::vector<int>> block_tri_map(const double *tris, int ntri,
                                                   const std::vector<B3> &blocks, double dx,
                                                   const double *off, double margin) {
  std::vector<std::vector<int>> out(blocks.size());
  std::vector<int> lut;
  int bxm = 0, bym = 0, bzm = 0;
  for (const B3 &b : blocks) { bxm = std::max(bxm, b[0]); bym = std::max(bym, b[1]); bzm = std::max(bzm, b[2]); }
  lut.assign((size_t)bxm * bym * bzm, -1);
  for (size_t i = 0; i < blocks.size(); ++i)
    lut[(blocks[i][0] - 1) + (size_t)bxm * ((blocks[i][1] - 1) + (size_t)bym * (blocks[i][2] - 1))] = (int)i;
  const double bsd = BS * dx;
  for (int t = 0; t < ntri; ++t) {
    V3 o{off[0], off[1], off[2]};
    V3 mn = add(vert(tris, t, 0), o), mx = mn;
    for (int v = 0; v < 3; ++v) {
      V3 p = add(vert(tris, t, v), o);
      mn = {std::min(mn.x, p.x), std::min(mn.y, p.y), std::min(mn.z, p.z)};
      mx = {std::max(mx.x, p.x), std::max(mx.y, p.y), std::max(mx.z, p.z)};
    }
    long x0 = ifloor((mn.x - margin) / bsd) + 1, y0 = ifloor((mn.y - margin) / bsd) + 1,
         z0 = ifloor((mn.z - margin) / bsd) + 1;
    long x1 = ifloor((mx.x + margin) / bsd) + 1, y1 = ifloor((mx.y + margin) / bsd) + 1,
         z1 = ifloor((mx.z + margin) / bsd) + 1;
    for (long bz = std::max(1L, z0); bz <= z1; ++bz)
      for (long by = std::max(1L, y0); by <= y1; ++by)
        for (long bx = std::max(1L, x0); bx <= x1; ++bx) {
          if (bx > bxm || by > bym || bz > bzm) continue;
          int i = lut[(bx - 1) + (size_t)bxm * ((by - 1) + (size_t)bym * (bz - 1))];
          if (i >= 0) out[i].push_back(t);
        }
  }
  return out;
}

// domain_generation.jl:10-32 (no triangle-normal axis, as in the reference)
static bool tri_box(V3 c, double h0, V3 v1, V3 v2, V3 v3) {
  const double h = h0 * 1.001;
  V3 t1 = sub(v1, c), t2 = sub(v2, c), t3 = sub(v3, c);
  if (std::min({t1.x, t2.x, t3.x}) > h || std::max({t1.x, t2.x, t3.x}) < -h) return false;
  if (std::min({t1.y, t2.y, t3.y}) > h || std::max({t1.y, t2.y, t3.y}) < -h) return false;
  if (std::min({t1.z, t2.z, t3.z}) > h || std::max({t1.z, t2.z, t3.z}) < -h) return false;
  V3 f[3] = {sub(t2, t1), sub(t3, t2), sub(t1, t3)};
  V3 u[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      V3 a = cross(u[i], f[j]);
      if (dot(a, a) < 1e-10) continue;
      double p1 = dot(t1, a), p2 = dot(t2, a), p3 = dot(t3, a);
      double r = h * std::fabs(a.x) + h * std::fabs(a.y) + h * std::fabs(a.z);
      if (std::min(p1, std::min(p2, p3)) > r || std::max(p1, std::max(p2, p3)) < -r) return false;
    }
  return true;
}

// bouzidi_math.jl:9-47
static bool ray_tri(V3 o, V3 d, V3 v1, V3 v2, V3 v3, double &t) {
  const double EPS = 1e-9;
  V3 e1 = sub(v2, v1), e2 = sub(v3, v1);
  V3 h = cross(d, e2);
  double a = dot(e1, h);
  if (std::fabs(a) < EPS) return false;
  double f = 1.0 / a;
  V3 s = sub(o, v1);
  double u = f * dot(s, h);
  if (u < 0.0 || u > 1.0) return false;
  V3 q = cross(s, e1);
  double v = f * dot(d, q);
  if (v < 0.0 || u + v > 1.0) return false;
  t = f * dot(e2, q);
  return t > EPS;
}

// Correctly rounded binary64 -> binary16 (round to nearest, ties to even),
// as Julia's Float16(::Float64).
static uint16_t d2h(double x) {
  uint64_t b;
  std::memcpy(&b, &x, 8);
  uint16_t sign = (uint16_t)((b >> 48) & 0x8000);
  double a = std::fabs(x);
  if (std::isnan(x)) return sign | 0x7e00;
  if (a >= 65520.0) return sign | 0x7c00;
  if (a < std::ldexp(1.0, -25)) {  // below half the smallest subnormal (ties handled below)
    if (a == std::ldexp(1.0, -25)) return sign;  // tie to even (0)
    return sign;
  }
  int e;
  std::frexp(a, &e);  // a = m * 2^e, m in [0.5, 1)
  int exp16 = e - 1;  // a in [2^exp16, 2^(exp16+1))
  double quantum = exp16 < -14 ? std::ldexp(1.0, -24) : std::ldexp(1.0, exp16 - 10);
  double n = a / quantum;  // exact (power-of-two scaling)
  double fl = std::floor(n);
  double rem = n - fl;
  uint64_t m = (uint64_t)fl;
  if (rem > 0.5 || (rem == 0.5 && (m & 1))) ++m;
  // assemble
  if (exp16 < -14) {  // subnormal range: value = m * 2^-24
    if (m >= 1024) return sign | (uint16_t)(1 << 10);  // rounded up to min normal
    return sign | (uint16_t)m;
  }
  if (m == 2048) { m = 1024; ++exp16; }
  if (exp16 > 15) return sign | 0x7c00;
  return sign | (uint16_t)(((exp16 + 15) << 10) | (m - 1024));
}

}  // namespace orcd

using namespace orcd;

extern "C" {

/* Block set of level `lvl` (domain.jl:39-152): level 1 = every block of the
 * dims; finer = triangle AABB blocks (+ wake box over parent blocks), orphan
 * filter against the parent set, `margin` halo layers with sibling
 * completion, full parent coverage.  Output sorted lexicographically
 * (bx, by, bz) into out[cap][3]; returns the count (or -needed if cap is short). */
int orc_level_blocks(int lvl, const double *tris, int ntri, double dx, const double *off, int bxm,
                     int bym, int bzm, const int32_t *prev, int nprev, double prev_bs_phys,
                     int wake_enabled, const double *wake_box /* x0,x1,y0,y1,z0,z1 */,
                     int margin_layers, int32_t *out, int cap) {
  std::set<B3> s;
  if (lvl == 1) {
    for (int bz = 1; bz <= bzm; ++bz)
      for (int by = 1; by <= bym; ++by)
        for (int bx = 1; bx <= bxm; ++bx) s.insert({bx, by, bz});
  } else {
    s = active_blocks(tris, ntri, dx, off, bxm, bym, bzm);
    if (wake_enabled) {
      for (int i = 0; i < nprev; ++i) {
        int cbx = prev[3 * i], cby = prev[3 * i + 1], cbz = prev[3 * i + 2];
        double bx0 = (cbx - 1) * prev_bs_phys, bx1 = cbx * prev_bs_phys;
        double by0 = (cby - 1) * prev_bs_phys, by1 = cby * prev_bs_phys;
        double bz0 = (cbz - 1) * prev_bs_phys, bz1 = cbz * prev_bs_phys;
        bool ox = bx0 <= wake_box[1] && bx1 >= wake_box[0];
        bool oy = by0 <= wake_box[3] && by1 >= wake_box[2];
        bool oz = bz0 <= wake_box[5] && bz1 >= wake_box[4];
        if (ox && oy && oz)
          for (int dz = 0; dz <= 1; ++dz)
            for (int dy = 0; dy <= 1; ++dy)
              for (int dx2 = 0; dx2 <= 1; ++dx2) {
                int fx = 2 * cbx - 1 + dx2, fy = 2 * cby - 1 + dy, fz = 2 * cbz - 1 + dz;
                if (in_dims(fx, fy, fz, bxm, bym, bzm)) s.insert({fx, fy, fz});
              }
      }
    }
    std::set<B3> ps;
    for (int i = 0; i < nprev; ++i) ps.insert({prev[3 * i], prev[3 * i + 1], prev[3 * i + 2]});
    std::set<B3> fin;
    for (const B3 &b : s)
      if (ps.count({jdiv2(b[0]), jdiv2(b[1]), jdiv2(b[2])})) fin.insert(b);
    s.swap(fin);
  }
  add_halo(s, margin_layers, bxm, bym, bzm);
  parent_coverage(s, bxm, bym, bzm);
  int n = (int)s.size();
  if (n > cap) return -n;
  int i = 0;
  for (const B3 &b : s) {  // std::set<array> iterates lexicographically
    out[3 * i] = b[0]; out[3 * i + 1] = b[1]; out[3 * i + 2] = b[2];
    ++i;
  }
  return n;
}

/* domain_topology.jl:135-159: table[b + n*dir] (1-based ids, 0 = none) */
void orc_neighbor_table(const int32_t *coords, int n, int bxm, int bym, int bzm, int32_t *table) {
  std::vector<int32_t> ptr((size_t)bxm * bym * bzm, 0);
  for (int i = 0; i < n; ++i) {
    int bx = coords[3 * i], by = coords[3 * i + 1], bz = coords[3 * i + 2];
    if (in_dims(bx, by, bz, bxm, bym, bzm))
      ptr[(bx - 1) + (size_t)bxm * ((by - 1) + (size_t)bym * (bz - 1))] = i + 1;
  }
  for (int i = 0; i < n; ++i)
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int dir = (dx + 1) + (dy + 1) * 3 + (dz + 1) * 9;
          int nx = coords[3 * i] + dx, ny = coords[3 * i + 1] + dy, nz = coords[3 * i + 2] + dz;
          table[i + (size_t)n * dir] =
              in_dims(nx, ny, nz, bxm, bym, bzm) ? ptr[(nx - 1) + (size_t)bxm * ((ny - 1) + (size_t)bym * (nz - 1))] : 0;
        }
}

/* domain_generation.jl:74-112 SAT surface marking -> obstacle[n*512] (0/1) */
void orc_voxelize(const int32_t *coords, int n, const double *tris, int ntri, double dx,
                  const double *off, uint8_t *obstacle) {
  std::vector<B3> blocks(n);
  for (int i = 0; i < n; ++i) blocks[i] = {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
  auto map = block_tri_map(tris, ntri, blocks, dx, off, dx * 2);
  const double h = 0.75 * dx;
  V3 o{off[0], off[1], off[2]};
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < n; ++i) {
    if (map[i].empty()) continue;
    for (int lz = 1; lz <= BS; ++lz)
      for (int ly = 1; ly <= BS; ++ly)
        for (int lx = 1; lx <= BS; ++lx) {
          V3 c{((blocks[i][0] - 1) * BS + lx - 0.5) * dx, ((blocks[i][1] - 1) * BS + ly - 0.5) * dx,
               ((blocks[i][2] - 1) * BS + lz - 0.5) * dx};
          bool shell = false;
          for (int t : map[i])
            if (tri_box(c, h, add(vert(tris, t, 0), o), add(vert(tris, t, 1), o), add(vert(tris, t, 2), o))) {
              shell = true;
              break;
            }
          if (shell) obstacle[(size_t)i * 512 + (lx - 1) + 8 * (ly - 1) + 64 * (lz - 1)] = 1;
        }
  }
}

/* domain_generation.jl:114-203: fill every non-obstacle cell not 6-connected
 * to a non-obstacle cell of the min-x block layer. */
void orc_flood_fill(const int32_t *coords, int n, int bxm, int bym, int bzm, uint8_t *obstacle) {
  if (n == 0) return;
  std::vector<int32_t> ptr((size_t)bxm * bym * bzm, 0);
  int minx = coords[0];
  for (int i = 0; i < n; ++i) {
    ptr[(coords[3 * i] - 1) + (size_t)bxm * ((coords[3 * i + 1] - 1) + (size_t)bym * (coords[3 * i + 2] - 1))] = i + 1;
    minx = std::min(minx, coords[3 * i]);
  }
  std::vector<uint8_t> vis((size_t)n * 512, 0);
  std::vector<int64_t> q;
  for (int i = 0; i < n; ++i)
    if (coords[3 * i] == minx)
      for (int c = 0; c < 512; ++c)
        if (!obstacle[(size_t)i * 512 + c]) { vis[(size_t)i * 512 + c] = 1; q.push_back((int64_t)i * 512 + c); }
  const int ddx[6] = {1, -1, 0, 0, 0, 0}, ddy[6] = {0, 0, 1, -1, 0, 0}, ddz[6] = {0, 0, 0, 0, 1, -1};
  for (size_t head = 0; head < q.size(); ++head) {
    int b = (int)(q[head] / 512), c = (int)(q[head] % 512);
    int lx = c % 8, ly = (c / 8) % 8, lz = c / 64;
    for (int j = 0; j < 6; ++j) {
      int nx = lx + ddx[j], ny = ly + ddy[j], nz = lz + ddz[j];
      int nb = b;
      if (nx < 0 || nx > 7 || ny < 0 || ny > 7 || nz < 0 || nz > 7) {
        int bx = coords[3 * b] + ddx[j], by = coords[3 * b + 1] + ddy[j], bz = coords[3 * b + 2] + ddz[j];
        if (!in_dims(bx, by, bz, bxm, bym, bzm)) continue;
        int id = ptr[(bx - 1) + (size_t)bxm * ((by - 1) + (size_t)bym * (bz - 1))];
        if (id <= 0) continue;
        nb = id - 1;
        nx = (nx + 8) % 8; ny = (ny + 8) % 8; nz = (nz + 8) % 8;
      }
      size_t ci = (size_t)nb * 512 + nx + 8 * ny + 64 * nz;
      if (!vis[ci] && !obstacle[ci]) { vis[ci] = 1; q.push_back((int64_t)ci); }
    }
  }
  for (size_t i = 0; i < (size_t)n * 512; ++i)
    if (!obstacle[i] && !vis[i]) obstacle[i] = 1;
}

static double sponge_prof(double x, double thk) {
  if (x <= 0.0) return 1.0;
  if (x >= thk) return 0.0;
  return 0.5 * (1.0 + std::cos(M_PI * x / thk));
}

/* domain_generation.jl:215-289 */
void orc_sponge(const int32_t *coords, int n, double dx, double Lx, double Ly, double Lz,
                float sponge_thickness, int symmetric, float *sponge) {
  const double st = (double)sponge_thickness;
  const double out_thk = Lx * std::max(st, 0.08);
  const double in_thk = Lx * 0.02;
  const double y_thk = Ly * st * 0.5, z_thk = Lz * st * 0.5;
  const double out_start = Lx - out_thk, y_top = Ly - y_thk, z_back = Lz - z_thk;
  for (int i = 0; i < n; ++i)
    for (int lz = 1; lz <= BS; ++lz)
      for (int ly = 1; ly <= BS; ++ly)
        for (int lx = 1; lx <= BS; ++lx) {
          double px = ((coords[3 * i] - 1) * BS + lx - 0.5) * dx;
          double py = ((coords[3 * i + 1] - 1) * BS + ly - 0.5) * dx;
          double pz = ((coords[3 * i + 2] - 1) * BS + lz - 0.5) * dx;
          double s = 0.0;
          if (px > out_start) s = std::max(s, sponge_prof(out_thk - (px - out_start), out_thk) * 1.0);
          if (px < in_thk) s = std::max(s, sponge_prof(px, in_thk) * 0.05);
          if (!symmetric && py < y_thk) s = std::max(s, sponge_prof(py, y_thk) * 0.1);
          if (py > y_top) s = std::max(s, sponge_prof(y_thk - (py - y_top), y_thk) * 0.1);
          if (pz < z_thk) s = std::max(s, sponge_prof(pz, z_thk) * 0.1);
          if (pz > z_back) s = std::max(s, sponge_prof(z_thk - (pz - z_back), z_thk) * 0.1);
          sponge[(size_t)i * 512 + (lx - 1) + 8 * (ly - 1) + 64 * (lz - 1)] = (float)s;
        }
}

/* domain_generation.jl:371-434 (distance in the units of dx) */
void orc_wall_dist(const int32_t *coords, int n, const uint8_t *obstacle, double dx, float *wd) {
  int bxm = 0, bym = 0, bzm = 0;
  for (int i = 0; i < n; ++i) {
    bxm = std::max(bxm, coords[3 * i]); bym = std::max(bym, coords[3 * i + 1]); bzm = std::max(bzm, coords[3 * i + 2]);
  }
  std::vector<int32_t> ptr((size_t)bxm * bym * bzm, 0);
  for (int i = 0; i < n; ++i)
    ptr[(coords[3 * i] - 1) + (size_t)bxm * ((coords[3 * i + 1] - 1) + (size_t)bym * (coords[3 * i + 2] - 1))] = i + 1;
  const float fdx = (float)dx;
  for (int b = 0; b < n; ++b)
    for (int lz = 1; lz <= BS; ++lz)
      for (int ly = 1; ly <= BS; ++ly)
        for (int lx = 1; lx <= BS; ++lx) {
          size_t own = (size_t)b * 512 + (lx - 1) + 8 * (ly - 1) + 64 * (lz - 1);
          if (obstacle[own]) continue;
          bool near = false;
          float md = 100.0f;
          for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
              for (int dxo = -1; dxo <= 1; ++dxo) {
                if (!dxo && !dy && !dz) continue;
                int nx = lx + dxo, ny = ly + dy, nz = lz + dz, nb = b;
                if (nx < 1 || nx > BS || ny < 1 || ny > BS || nz < 1 || nz > BS) {
                  int bx = coords[3 * b] + (nx < 1 ? -1 : (nx > BS ? 1 : 0));
                  int by = coords[3 * b + 1] + (ny < 1 ? -1 : (ny > BS ? 1 : 0));
                  int bz = coords[3 * b + 2] + (nz < 1 ? -1 : (nz > BS ? 1 : 0));
                  if (!(bx >= 1 && bx <= bxm && by >= 1 && by <= bym && bz >= 1 && bz <= bzm)) continue;
                  int id = ptr[(bx - 1) + (size_t)bxm * ((by - 1) + (size_t)bym * (bz - 1))];
                  if (id <= 0) continue;
                  nb = id - 1;
                  nx = nx < 1 ? nx + BS : (nx > BS ? nx - BS : nx);
                  ny = ny < 1 ? ny + BS : (ny > BS ? ny - BS : ny);
                  nz = nz < 1 ? nz + BS : (nz > BS ? nz - BS : nz);
                }
                if (obstacle[(size_t)nb * 512 + (nx - 1) + 8 * (ny - 1) + 64 * (nz - 1)]) {
                  near = true;
                  float d = std::sqrt((float)(dxo * dxo + dy * dy + dz * dz)) * fdx;
                  md = std::min(md, d);
                }
              }
          if (near) wd[own] = md;
        }
}

/* bouzidi_setup.jl:64-166 + bouzidi_math.jl:53-101.  q16 / tri: [n*512*27]
 * (zero-initialised by the caller); cells: [cap][4] = (block 1-based, x, y, z
 * 1-based) in block order then cell order (x fastest).  Returns the count. */
int orc_bouzidi_qmap(const int32_t *coords, int n, const double *tris, int ntri, double dx,
                     const double *off, uint16_t *q16, int32_t *tri_map, int32_t *cells, int cap) {
  std::vector<B3> blocks(n);
  for (int i = 0; i < n; ++i) blocks[i] = {coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
  auto map = block_tri_map(tris, ntri, blocks, dx, off, dx * 2.5);
  const size_t S = (size_t)n * 512;
  V3 o{off[0], off[1], off[2]};
  std::vector<std::vector<std::array<int32_t, 4>>> per(n);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < n; ++i) {
    if (map[i].empty()) continue;
    for (int lz = 1; lz <= BS; ++lz)
      for (int ly = 1; ly <= BS; ++ly)
        for (int lx = 1; lx <= BS; ++lx) {
          V3 c{((blocks[i][0] - 1) * BS + lx - 0.5) * dx, ((blocks[i][1] - 1) * BS + ly - 0.5) * dx,
               ((blocks[i][2] - 1) * BS + lz - 0.5) * dx};
          size_t own = (size_t)i * 512 + (lx - 1) + 8 * (ly - 1) + 64 * (lz - 1);
          bool has = false;
          int k = 0;
          for (int cz = -1; cz <= 1; ++cz)
            for (int cy = -1; cy <= 1; ++cy)
              for (int cx = -1; cx <= 1; ++cx, ++k) {
                if (!cx && !cy && !cz) continue;
                double nrm = std::sqrt((double)(cx * cx) + (double)(cy * cy) + (double)(cz * cz));
                V3 d{cx / nrm, cy / nrm, cz / nrm};
                double mt = INFINITY;
                int best = -1;
                for (int t : map[i]) {
                  double tt;
                  if (ray_tri(c, d, add(vert(tris, t, 0), o), add(vert(tris, t, 1), o), add(vert(tris, t, 2), o), tt) &&
                      tt < mt) {
                    mt = tt;
                    best = t + 1;
                  }
                }
                if (mt < INFINITY) {
                  double qv = mt / (dx * nrm);
                  if (qv > 0.0 && qv <= 1.0) {
                    q16[own + k * S] = d2h(qv);
                    tri_map[own + k * S] = best;
                    has = true;
                  }
                }
              }
          if (has) per[i].push_back({i + 1, lx, ly, lz});
        }
  }
  int cnt = 0;
  for (int i = 0; i < n; ++i)
    for (auto &c : per[i]) {
      if (cnt < cap) std::memcpy(cells + 4 * cnt, c.data(), 16);
      ++cnt;
    }
  return cnt > cap ? -cnt : cnt;
}

uint16_t orc_double_to_half(double x) { return d2h(x); }

/* Case scaling (physics_scaling.jl:63-191, compute_domain_from_mesh), FP64 in
 * the reference's expression order.  Inputs are the configuration globals
 * the reference reads (config_loader.jl); u_lattice and tau_min arrive as
 * the Float32 values the loader stores. */
struct OrcScaleIn {
  double mesh_min[3], mesh_max[3];
  double ref_length_cfg;   // REFERENCE_LENGTH_FOR_MESHING (<= 0: from the mesh)
  int32_t ref_dim;         // 0 :x, 1 :y, 2 :z, other: maximum extent
  double ref_chord_cfg, ref_area_cfg;
  int32_t symmetric;
  double moment_center[3];
  double u_phys, nu_phys, rho_phys;
  int32_t surface_resolution;
  float u_lattice, tau_min;
  double upstream, downstream, lateral, height;
  int32_t block_size, min_coarse_blocks, num_levels_cfg, auto_levels, max_levels;
  int32_t ddf_enabled;
  double prandtl;
};

struct OrcScaleOut {
  int32_t num_levels, nx, ny, nz, bx, by, bz;
  double ref_length, ref_chord, ref_area, re, tau_fine;
  double domain[3], offset[3], moment_center[3];
  double dx_fine, dx_coarse, dx_levels[16];
  double length_scale, velocity_scale, time_scale, nu_lattice, force_scale;
  float tau_levels[16];
  double tau_g_fine;
  float tau_g_levels[16];
};

int orc_domain_scaling(const OrcScaleIn *in, OrcScaleOut *o) {
  std::memset(o, 0, sizeof(*o));
  const double *mn = in->mesh_min, *mx = in->mesh_max;
  double ctr[3], ext[3];
  for (int i = 0; i < 3; ++i) {
    ctr[i] = (mn[i] + mx[i]) / 2;
    ext[i] = mx[i] - mn[i];
  }
  double L;
  if (in->ref_length_cfg > 0) L = in->ref_length_cfg;
  else if (in->ref_dim == 0) L = ext[0];
  else if (in->ref_dim == 1) L = ext[1];
  else if (in->ref_dim == 2) L = ext[2];
  else L = std::max(ext[0], std::max(ext[1], ext[2]));
  o->ref_length = L;
  o->ref_chord = in->ref_chord_cfg > 0 ? in->ref_chord_cfg : ext[0];
  o->ref_area = in->ref_area_cfg > 0 ? in->ref_area_cfg
                                     : (in->symmetric ? ext[1] * ext[2] * 2 : ext[1] * ext[2]);
  const double re = in->u_phys * L / in->nu_phys;
  o->re = re;
  // compute_tau_for_levels (:63-66): nu = Float64(u_lattice) * N / Re; tau = 3 nu + 1/2
  const double nu_f = (double)in->u_lattice * in->surface_resolution / re;
  const double tau_c = 3.0 * nu_f + 0.5;
  const double tau_fine = std::max(tau_c, (double)in->tau_min);
  o->tau_fine = tau_fine;
  double dx = L * (in->upstream + in->downstream) + ext[0];
  double dy = in->symmetric ? (mx[1] + L * in->lateral) : (ext[1] + 2 * L * in->lateral);
  double dz = ext[2] + 2 * L * in->height;
  const double dx_fine = L / in->surface_resolution;
  // compute_max_levels_for_domain (:68-71)
  const double ratio = std::min(dx, std::min(dy, dz)) / (dx_fine * in->min_coarse_blocks * in->block_size);
  const int max_lv = ratio < 1.0 ? 1 : (int)std::floor(1 + std::log2(ratio));
  int nl;
  if (in->num_levels_cfg > 0) nl = std::min(in->num_levels_cfg, max_lv);
  else nl = in->auto_levels ? std::min(max_lv, in->max_levels) : std::min(8, max_lv);
  if (nl < 1 || nl > 16) return -1;
  o->num_levels = nl;
  const double dxc = dx_fine * (double)(1L << (nl - 1));
  o->dx_fine = dx_fine;
  o->dx_coarse = dxc;
  for (int l = 1; l <= nl; ++l) o->dx_levels[l - 1] = dx_fine * (double)(1L << (nl - l));
  const int bs = in->block_size;
  auto cells = [&](double d) {
    const double c = std::ceil(std::ceil(d / dxc) / bs) * bs;
    return std::max(bs, (int)c);
  };
  o->nx = cells(dx);
  o->ny = cells(dy);
  o->nz = cells(dz);
  dx = o->nx * dxc;
  dy = o->ny * dxc;
  dz = o->nz * dxc;
  o->domain[0] = dx;
  o->domain[1] = dy;
  o->domain[2] = dz;
  o->bx = o->nx / bs;
  o->by = o->ny / bs;
  o->bz = o->nz / bs;
  const double mesh_x = L * in->upstream;
  const double mesh_y = in->symmetric ? 0.0 : (dy / 2 - ctr[1]);
  const double mesh_z = dz / 2 - ctr[2];
  o->offset[0] = mesh_x - mn[0];
  o->offset[1] = mesh_y;
  o->offset[2] = mesh_z;
  o->length_scale = dx_fine;
  o->velocity_scale = in->u_phys / (double)in->u_lattice;
  o->time_scale = o->length_scale / o->velocity_scale;
  o->nu_lattice = in->nu_phys * o->time_scale / (o->length_scale * o->length_scale);
  // tau per level (:136-140): tau_l = 1/2 + (tau_f - 1/2) 2^(L-l), stored as Float32
  for (int l = 1; l <= nl; ++l) {
    const double t = l == nl ? tau_fine : 0.5 + (tau_fine - 0.5) * std::pow(2.0, nl - l);
    o->tau_levels[l - 1] = (float)t;
  }
  // rho L^4 / T^2 (:142).  Julia evaluates x^2 as x*x and x^4 by compensated
  // squaring (correctly rounded here), which libm's pow matches.
  o->force_scale = in->rho_phys * std::pow(o->length_scale, 4.0) / (o->time_scale * o->time_scale);
  o->moment_center[0] = mn[0] + o->offset[0] + in->moment_center[0] * o->ref_chord;
  o->moment_center[1] = ctr[1] + o->offset[1] + in->moment_center[1] * o->ref_chord;
  o->moment_center[2] = ctr[2] + o->offset[2] + in->moment_center[2] * o->ref_chord;
  if (in->ddf_enabled) {
    // thermal relaxation (:148-159): kappa = nu_lattice / Pr
    const double kappa = o->nu_lattice / in->prandtl;
    o->tau_g_fine = 0.5 + 3.0 * kappa;
    for (int l = 1; l <= nl; ++l) {
      const double t = l == nl ? o->tau_g_fine : 0.5 + (o->tau_g_fine - 0.5) * std::pow(2.0, nl - l);
      o->tau_g_levels[l - 1] = (float)t;
    }
  }
  return 0;
}

}  // extern "C"
