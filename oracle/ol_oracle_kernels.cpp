/*
 * ol_oracle_kernels.cpp -- CPU restatement of the reference's device kernels.
 *
 * TEST INFRASTRUCTURE.  Only the tests, the smoke check and the CPU-baseline
 * leg of bench.py may load this code; it is the checker, never the product.
 * The reference (Julia, KernelAbstractions) cannot run in this environment
 * (no Julia toolchain), so this file restates its arithmetic cell by cell in
 * the reference's own expression order, compiled with -ffp-contract=off so
 * that every product and sum rounds exactly as the written Julia does.
 * Parity is UNPINNED against the reference itself: the reference ships no
 * tests, golden vectors or fixtures for this path.
 *
 * Each routine is a template over the arithmetic type: float is the parity
 * oracle of the FP32 GPU kernels, double is the accuracy oracle.
 *
 * Layout and index conventions are those of the reference's arrays (see
 * include/openludwig_b200.h); loops here are 0-based and convert where the
 * reference stores 1-based values.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ol_oracle_cell.h"

namespace orc {

template <class R>
void stream_collide(const Level<R> &L, const Parent<R> &P, const StepParams &sp) {
#pragma omp parallel for schedule(static)
  for (int b = 0; b < L.nB; ++b)
    for (int z = 1; z <= BS; ++z)
      for (int y = 1; y <= BS; ++y)
        for (int x = 1; x <= BS; ++x) cell_step(L, P, sp, b, x, y, z);
}

// bouzidi_kernel.jl:13-92 over the boundary-cell list
template <class R>
void bouzidi(R *f_out, const R *f_post, const uint16_t *q, const int32_t *cb, const int8_t *cxl,
             const int8_t *cyl, const int8_t *czl, int nbnd, const int32_t *nbr, int nB, float qmin) {
  for (int i = 0; i < nbnd; ++i) bouzidi_cell(f_out, f_post, q, cb, cxl, cyl, czl, i, nbr, nB, qmin);
}

// kernel_thermal.jl:14-202 over a level
template <class R>
void thermal(R *g_out, const R *g_in, R *g_post, R *T_out, const R *vel, const uint8_t *obs,
             const float *sponge, const int32_t *nbr, const int32_t *mx, const int32_t *my,
             const int32_t *mz, int nB, const Parent<R> &P, const ThermalParams &tp) {
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nB; ++b)
    for (int z = 1; z <= BS; ++z)
      for (int y = 1; y <= BS; ++y)
        for (int x = 1; x <= BS; ++x)
          thermal_cell(g_out, g_in, g_post, T_out, vel, obs, sponge, nbr, mx, my, mz, nB, P, tp, b,
                       x, y, z);
}

// ---------------------------------------------------------------------------
// Surface forces (surface.jl:143-507 map, 702-762 integrate), FP32 per
// triangle.  The reference adds the per-triangle terms with FP32 atomics in
// arbitrary order; here they are summed in FP64 in triangle order.
// ---------------------------------------------------------------------------
struct ForceP {
  float dx; int32_t dim_x, dim_y, dim_z;
  float off_x, off_y, off_z, pressure_scale, stress_scale, tau;
  int32_t search_radius;
  float c_wale, nu_bg, ref_x, ref_y, ref_z;
};

static bool cell_at(const int32_t *bptr, const ForceP &fp, int gx, int gy, int gz, size_t &ci) {
  if (gx < 1 || gy < 1 || gz < 1) return false;
  int bx = (gx - 1) / BS + 1, by = (gy - 1) / BS + 1, bz = (gz - 1) / BS + 1;
  if (bx < 1 || bx > fp.dim_x || by < 1 || by > fp.dim_y || bz < 1 || bz > fp.dim_z) return false;
  int b = bptr[(bx - 1) + fp.dim_x * ((by - 1) + fp.dim_y * (bz - 1))];
  if (b <= 0) return false;
  ci = (size_t)(b - 1) * NC + (gx - 1) % BS + BS * ((gy - 1) % BS) + BS * BS * ((gz - 1) % BS);
  return true;
}

static bool trilinear(const float *rho, const float *vel, const uint8_t *obs, const int32_t *bptr,
                      size_t S, const ForceP &fp, float px, float py, float pz, float &r, float &ux,
                      float &uy, float &uz, float &wq) {
  float inv = 1.0f / fp.dx;
  float fx = px * inv - 0.5f, fy = py * inv - 0.5f, fz = pz * inv - 0.5f;
  int ix0 = (int)std::floor(fx) + 1, iy0 = (int)std::floor(fy) + 1, iz0 = (int)std::floor(fz) + 1;
  float wx = rclamp(fx - (float)(ix0 - 1), 0.0f, 1.0f);
  float wy = rclamp(fy - (float)(iy0 - 1), 0.0f, 1.0f);
  float wz = rclamp(fz - (float)(iz0 - 1), 0.0f, 1.0f);
  float w0x = 1.0f - wx, w1x = wx, w0y = 1.0f - wy, w1y = wy, w0z = 1.0f - wz, w1z = wz;
  float ra = 0, xa = 0, ya = 0, za = 0, wa = 0;
  const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  for (int s = 0; s < 8; ++s) {
    float w = (ox[s] ? w1x : w0x) * (oy[s] ? w1y : w0y) * (oz[s] ? w1z : w0z);
    size_t ci;
    if (cell_at(bptr, fp, ix0 + ox[s], iy0 + oy[s], iz0 + oz[s], ci) && !obs[ci]) {
      ra += w * rho[ci];
      xa += w * vel[ci];
      ya += w * vel[ci + S];
      za += w * vel[ci + 2 * S];
      wa += w;
    }
  }
  if (wa > 0.01f) {
    float iw = 1.0f / wa;
    r = ra * iw; ux = xa * iw; uy = ya * iw; uz = za * iw; wq = wa;
    return true;
  }
  r = 1.0f; ux = uy = uz = 0.0f; wq = 0.0f;
  return false;
}

static void stress(const ForceP &fp, float rho, float ux, float uy, float uz, float nx, float ny,
                   float nz, float d, float &p, float &tx, float &ty, float &tz) {
  p = (rho - 1.0f) / 3.0f * fp.pressure_scale;
  float un = ux * nx + uy * ny + uz * nz;
  float utx = ux - un * nx, uty = uy - un * ny, utz = uz - un * nz;
  float ut = std::sqrt(utx * utx + uty * uty + utz * utz);
  float nu_mol = (fp.tau - 0.5f) / 3.0f;
  float nu_sgs = 0.0f;
  if (fp.c_wale > 0.0f && d > 0.01f && ut > 1e-10f) nu_sgs = (fp.c_wale * fp.c_wale) * (ut / d);
  nu_sgs = rmax(nu_sgs, fp.nu_bg);
  float nu_eff = nu_mol + nu_sgs;
  tx = ty = tz = 0.0f;
  if (ut > 1e-10f && d > 0.01f) {
    float tl = rho * nu_eff * ut / d;
    float tph = tl * fp.stress_scale;
    tx = (utx / ut) * tph; ty = (uty / ut) * tph; tz = (utz / ut) * tph;
  }
}

// Flow sample on one side of a triangle: side +1 follows map_stresses_kernel!
// (surface.jl:380-483, probes along +n, shell search accepts dot > 0), side -1
// map_minus_side_only_kernel! (surface.jl:545-640, probes along -n, accepts
// dot < 0, wall distance |dot| / dx).
static bool probe_side(int side, const float *rho, const float *vel, const uint8_t *obs,
                       const int32_t *bptr, size_t S, const ForceP &fp, float tx, float ty,
                       float tz, float n_x, float n_y, float n_z, float &br, float &bux,
                       float &buy, float &buz, float &bd) {
  br = 1.0f; bux = buy = buz = 0.0f; bd = 1.0f;
  float bq = 0.0f;
  bool found = false;
  for (int pi = 1; pi <= fp.search_radius; ++pi) {
    float dc = (float)pi + 0.5f;
    float px, py, pz;
    if (side > 0) {
      px = tx + n_x * dc * fp.dx; py = ty + n_y * dc * fp.dx; pz = tz + n_z * dc * fp.dx;
    } else {
      px = tx - n_x * dc * fp.dx; py = ty - n_y * dc * fp.dx; pz = tz - n_z * dc * fp.dx;
    }
    float r, ux, uy, uz, wq;
    bool ok = trilinear(rho, vel, obs, bptr, S, fp, px, py, pz, r, ux, uy, uz, wq);
    if (ok && wq >= 0.5f) { br = r; bux = ux; buy = uy; buz = uz; bd = dc; bq = wq; found = true; break; }
    if (ok && wq > bq) { br = r; bux = ux; buy = uy; buz = uz; bd = dc; bq = wq; found = true; }
  }
  if (found) return true;
  int gx0 = (int)std::floor(tx / fp.dx) + 1, gy0 = (int)std::floor(ty / fp.dx) + 1,
      gz0 = (int)std::floor(tz / fp.dx) + 1;
  float best = 1e10f;
  for (int rad = 1; rad <= fp.search_radius; ++rad) {
    if (found) break;
    for (int dz = -rad; dz <= rad; ++dz)
      for (int dy = -rad; dy <= rad; ++dy)
        for (int ddx = -rad; ddx <= rad; ++ddx) {
          if (!(std::abs(ddx) == rad || std::abs(dy) == rad || std::abs(dz) == rad)) continue;
          int gx = gx0 + ddx, gy = gy0 + dy, gz = gz0 + dz;
          size_t ci;
          if (!cell_at(bptr, fp, gx, gy, gz, ci) || obs[ci]) continue;
          float ddxp = ((float)gx - 0.5f) * fp.dx - tx, ddyp = ((float)gy - 0.5f) * fp.dx - ty,
                ddzp = ((float)gz - 0.5f) * fp.dx - tz;
          float dn = ddxp * n_x + ddyp * n_y + ddzp * n_z;
          if (side > 0 ? dn <= 0.0f : dn >= 0.0f) continue;
          float d2 = ddxp * ddxp + ddyp * ddyp + ddzp * ddzp;
          if (d2 < best) {
            best = d2; br = rho[ci]; bux = vel[ci]; buy = vel[ci + S]; buz = vel[ci + 2 * S];
            bd = (side > 0 ? dn : std::fabs(dn)) / fp.dx; found = true;
          }
        }
  }
  return found;
}

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------------------
// C entry points (ctypes).  Suffix _f32 / _f64 = arithmetic type.
// ---------------------------------------------------------------------------
#define ORC_LEVEL_ARGS(R)                                                                     \
  R *f_out, const R *f_in, R *f_post, R *rho, R *vel_out, const R *vel_in,                    \
      const uint8_t *obstacle, const float *sponge, const float *wall_dist, const int32_t *nbr, \
      const int32_t *mx, const int32_t *my, const int32_t *mz, int32_t nB, const R *pf,       \
      const R *prho, const R *pvel, const R *pf_old, const R *prho_old, const R *pvel_old,     \
      const int32_t *pptr, int32_t pdx, int32_t pdy, int32_t pdz, int32_t pnB,                \
      const StepParams *sp

#define ORC_LEVEL_BODY(R)                                                                     \
  Level<R> L{f_out, f_in, f_post, rho, vel_out, vel_in, obstacle, sponge, wall_dist, nbr, mx, my, \
             mz, nB};                                                                        \
  Parent<R> P{pf, prho, pvel, pf_old, prho_old, pvel_old, pptr, pdx, pdy, pdz, pnB};          \
  stream_collide(L, P, *sp);

extern "C" {
void orc_stream_collide_f32(ORC_LEVEL_ARGS(float)) { ORC_LEVEL_BODY(float) }
void orc_stream_collide_f64(ORC_LEVEL_ARGS(double)) { ORC_LEVEL_BODY(double) }

void orc_bouzidi_f32(float *f_out, const float *f_post, const uint16_t *q, const int32_t *cb,
                     const int8_t *cx, const int8_t *cy, const int8_t *cz, int32_t n,
                     const int32_t *nbr, int32_t nB, float qmin) {
  bouzidi(f_out, f_post, q, cb, cx, cy, cz, n, nbr, nB, qmin);
}
void orc_bouzidi_f64(double *f_out, const double *f_post, const uint16_t *q, const int32_t *cb,
                     const int8_t *cx, const int8_t *cy, const int8_t *cz, int32_t n,
                     const int32_t *nbr, int32_t nB, float qmin) {
  bouzidi(f_out, f_post, q, cb, cx, cy, cz, n, nbr, nB, qmin);
}

// Fine-to-coarse restriction, the opt-in extension of this package (no
// reference counterpart): each coarse cell covered by a fine block takes the
// average of its 8 children, non-equilibrium part rescaled by
// clamp((tau_c - 1/2) / (tau_f - 1/2), 0.01, 100); solid cells are skipped.
#define ORC_RESTRICT_BODY(R)                                                                  \
  const size_t fS = (size_t)nF * NC, cS = (size_t)nC * NC;                                   \
  for (int fb = 0; fb < nF; ++fb)                                                             \
    for (int q = 0; q < 64; ++q) {                                                            \
      const int i = q & 3, j = (q >> 2) & 3, l = q >> 4;                                      \
      const int gx = (mx[fb] - 1) * 4 + i + 1, gy = (my[fb] - 1) * 4 + j + 1,                \
                gz = (mz[fb] - 1) * 4 + l + 1;                                                \
      const int bx = (gx - 1) / 8 + 1, by = (gy - 1) / 8 + 1, bz = (gz - 1) / 8 + 1;          \
      if (bx > dx || by > dy || bz > dz) continue;                                            \
      const int pb = bptr[(bx - 1) + dx * ((by - 1) + dy * (bz - 1))];                        \
      if (pb <= 0) continue;                                                                  \
      const size_t cc = (size_t)(pb - 1) * NC + (gx - 1) % 8 + 8 * ((gy - 1) % 8) +           \
                        64 * ((gz - 1) % 8);                                                  \
      if (obs_c[cc]) continue;                                                                \
      size_t fc[8];                                                                           \
      bool solid = false;                                                                     \
      for (int s = 0; s < 8; ++s) {                                                           \
        fc[s] = (size_t)fb * NC + (2 * i + (s & 1)) + 8 * (2 * j + ((s >> 1) & 1)) +          \
                64 * (2 * l + (s >> 2));                                                      \
        solid = solid || obs_f[fc[s]];                                                        \
      }                                                                                       \
      if (solid) continue;                                                                    \
      R fbar[27], rho = 0, jx = 0, jy = 0, jz = 0;                                            \
      for (int k = 0; k < 27; ++k) {                                                          \
        R acc = 0;                                                                            \
        for (int s = 0; s < 8; ++s) acc = acc + f_f[fc[s] + k * fS];                          \
        fbar[k] = acc * (R)0.125;                                                             \
      }                                                                                       \
      for (int k = 0; k < 27; ++k) {                                                          \
        rho = rho + fbar[k];                                                                  \
        if (lat_cx(k) == 1) jx = jx + fbar[k]; else if (lat_cx(k) == -1) jx = jx - fbar[k];   \
        if (lat_cy(k) == 1) jy = jy + fbar[k]; else if (lat_cy(k) == -1) jy = jy - fbar[k];   \
        if (lat_cz(k) == 1) jz = jz + fbar[k]; else if (lat_cz(k) == -1) jz = jz - fbar[k];   \
      }                                                                                       \
      const R ux = jx / rho, uy = jy / rho, uz = jz / rho;                                    \
      const R tf = (R)tau_f - (R)0.5, tc = (R)tau_c - (R)0.5;                                 \
      const R sc = tf > (R)1e-6f ? rclamp(tc / tf, (R)0.01f, (R)100.0f) : (R)1;               \
      for (int k = 0; k < 27; ++k) {                                                          \
        const R fe = feq_auto(rho, ux, uy, uz, wk<R>(k), (R)lat_cx(k), (R)lat_cy(k),          \
                              (R)lat_cz(k), comp);                                            \
        f_c[cc + k * cS] = fe + (fbar[k] - fe) * sc;                                          \
      }                                                                                       \
      rho_c[cc] = rho;                                                                        \
      vel_c[cc] = ux; vel_c[cc + cS] = uy; vel_c[cc + 2 * cS] = uz;                           \
    }

void orc_restrict_f32(const float *f_f, const uint8_t *obs_f, const int32_t *mx,
                      const int32_t *my, const int32_t *mz, int32_t nF, float *f_c, float *rho_c,
                      float *vel_c, const uint8_t *obs_c, const int32_t *bptr, int32_t dx,
                      int32_t dy, int32_t dz, int32_t nC, float tau_f, float tau_c, int32_t comp) {
  ORC_RESTRICT_BODY(float)
}
void orc_restrict_f64(const double *f_f, const uint8_t *obs_f, const int32_t *mx,
                      const int32_t *my, const int32_t *mz, int32_t nF, double *f_c,
                      double *rho_c, double *vel_c, const uint8_t *obs_c, const int32_t *bptr,
                      int32_t dx, int32_t dy, int32_t dz, int32_t nC, float tau_f, float tau_c,
                      int32_t comp) {
  ORC_RESTRICT_BODY(double)
}

#define ORC_THERMAL_ARGS(R)                                                                   \
  R *g_out, const R *g_in, R *g_post, R *T_out, const R *vel, const uint8_t *obs,             \
      const float *sponge, const int32_t *nbr, const int32_t *mx, const int32_t *my,          \
      const int32_t *mz, int32_t nB, const R *pg, const R *pT, const R *pvel, const R *pg_old, \
      const R *pT_old, const R *pvel_old, const int32_t *pptr, int32_t pdx, int32_t pdy,      \
      int32_t pdz, int32_t pnB, const ThermalParams *tp
#define ORC_THERMAL_BODY(R)                                                                   \
  Parent<R> P{pg, pT, pvel, pg_old, pT_old, pvel_old, pptr, pdx, pdy, pdz, pnB};              \
  thermal(g_out, g_in, g_post, T_out, vel, obs, sponge, nbr, mx, my, mz, nB, P, *tp);

void orc_thermal_f32(ORC_THERMAL_ARGS(float)) { ORC_THERMAL_BODY(float) }
void orc_thermal_f64(ORC_THERMAL_ARGS(double)) { ORC_THERMAL_BODY(double) }


void orc_surface_forces(const float *cx, const float *cy, const float *cz, const float *nx,
                        const float *ny, const float *nz, const float *area, int32_t ntri,
                        const float *rho, const float *vel, const uint8_t *obs,
                        const int32_t *bptr, int32_t nB, const ForceP *fpp, float *pmap,
                        float *sxm, float *sym, float *szm, double *out) {
  const ForceP &fp = *fpp;
  const size_t S = (size_t)NC * nB;
  for (int j = 0; j < 9; ++j) out[j] = 0.0;
  for (int i = 0; i < ntri; ++i) {
    float tx = cx[i] + fp.off_x, ty = cy[i] + fp.off_y, tz = cz[i] + fp.off_z;
    float n_x = nx[i], n_y = ny[i], n_z = nz[i];
    float br, bux, buy, buz, bd;
    bool found = probe_side(1, rho, vel, obs, bptr, S, fp, tx, ty, tz, n_x, n_y, n_z, br, bux, buy,
                            buz, bd);
    float p = 0, sx = 0, sy = 0, sz = 0;
    if (found) stress(fp, br, bux, buy, buz, n_x, n_y, n_z, rmax(bd, 0.5f), p, sx, sy, sz);
    if (pmap) { pmap[i] = p; sxm[i] = sx; sym[i] = sy; szm[i] = sz; }
    float A = area[i];
    float fpx = -p * n_x * A, fpy = -p * n_y * A, fpz = -p * n_z * A;
    float fvx = sx * A, fvy = sy * A, fvz = sz * A;
    float Fx = fpx + fvx, Fy = fpy + fvy, Fz = fpz + fvz;
    float rx = tx - fp.ref_x, ry = ty - fp.ref_y, rz = tz - fp.ref_z;
    out[0] += fpx; out[1] += fpy; out[2] += fpz; out[3] += fvx; out[4] += fvy; out[5] += fvz;
    out[6] += (double)(ry * Fz - rz * Fy);
    out[7] += (double)(rz * Fx - rx * Fz);
    out[8] += (double)(rx * Fy - ry * Fx);
  }
}

// Two-sided per-triangle net force, compute_net_aerodynamics! (surface.jl:980-1034):
// plus-side stresses as map_stresses_kernel!; minus side zero for a closed body
// (surface.jl:987-997), else map_minus_side_only_kernel! (surface.jl:511-662,
// stress evaluated with the normal -n); then compute_net_triangle_forces_kernel!
// (surface.jl:665-700): F = -(p+ - p-) n A + (tau+ - tau-) A.
// maps: [8][ntri] = p+, tau+ x/y/z, p-, tau- x/y/z; net: [3][ntri].
void orc_surface_net_forces(const float *cx, const float *cy, const float *cz, const float *nx,
                            const float *ny, const float *nz, const float *area, int32_t ntri,
                            const float *rho, const float *vel, const uint8_t *obs,
                            const int32_t *bptr, int32_t nB, const ForceP *fpp,
                            int32_t closed_body, float *maps, float *net) {
  const ForceP &fp = *fpp;
  const size_t S = (size_t)NC * nB;
  const size_t T = (size_t)ntri;
  for (int i = 0; i < ntri; ++i) {
    float tx = cx[i] + fp.off_x, ty = cy[i] + fp.off_y, tz = cz[i] + fp.off_z;
    float n_x = nx[i], n_y = ny[i], n_z = nz[i];
    float br, bux, buy, buz, bd;
    float p = 0, sx = 0, sy = 0, sz = 0;
    if (probe_side(1, rho, vel, obs, bptr, S, fp, tx, ty, tz, n_x, n_y, n_z, br, bux, buy, buz, bd))
      stress(fp, br, bux, buy, buz, n_x, n_y, n_z, rmax(bd, 0.5f), p, sx, sy, sz);
    float pm = 0, sxm = 0, sym = 0, szm = 0;
    if (!closed_body &&
        probe_side(-1, rho, vel, obs, bptr, S, fp, tx, ty, tz, n_x, n_y, n_z, br, bux, buy, buz, bd))
      stress(fp, br, bux, buy, buz, -n_x, -n_y, -n_z, rmax(bd, 0.5f), pm, sxm, sym, szm);
    maps[i] = p; maps[T + i] = sx; maps[2 * T + i] = sy; maps[3 * T + i] = sz;
    maps[4 * T + i] = pm; maps[5 * T + i] = sxm; maps[6 * T + i] = sym; maps[7 * T + i] = szm;
    float pn = p - pm, snx = sx - sxm, sny = sy - sym, snz = sz - szm;
    float A = area[i];
    net[i] = -pn * n_x * A + snx * A;
    net[T + i] = -pn * n_y * A + sny * A;
    net[2 * T + i] = -pn * n_z * A + snz * A;
  }
}

float orc_half_to_float(uint16_t h) { return h2f(h); }
float orc_gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
  return gradient_noise(gx, gy, gz, seed);
}
}
