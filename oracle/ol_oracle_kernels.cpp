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

namespace orc {

constexpr int BS = 8, NC = 512, Q = 27;

// lattice.jl:5-56 / timestep.jl:161-179 (k-order: x fastest)
struct Lattice {
  int cx[27], cy[27], cz[27], opp[27], my[27], mz[27];
  float wf[27];
  Lattice() {
    int k = 0;
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x, ++k) {
          cx[k] = x; cy[k] = y; cz[k] = z;
          const int d2 = x * x + y * y + z * z;
          wf[k] = d2 == 0 ? 8.0f / 27.0f : d2 == 1 ? 2.0f / 27.0f : d2 == 2 ? 1.0f / 54.0f
                                                                           : 1.0f / 216.0f;
        }
    for (int i = 0; i < 27; ++i)
      for (int j = 0; j < 27; ++j) {
        if (cx[j] == -cx[i] && cy[j] == -cy[i] && cz[j] == -cz[i]) opp[i] = j;
        if (cx[j] == cx[i] && cy[j] == -cy[i] && cz[j] == cz[i]) my[i] = j;
        if (cx[j] == cx[i] && cy[j] == cy[i] && cz[j] == -cz[i]) mz[i] = j;
      }
  }
};
static const Lattice LAT;

// Weights: the Float32 quotients of the reference for float; exact quotients
// for the double (accuracy-oracle) instantiation.
template <class R> inline R wk(int k) { return (R)LAT.wf[k]; }
template <> inline double wk<double>(int k) {
  const int d2 = LAT.cx[k] * LAT.cx[k] + LAT.cy[k] * LAT.cy[k] + LAT.cz[k] * LAT.cz[k];
  return d2 == 0 ? 8.0 / 27.0 : d2 == 1 ? 2.0 / 27.0 : d2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
}
// c_s^2: the reference's literal 0.333333333f0 (kernel_cumulant.jl:420); exact for double.
template <class R> inline R cs2_lit() { return (R)0.333333333f; }
template <> inline double cs2_lit<double>() { return 1.0 / 3.0; }
template <class R> inline R third_lit() { return (R)(1.0f / 3.0f); }
template <> inline double third_lit<double>() { return 1.0 / 3.0; }
template <class R> inline R rmax(R a, R b) { return a > b ? a : b; }
template <class R> inline R rmin(R a, R b) { return a < b ? a : b; }
template <class R> inline R rclamp(R x, R lo, R hi) { return x > hi ? hi : (x < lo ? lo : x); }

// physics_utils.jl:19-24
template <class R>
R feq(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz) {
  R cu = cx * ux + cy * uy + cz * uz;
  R usq = ux * ux + uy * uy + uz * uz;
  return rho * w * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
}
// physics_utils.jl:39-61
template <class R>
R feq_comp(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz) {
  R cu = cx * ux + cy * uy + cz * uz;
  R usq = ux * ux + uy * uy + uz * uz;
  R cu2 = cu * cu, cu3 = cu2 * cu, cu4 = cu2 * cu2, usq2 = usq * usq;
  R val = (R)1 + (R)3 * cu + (R)4.5 * cu2 - (R)1.5 * usq;
  val += (R)4.5 * cu3 - (R)4.5 * cu * usq;
  val += (R)3.375 * cu4 - (R)6.75 * cu2 * usq + (R)1.125 * usq2;
  return rho * w * val;
}
template <class R>
R feq_auto(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz, int comp) {
  return comp == 1 ? feq_comp(rho, ux, uy, uz, w, cx, cy, cz) : feq(rho, ux, uy, uz, w, cx, cy, cz);
}
// physics_utils.jl:78-83
template <class R>
R geq(R T, R ux, R uy, R uz, R w, R cx, R cy, R cz) {
  R cu = cx * ux + cy * uy + cz * uz;
  return w * T * ((R)1 + (R)3 * cu);
}
// physics_utils.jl:5-17
inline uint32_t gpu_hash(int32_t x) {
  uint32_t h = (uint32_t)x;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  return h ^ (h >> 16);
}
inline float gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
  uint32_t c = (uint32_t)gx * 374761393u + (uint32_t)gy * 668265263u + (uint32_t)gz * 1274126177u +
               (uint32_t)seed;
  uint32_t h = gpu_hash((int32_t)c);
  return (float)(h & 0xFFFFu) / 32768.0f - 1.0f;
}

struct StepParams {  // mirrors ol_step_params
  int32_t op;
  float tau_molecular, tau_parent, c_wale, nu_sgs_background;
  int32_t is_level_1, is_symmetric;
  int32_t nx_global, ny_global, nz_global;
  float u_inlet;
  int32_t wall_model_active, time_step_seed, store_post_collision;
  float inlet_turbulence, temporal_weight;
  int32_t use_temporal_interp, sponge_blend_distributions;
  float omega_bulk, omega_3, omega_4;
  int32_t adaptive_omega4;
  float lambda_param;
  int32_t limiter_type, compressible_corr;
};

template <class R>
struct Level {  // one level's arrays (host)
  R *f_out; const R *f_in; R *f_post;
  R *rho; R *vel_out; const R *vel_in;
  const uint8_t *obstacle; const float *sponge; const float *wall_dist;
  const int32_t *nbr; const int32_t *mx, *my, *mz;
  int32_t nB;
};
template <class R>
struct Parent {
  const R *f, *rho, *vel, *f_old, *rho_old, *vel_old;
  const int32_t *ptr; int32_t dx, dy, dz, nB;
};

// physics_interpolation.jl:4-127 (flow) and :135-247 (thermal: thermal=true)
template <class R>
R interpolate(const Parent<R> &P, int fgx, int fgy, int fgz, int k, R w, R cx, R cy, R cz,
              R tau_coarse, R tau_fine, R tw, int use_temporal, int comp, bool thermal) {
  R pxc = ((R)fgx - (R)0.5) * (R)0.5;
  R pyc = ((R)fgy - (R)0.5) * (R)0.5;
  R pzc = ((R)fgz - (R)0.5) * (R)0.5;
  int px0 = (int)std::floor(pxc), py0 = (int)std::floor(pyc), pz0 = (int)std::floor(pzc);
  int px1 = px0 + 1, py1 = py0 + 1, pz1 = pz0 + 1;
  R wx = pxc - (R)px0, wy = pyc - (R)py0, wz = pzc - (R)pz0;
  px0 = px0 > 1 ? px0 : 1;
  py0 = py0 > 1 ? py0 : 1;
  pz0 = pz0 > 1 ? pz0 : 1;
  const size_t S = (size_t)NC * P.nB;
  auto blended = [&](int pgx, int pgy, int pgz, R *out) -> bool {
    int pbx = (pgx - 1) / BS + 1, pby = (pgy - 1) / BS + 1, pbz = (pgz - 1) / BS + 1;
    if (pbx >= 1 && pbx <= P.dx && pby >= 1 && pby <= P.dy && pbz >= 1 && pbz <= P.dz) {
      int pb = P.ptr[(pbx - 1) + P.dx * ((pby - 1) + P.dy * (pbz - 1))];
      if (pb > 0) {
        size_t c = (size_t)(pb - 1) * NC + (pgx - 1) % BS + BS * ((pgy - 1) % BS) +
                   BS * BS * ((pgz - 1) % BS);
        R fn = P.f[c + k * S], rn = P.rho[c], uxn = P.vel[c], uyn = P.vel[c + S], uzn = P.vel[c + 2 * S];
        if (use_temporal == 1 && tw < (R)0.99) {
          R fo = P.f_old[c + k * S], ro = P.rho_old[c], uxo = P.vel_old[c], uyo = P.vel_old[c + S],
            uzo = P.vel_old[c + 2 * S];
          out[0] = fo * ((R)1 - tw) + fn * tw;
          out[1] = ro * ((R)1 - tw) + rn * tw;
          out[2] = uxo * ((R)1 - tw) + uxn * tw;
          out[3] = uyo * ((R)1 - tw) + uyn * tw;
          out[4] = uzo * ((R)1 - tw) + uzn * tw;
          return true;
        }
        out[0] = fn; out[1] = rn; out[2] = uxn; out[3] = uyn; out[4] = uzn;
        return true;
      }
    }
    out[0] = w; out[1] = (R)1; out[2] = (R)0; out[3] = (R)0; out[4] = (R)0;
    return false;
  };
  R d[8][5];
  bool ok[8];
  ok[0] = blended(px0, py0, pz0, d[0]);
  ok[1] = blended(px1, py0, pz0, d[1]);
  ok[2] = blended(px0, py1, pz0, d[2]);
  ok[3] = blended(px1, py1, pz0, d[3]);
  ok[4] = blended(px0, py0, pz1, d[4]);
  ok[5] = blended(px1, py0, pz1, d[5]);
  ok[6] = blended(px0, py1, pz1, d[6]);
  ok[7] = blended(px1, py1, pz1, d[7]);
  for (int s = 1; s < 8; ++s)
    if (!ok[s]) std::memcpy(d[s], d[0], sizeof(d[0]));
  R v[5];
  for (int i = 0; i < 5; ++i) {
    R c00 = d[0][i] * ((R)1 - wx) + d[1][i] * wx;
    R c01 = d[4][i] * ((R)1 - wx) + d[5][i] * wx;
    R c10 = d[2][i] * ((R)1 - wx) + d[3][i] * wx;
    R c11 = d[6][i] * ((R)1 - wx) + d[7][i] * wx;
    R c0 = c00 * ((R)1 - wy) + c10 * wy;
    R c1 = c01 * ((R)1 - wy) + c11 * wy;
    v[i] = c0 * ((R)1 - wz) + c1 * wz;
  }
  R fe = thermal ? geq(v[1], v[2], v[3], v[4], w, cx, cy, cz)
                 : feq_auto(v[1], v[2], v[3], v[4], w, cx, cy, cz, comp);
  R fneq = v[0] - fe;
  R tc = tau_coarse - (R)0.5, tf = tau_fine - (R)0.5;
  R sc = tc > (R)1e-6 ? rclamp(tf / tc, (R)0.01, (R)100) : (R)1;
  return fe + fneq * sc;
}

// physics_utils.jl:85-123
template <class R>
void vel_nb(const Level<R> &L, int x, int y, int z, int b, int dx, int dy, int dz, R &ux, R &uy,
            R &uz) {
  const size_t S = (size_t)NC * L.nB;
  int nx = x + dx, ny = y + dy, nz = z + dz;  // 1-based
  size_t c;
  if (nx >= 1 && nx <= BS && ny >= 1 && ny <= BS && nz >= 1 && nz <= BS) {
    c = (size_t)b * NC + (nx - 1) + BS * (ny - 1) + BS * BS * (nz - 1);
  } else {
    int ox = nx < 1 ? -1 : (nx > BS ? 1 : 0), oy = ny < 1 ? -1 : (ny > BS ? 1 : 0),
        oz = nz < 1 ? -1 : (nz > BS ? 1 : 0);
    int dir = (ox + 1) + (oy + 1) * 3 + (oz + 1) * 9;
    int nb = L.nbr[b + (size_t)L.nB * dir];
    if (nb > 0) {
      int nnx = nx < 1 ? nx + BS : (nx > BS ? nx - BS : nx);
      int nny = ny < 1 ? ny + BS : (ny > BS ? ny - BS : ny);
      int nnz = nz < 1 ? nz + BS : (nz > BS ? nz - BS : nz);
      c = (size_t)(nb - 1) * NC + (nnx - 1) + BS * (nny - 1) + BS * BS * (nnz - 1);
    } else {
      c = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
    }
  }
  ux = L.vel_in[c]; uy = L.vel_in[c + S]; uz = L.vel_in[c + 2 * S];
}

template <class R>
inline void chim_f(R &a, R &b, R &c, R u) {
  R m0 = a + b + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = m1 - u * m0;
  c = m2 - (R)2 * u * m1 + u * u * m0;
}
template <class R>
inline void chim_b(R &a, R &b, R &c, R u) {
  R m0 = a, m1 = b + u * a, m2 = c + (R)2 * u * b + u * u * a;
  R fp = (m2 + m1) * (R)0.5, fm = (m2 - m1) * (R)0.5, f0 = m0 - m2;
  a = fm; b = f0; c = fp;
}

// kernel_cumulant.jl:29-627 and kernel_regularized_bgk.jl:4-325 (op == 1),
// one cell (x, y, z 1-based; b 0-based).
template <class R>
void cell_step(const Level<R> &L, const Parent<R> &P, const StepParams &sp, int b, int x, int y,
               int z) {
  const size_t S = (size_t)NC * L.nB;
  const size_t own = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
  const int gx = (L.mx[b] - 1) * BS + x, gy = (L.my[b] - 1) * BS + y, gz = (L.mz[b] - 1) * BS + z;
  const bool is_obs = L.obstacle[own] != 0;
  const R u_in = (R)sp.u_inlet;
  R rho = 0, jx = 0, jy = 0, jz = 0;
  R fs[27];
  for (int k = 0; k < 27; ++k) {
    int cx = LAT.cx[k], cy = LAT.cy[k], cz = LAT.cz[k];
    int sx = x - cx, sy = y - cy, sz = z - cz;
    R val = 0;
    if (sx >= 1 && sx <= BS && sy >= 1 && sy <= BS && sz >= 1 && sz <= BS) {
      val = L.f_in[(size_t)b * NC + (sx - 1) + BS * (sy - 1) + BS * BS * (sz - 1) + k * S];
    } else {
      int ox = sx < 1 ? -1 : (sx > BS ? 1 : 0), oy = sy < 1 ? -1 : (sy > BS ? 1 : 0),
          oz = sz < 1 ? -1 : (sz > BS ? 1 : 0);
      int dir = (ox + 1) + (oy + 1) * 3 + (oz + 1) * 9;
      int nb = L.nbr[b + (size_t)L.nB * dir];
      if (nb > 0) {
        int nsx = sx < 1 ? sx + BS : (sx > BS ? sx - BS : sx);
        int nsy = sy < 1 ? sy + BS : (sy > BS ? sy - BS : sy);
        int nsz = sz < 1 ? sz + BS : (sz > BS ? sz - BS : sz);
        val = L.f_in[(size_t)(nb - 1) * NC + (nsx - 1) + BS * (nsy - 1) + BS * BS * (nsz - 1) + k * S];
      } else {
        int sgx = gx - cx, sgy = gy - cy, sgz = gz - cz;
        if (sgx < 1) {
          R noise = sp.inlet_turbulence > 0.0f
                        ? (R)gradient_noise(gy, gz, sp.time_step_seed, 1234) * (R)sp.inlet_turbulence * u_in
                        : (R)0;
          R uinst = u_in + noise;
          val = feq_auto((R)1, uinst, (R)0, (R)0, wk<R>(k), (R)cx, (R)cy, (R)cz, sp.compressible_corr);
        } else if (sgx > sp.nx_global) {
          val = feq_auto((R)1, u_in, (R)0, (R)0, wk<R>(k), (R)cx, (R)cy, (R)cz, sp.compressible_corr);
        } else if ((sgy < 1 && sp.is_symmetric == 1) || sgy < 1 || sgy > sp.ny_global) {
          val = L.f_in[own + LAT.my[k] * S];
        } else if (sgz < 1 || sgz > sp.nz_global) {
          val = L.f_in[own + LAT.mz[k] * S];
        } else if (sp.is_level_1 == 0) {
          val = interpolate(P, sgx, sgy, sgz, k, wk<R>(k), (R)cx, (R)cy, (R)cz, (R)sp.tau_parent,
                            (R)sp.tau_molecular, (R)sp.temporal_weight, sp.use_temporal_interp,
                            sp.compressible_corr, false);
        } else {
          val = wk<R>(k);
        }
      }
    }
    fs[k] = val;
    rho += val;
    jx += val * (R)cx;
    jy += val * (R)cy;
    jz += val * (R)cz;
  }
  const bool post = sp.store_post_collision == 1 && L.f_post;
  if (is_obs) {
    L.vel_out[own] = 0; L.vel_out[own + S] = 0; L.vel_out[own + 2 * S] = 0;
    L.rho[own] = 1;
    for (int k = 0; k < 27; ++k) {
      R fc = fs[LAT.opp[k]];
      L.f_out[own + k * S] = fc;
      if (post) L.f_post[own + k * S] = fc;
    }
    return;
  }
  rho = rmax(rho, (R)0.01);
  R inv_rho = (R)1 / rho;
  R ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  R spg = (R)L.sponge[own];
  if (spg > (R)0) {
    R rho_t = 1, ux_t = u_in;
    rho = rho * ((R)1 - spg) + rho_t * spg;
    ux = ux * ((R)1 - spg) + ux_t * spg;
    uy = uy * ((R)1 - spg);
    uz = uz * ((R)1 - spg);
    if (sp.sponge_blend_distributions == 1)
      for (int k = 0; k < 27; ++k) {
        R ft = feq_auto(rho_t, ux_t, (R)0, (R)0, wk<R>(k), (R)LAT.cx[k], (R)LAT.cy[k], (R)LAT.cz[k],
                        sp.compressible_corr);
        fs[k] = fs[k] * ((R)1 - spg) + ft * spg;
      }
  }
  R Fx = 0, Fy = 0, Fz = 0;
  const R tau_mol = (R)sp.tau_molecular;
  if (sp.wall_model_active == 1) {
    R dw = (R)L.wall_dist[own];
    if (dw > (R)0 && dw < (R)10) {
      R umag = std::sqrt(ux * ux + uy * uy + uz * uz);
      R nuv = (tau_mol - (R)0.5) / (R)3;
      if (umag > (R)1e-6 && nuv > (R)1e-10) {
        R ut = umag * std::pow(nuv / (dw * umag + (R)1e-10), (R)1 / (R)7) *
               std::pow((R)2 * (R)8.3, -(R)1 / (R)7);
        ut = rmax(ut, (R)1e-6);
        R yp = ut * dw / nuv;
        if (yp > (R)11.81) {
          R upl = ((R)1 / (R)0.41) * std::log(yp) + (R)5.2;
          if (upl > (R)0.1) {
            ut = ut * ((umag / ut) / upl);
            ut = rmax(ut, (R)1e-6);
          }
        }
        R tw = rho * ut * ut, tr = rho * nuv * (umag / dw);
        if (tw > tr) {
          R fm = (tw - tr) / dw;
          Fx = -fm * ux / umag; Fy = -fm * uy / umag; Fz = -fm * uz / umag;
        }
      }
    }
  }
  R uxe = ux + (R)0.5 * Fx * inv_rho, uye = uy + (R)0.5 * Fy * inv_rho, uze = uz + (R)0.5 * Fz * inv_rho;
  L.vel_out[own] = ux; L.vel_out[own + S] = uy; L.vel_out[own + 2 * S] = uz;
  L.rho[own] = rho;

  // WALE from vel_in gradients
  R nu_eddy = 0;
  {
    R eX, eY, eZ, wX, wY, wZ, nX, nY, nZ, sX, sY, sZ, tX, tY, tZ, bX, bY, bZ;
    vel_nb(L, x, y, z, b, 1, 0, 0, eX, eY, eZ);
    vel_nb(L, x, y, z, b, -1, 0, 0, wX, wY, wZ);
    vel_nb(L, x, y, z, b, 0, 1, 0, nX, nY, nZ);
    vel_nb(L, x, y, z, b, 0, -1, 0, sX, sY, sZ);
    vel_nb(L, x, y, z, b, 0, 0, 1, tX, tY, tZ);
    vel_nb(L, x, y, z, b, 0, 0, -1, bX, bY, bZ);
    R h = (R)0.5;
    R g11 = h * (eX - wX), g12 = h * (nX - sX), g13 = h * (tX - bX);
    R g21 = h * (eY - wY), g22 = h * (nY - sY), g23 = h * (tY - bY);
    R g31 = h * (eZ - wZ), g32 = h * (nZ - sZ), g33 = h * (tZ - bZ);
    R q11 = g11 * g11 + g12 * g21 + g13 * g31, q12 = g11 * g12 + g12 * g22 + g13 * g32,
      q13 = g11 * g13 + g12 * g23 + g13 * g33;
    R q21 = g21 * g11 + g22 * g21 + g23 * g31, q22 = g21 * g12 + g22 * g22 + g23 * g32,
      q23 = g21 * g13 + g22 * g23 + g23 * g33;
    R q31 = g31 * g11 + g32 * g21 + g33 * g31, q32 = g31 * g12 + g32 * g22 + g33 * g32,
      q33 = g31 * g13 + g32 * g23 + g33 * g33;
    R tr = (q11 + q22 + q33) / (R)3;
    R d11 = q11 - tr, d22 = q22 - tr, d33 = q33 - tr;
    R d12 = h * (q12 + q21), d13 = h * (q13 + q31), d23 = h * (q23 + q32);
    R s12 = h * (g12 + g21), s13 = h * (g13 + g31), s23 = h * (g23 + g32);
    R OP1 = d11 * d11 + d22 * d22 + d33 * d33 + (R)2 * (d12 * d12 + d13 * d13 + d23 * d23);
    R OP2 = g11 * g11 + g22 * g22 + g33 * g33 + (R)2 * (s12 * s12 + s13 * s13 + s23 * s23);
    if (OP1 > (R)1e-12) {
      R o32 = OP1 * std::sqrt(OP1);
      R o52 = OP2 * OP2 * std::sqrt(rmax(OP2, (R)1e-12));
      R den = o52 + OP1 * std::sqrt(std::sqrt(rmax(OP1, (R)1e-12)));
      if (den > (R)1e-12) nu_eddy = ((R)sp.c_wale * (R)sp.c_wale) * o32 / den;
    }
  }
  nu_eddy = rmax(nu_eddy, (R)sp.nu_sgs_background);

  R A[27];
  R om;
  if (sp.op == 0) {
    R nu_mol = (tau_mol - (R)0.5) / (R)3;
    R tau_eff = (R)0.5 + (R)3 * (nu_mol + nu_eddy);
    R om1 = (R)1 / rmax(tau_eff, (R)0.500001);
    om = om1;
    R omb = (R)sp.omega_bulk, om3 = (R)sp.omega_3, om4 = (R)sp.omega_4, om4d = om4;
    if (sp.adaptive_omega4 == 1) {
      R a = om1 - (R)2;
      R den = (R)sp.lambda_param * om1 + (R)1e-10;
      R Av = -(a * a) / den;
      om4d = rclamp(Av, (R)0.01, (R)2);
    }
    for (int k = 0; k < 27; ++k) A[k] = fs[k];
    for (int iz = 0; iz < 3; ++iz)
      for (int iy = 0; iy < 3; ++iy) {
        int bse = 3 * iy + 9 * iz;
        chim_f(A[bse], A[bse + 1], A[bse + 2], uxe);
      }
    for (int iz = 0; iz < 3; ++iz)
      for (int ma = 0; ma < 3; ++ma) chim_f(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz], uye);
    for (int mb = 0; mb < 3; ++mb)
      for (int ma = 0; ma < 3; ++ma) chim_f(A[ma + 3 * mb], A[ma + 3 * mb + 9], A[ma + 3 * mb + 18], uze);
    R k000 = A[0];
    R ir = (R)1 / rmax(k000, (R)0.01);
    R c200 = A[2] * ir, c020 = A[6] * ir, c002 = A[18] * ir;
    R c110 = A[4] * ir, c101 = A[10] * ir, c011 = A[12] * ir;
    R c210 = A[5] * ir, c120 = A[7] * ir, c201 = A[11] * ir;
    R c021 = A[15] * ir, c102 = A[19] * ir, c012 = A[21] * ir;
    R c111 = A[13] * ir;
    R c220n = A[8] * ir, c202n = A[20] * ir, c022n = A[24] * ir;
    R c211n = A[14] * ir, c121n = A[16] * ir, c112n = A[22] * ir;
    R C220 = c220n - c200 * c020 - (R)2 * c110 * c110;
    R C202 = c202n - c200 * c002 - (R)2 * c101 * c101;
    R C022 = c022n - c020 * c002 - (R)2 * c011 * c011;
    R C211 = c211n - c200 * c011 - (R)2 * c110 * c101;
    R C121 = c121n - c020 * c101 - (R)2 * c110 * c011;
    R C112 = c112n - c002 * c110 - (R)2 * c101 * c011;
    R cs2 = cs2_lit<R>();
    R Dtr = c200 + c020 + c002;
    R Dtre = (R)3 * cs2;
    R Dtrs = ((R)1 - omb) * Dtr + omb * Dtre;
    R D1 = c200 - c020, D2 = c200 - c002;
    R D1s = ((R)1 - om1) * D1, D2s = ((R)1 - om1) * D2;
    R c200s = (Dtrs + D1s + D2s) / (R)3;
    R c020s = (Dtrs - (R)2 * D1s + D2s) / (R)3;
    R c002s = (Dtrs + D1s - (R)2 * D2s) / (R)3;
    R c110s = ((R)1 - om1) * c110, c101s = ((R)1 - om1) * c101, c011s = ((R)1 - om1) * c011;
    if (sp.limiter_type == 1) {
      R b110 = std::sqrt(rmax(c200s * c020s, (R)0));
      R b101 = std::sqrt(rmax(c200s * c002s, (R)0));
      R b011 = std::sqrt(rmax(c020s * c002s, (R)0));
      c110s = rclamp(c110s, -b110, b110);
      c101s = rclamp(c101s, -b101, b101);
      c011s = rclamp(c011s, -b011, b011);
    }
    R c210s = ((R)1 - om3) * c210, c120s = ((R)1 - om3) * c120, c201s = ((R)1 - om3) * c201;
    R c021s = ((R)1 - om3) * c021, c102s = ((R)1 - om3) * c102, c012s = ((R)1 - om3) * c012;
    R c111s = ((R)1 - om3) * c111;
    R C220s = ((R)1 - om4d) * C220, C202s = ((R)1 - om4d) * C202, C022s = ((R)1 - om4d) * C022;
    R C211s = ((R)1 - om4) * C211, C121s = ((R)1 - om4) * C121, C112s = ((R)1 - om4) * C112;
    R c220s = C220s + c200s * c020s + (R)2 * c110s * c110s;
    R c202s = C202s + c200s * c002s + (R)2 * c101s * c101s;
    R c022s = C022s + c020s * c002s + (R)2 * c011s * c011s;
    R c211s = C211s + c200s * c011s + (R)2 * c110s * c101s;
    R c121s = C121s + c020s * c101s + (R)2 * c110s * c011s;
    R c112s = C112s + c002s * c110s + (R)2 * c101s * c011s;
    R c221s = c200s * c021s + c020s * c201s + (R)4 * c110s * c111s + (R)2 * c101s * c120s +
              (R)2 * c011s * c210s;
    R c212s = c200s * c012s + c002s * c210s + (R)2 * c110s * c102s + (R)4 * c101s * c111s +
              (R)2 * c011s * c201s;
    R c122s = c020s * c102s + c002s * c120s + (R)2 * c110s * c012s + (R)4 * c011s * c111s +
              (R)2 * c101s * c021s;
    R c222s = c200s * C022s + c020s * C202s + c002s * C220s +
              (R)4 * (c110s * C112s + c101s * C121s + c011s * C211s);
    c222s += (R)2 * (c210s * c012s + c201s * c021s + c120s * c102s) + (R)4 * c111s * c111s;
    c222s += c200s * c020s * c002s +
             (R)2 * (c200s * c011s * c011s + c020s * c101s * c101s + c002s * c110s * c110s) +
             (R)8 * c110s * c101s * c011s;
    R r = k000;
    A[0] = r;
    A[1] = 0; A[3] = 0; A[9] = 0;
    A[2] = r * c200s; A[6] = r * c020s; A[18] = r * c002s;
    A[4] = r * c110s; A[10] = r * c101s; A[12] = r * c011s;
    A[5] = r * c210s; A[7] = r * c120s; A[11] = r * c201s;
    A[15] = r * c021s; A[19] = r * c102s; A[21] = r * c012s;
    A[13] = r * c111s;
    A[8] = r * c220s; A[20] = r * c202s; A[24] = r * c022s;
    A[14] = r * c211s; A[16] = r * c121s; A[22] = r * c112s;
    A[17] = r * c221s; A[23] = r * c212s; A[25] = r * c122s;
    A[26] = r * c222s;
    for (int mb = 0; mb < 3; ++mb)
      for (int ma = 0; ma < 3; ++ma) chim_b(A[ma + 3 * mb], A[ma + 3 * mb + 9], A[ma + 3 * mb + 18], uze);
    for (int iz = 0; iz < 3; ++iz)
      for (int ma = 0; ma < 3; ++ma) chim_b(A[ma + 9 * iz], A[ma + 3 + 9 * iz], A[ma + 6 + 9 * iz], uye);
    for (int iz = 0; iz < 3; ++iz)
      for (int iy = 0; iy < 3; ++iy) {
        int bse = 3 * iy + 9 * iz;
        chim_b(A[bse], A[bse + 1], A[bse + 2], uxe);
      }
    if (sp.limiter_type == 2) {
      R fmin_v = A[0];
      for (int k = 1; k < 27; ++k) fmin_v = rmin(fmin_v, A[k]);
      if (fmin_v < (R)0) {
        R alpha = 1;
        for (int k = 0; k < 27; ++k) {
          R fe = feq_auto(rho, uxe, uye, uze, wk<R>(k), (R)LAT.cx[k], (R)LAT.cy[k], (R)LAT.cz[k],
                          sp.compressible_corr);
          R fn = A[k] - fe;
          if (fn < (R)0 && fe > (R)1e-15) alpha = rmin(alpha, fe / (fe - fn + (R)1e-15));
        }
        alpha = rmax(alpha, (R)0);
        for (int k = 0; k < 27; ++k) {
          R fe = feq_auto(rho, uxe, uye, uze, wk<R>(k), (R)LAT.cx[k], (R)LAT.cy[k], (R)LAT.cz[k],
                          sp.compressible_corr);
          A[k] = fe + alpha * (A[k] - fe);
        }
      }
    }
  } else {
    R tau_t = tau_mol + nu_eddy * (R)3;
    om = (R)1 / rmax(tau_t, (R)0.500001);
    R Pxx = 0, Pyy = 0, Pzz = 0, Pxy = 0, Pyz = 0, Pzx = 0;
    for (int k = 0; k < 27; ++k) {
      R cx = (R)LAT.cx[k], cy = (R)LAT.cy[k], cz = (R)LAT.cz[k];
      R fe = feq_auto(rho, uxe, uye, uze, wk<R>(k), cx, cy, cz, sp.compressible_corr);
      R fn = fs[k] - fe;
      Pxx += fn * cx * cx; Pyy += fn * cy * cy; Pzz += fn * cz * cz;
      Pxy += fn * cx * cy; Pyz += fn * cy * cz; Pzx += fn * cz * cx;
    }
    const R cs2p = third_lit<R>();
    for (int k = 0; k < 27; ++k) {
      R cx = (R)LAT.cx[k], cy = (R)LAT.cy[k], cz = (R)LAT.cz[k], w = wk<R>(k);
      R fe = feq_auto(rho, uxe, uye, uze, w, cx, cy, cz, sp.compressible_corr);
      R Qxx = cx * cx - cs2p, Qyy = cy * cy - cs2p, Qzz = cz * cz - cs2p;
      R fr = w * (R)4.5 * (Pxx * Qxx + Pyy * Qyy + Pzz * Qzz + (R)2 * (Pxy * cx * cy + Pyz * cy * cz + Pzx * cz * cx));
      A[k] = fe + ((R)1 - om) * fr;
    }
  }
  // Guo forcing + store (kernel_cumulant.jl:604-623; BGK :292-321 with cu = c.u_eq)
  for (int k = 0; k < 27; ++k) {
    R cx = (R)LAT.cx[k], cy = (R)LAT.cy[k], cz = (R)LAT.cz[k], w = wk<R>(k);
    R cu = cx * uxe + cy * uye + cz * uze;
    R ft = w * (R)3 * ((cx - ux + (R)3 * cu * cx) * Fx + (cy - uy + (R)3 * cu * cy) * Fy +
                       (cz - uz + (R)3 * cu * cz) * Fz);
    R fc = A[k] + ((R)1 - (R)0.5 * om) * ft;
    if (post) L.f_post[own + k * S] = fc;
    L.f_out[own + k * S] = fc;
  }
}

template <class R>
void stream_collide(const Level<R> &L, const Parent<R> &P, const StepParams &sp) {
#pragma omp parallel for schedule(static)
  for (int b = 0; b < L.nB; ++b)
    for (int z = 1; z <= BS; ++z)
      for (int y = 1; y <= BS; ++y)
        for (int x = 1; x <= BS; ++x) cell_step(L, P, sp, b, x, y, z);
}

// binary16 bits -> float (IEEE round trip, exact)
inline float h2f(uint16_t h) {
  uint32_t s = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1f, m = h & 0x3ff, u;
  if (e == 0) {
    if (m == 0) u = s;
    else {
      int ee = -1;
      do { ++ee; m <<= 1; } while (!(m & 0x400));
      u = s | ((uint32_t)(127 - 15 - ee) << 23) | ((m & 0x3ff) << 13);
    }
  } else if (e == 31) {
    u = s | 0x7f800000u | (m << 13);
  } else {
    u = s | ((e + 127 - 15) << 23) | (m << 13);
  }
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// bouzidi_kernel.jl:13-92 (reads f_post, writes f_out)
template <class R>
void bouzidi(R *f_out, const R *f_post, const uint16_t *q, const int32_t *cb, const int8_t *cxl,
             const int8_t *cyl, const int8_t *czl, int nbnd, const int32_t *nbr, int nB, float qmin) {
  const size_t S = (size_t)NC * nB;
  for (int i = 0; i < nbnd; ++i) {
    int b = cb[i] - 1, x = cxl[i], y = cyl[i], z = czl[i];
    size_t own = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
    for (int k = 0; k < 27; ++k) {
      R qv = (R)h2f(q[own + k * S]);
      if (qv > (R)qmin && qv <= (R)1) {
        int ko = LAT.opp[k];
        R fk = f_post[own + k * S];
        if (qv < (R)0.5) {
          int nx = x + LAT.cx[ko], ny = y + LAT.cy[ko], nz = z + LAT.cz[ko];
          R fff = fk;
          if (nx >= 1 && nx <= BS && ny >= 1 && ny <= BS && nz >= 1 && nz <= BS) {
            fff = f_post[(size_t)b * NC + (nx - 1) + BS * (ny - 1) + BS * BS * (nz - 1) + k * S];
          } else {
            int ox = nx < 1 ? -1 : (nx > BS ? 1 : 0), oy = ny < 1 ? -1 : (ny > BS ? 1 : 0),
                oz = nz < 1 ? -1 : (nz > BS ? 1 : 0);
            int nb = nbr[b + (size_t)nB * ((ox + 1) + (oy + 1) * 3 + (oz + 1) * 9)];
            if (nb > 0) {
              int nnx = nx < 1 ? nx + BS : (nx > BS ? nx - BS : nx);
              int nny = ny < 1 ? ny + BS : (ny > BS ? ny - BS : ny);
              int nnz = nz < 1 ? nz + BS : (nz > BS ? nz - BS : nz);
              fff = f_post[(size_t)(nb - 1) * NC + (nnx - 1) + BS * (nny - 1) + BS * BS * (nnz - 1) + k * S];
            }
          }
          R c1 = (R)2 * qv;
          f_out[own + ko * S] = c1 * fk + ((R)1 - c1) * fff;
        } else {
          R fo = f_post[own + ko * S];
          R i2q = (R)1 / ((R)2 * qv);
          R c2 = ((R)2 * qv - (R)1) * i2q;
          f_out[own + ko * S] = i2q * fk + c2 * fo;
        }
      }
    }
  }
}

struct ThermalParams {  // mirrors ol_thermal_params
  float tau_g, tau_g_parent;
  int32_t is_level_1, is_symmetric, nx_global, ny_global, nz_global;
  float u_inlet, T_inlet, T_wall;
  int32_t wall_bc_adiabatic, store_post_collision;
  float temporal_weight;
  int32_t use_temporal_interp, sponge_blend_distributions;
};

// kernel_thermal.jl:14-202
template <class R>
void thermal(R *g_out, const R *g_in, R *g_post, R *T_out, const R *vel, const uint8_t *obs,
             const float *sponge, const int32_t *nbr, const int32_t *mx, const int32_t *my,
             const int32_t *mz, int nB, const Parent<R> &P, const ThermalParams &tp) {
  const size_t S = (size_t)NC * nB;
  const bool post = tp.store_post_collision == 1 && g_post;
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nB; ++b)
    for (int z = 1; z <= BS; ++z)
      for (int y = 1; y <= BS; ++y)
        for (int x = 1; x <= BS; ++x) {
          size_t own = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
          int gx = (mx[b] - 1) * BS + x, gy = (my[b] - 1) * BS + y, gz = (mz[b] - 1) * BS + z;
          bool is_obs = obs[own] != 0;
          R ux = vel[own], uy = vel[own + S], uz = vel[own + 2 * S];
          R Tsum = 0;
          R gs[27];
          for (int k = 0; k < 27; ++k) {
            int cx = LAT.cx[k], cy = LAT.cy[k], cz = LAT.cz[k];
            int sx = x - cx, sy = y - cy, sz = z - cz;
            R val = 0;
            if (sx >= 1 && sx <= BS && sy >= 1 && sy <= BS && sz >= 1 && sz <= BS) {
              val = g_in[(size_t)b * NC + (sx - 1) + BS * (sy - 1) + BS * BS * (sz - 1) + k * S];
            } else {
              int ox = sx < 1 ? -1 : (sx > BS ? 1 : 0), oy = sy < 1 ? -1 : (sy > BS ? 1 : 0),
                  oz = sz < 1 ? -1 : (sz > BS ? 1 : 0);
              int nb = nbr[b + (size_t)nB * ((ox + 1) + (oy + 1) * 3 + (oz + 1) * 9)];
              if (nb > 0) {
                int nsx = sx < 1 ? sx + BS : (sx > BS ? sx - BS : sx);
                int nsy = sy < 1 ? sy + BS : (sy > BS ? sy - BS : sy);
                int nsz = sz < 1 ? sz + BS : (sz > BS ? sz - BS : sz);
                val = g_in[(size_t)(nb - 1) * NC + (nsx - 1) + BS * (nsy - 1) + BS * BS * (nsz - 1) + k * S];
              } else {
                int sgx = gx - cx, sgy = gy - cy, sgz = gz - cz;
                if (sgx < 1 || sgx > tp.nx_global) {
                  val = geq((R)tp.T_inlet, (R)tp.u_inlet, (R)0, (R)0, wk<R>(k), (R)cx, (R)cy, (R)cz);
                } else if (sgy < 1 || sgy > tp.ny_global) {
                  val = g_in[own + LAT.my[k] * S];
                } else if (sgz < 1 || sgz > tp.nz_global) {
                  val = g_in[own + LAT.mz[k] * S];
                } else if (tp.is_level_1 == 0) {
                  val = interpolate(P, sgx, sgy, sgz, k, wk<R>(k), (R)cx, (R)cy, (R)cz,
                                    (R)tp.tau_g_parent, (R)tp.tau_g, (R)tp.temporal_weight,
                                    tp.use_temporal_interp, 0, true);
                } else {
                  val = wk<R>(k) * (R)tp.T_inlet;
                }
              }
            }
            Tsum += val;
            if (is_obs) {
              R go;
              if (tp.wall_bc_adiabatic == 1) {
                go = g_in[own + LAT.opp[k] * S];
              } else {
                R gw = geq((R)tp.T_wall, (R)0, (R)0, (R)0, wk<R>(k), (R)cx, (R)cy, (R)cz);
                go = (R)2 * gw - g_in[own + LAT.opp[k] * S];
              }
              g_out[own + k * S] = go;
              if (post) g_post[own + k * S] = go;
            } else {
              gs[k] = val;
            }
          }
          if (is_obs) {
            T_out[own] = tp.wall_bc_adiabatic == 1 ? Tsum : (R)tp.T_wall;
            continue;
          }
          R Tl = rmax(Tsum, (R)0.01);
          R spg = (R)sponge[own];
          if (spg > (R)0) {
            Tl = Tl * ((R)1 - spg) + (R)tp.T_inlet * spg;
            ux = ux * ((R)1 - spg) + (R)tp.u_inlet * spg;
            uy = uy * ((R)1 - spg);
            uz = uz * ((R)1 - spg);
          }
          T_out[own] = Tl;
          R og = (R)1 / rmax((R)tp.tau_g, (R)0.500001);
          for (int k = 0; k < 27; ++k) {
            R cx = (R)LAT.cx[k], cy = (R)LAT.cy[k], cz = (R)LAT.cz[k];
            R g = gs[k];
            if (spg > (R)0 && tp.sponge_blend_distributions == 1) {
              R gt = geq((R)tp.T_inlet, (R)tp.u_inlet, (R)0, (R)0, wk<R>(k), cx, cy, cz);
              g = g * ((R)1 - spg) + gt * spg;
            }
            R ge = geq(Tl, ux, uy, uz, wk<R>(k), cx, cy, cz);
            R gc = g - og * (g - ge);
            if (post) g_post[own + k * S] = gc;
            g_out[own + k * S] = gc;
          }
        }
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
        if (LAT.cx[k] == 1) jx = jx + fbar[k]; else if (LAT.cx[k] == -1) jx = jx - fbar[k];   \
        if (LAT.cy[k] == 1) jy = jy + fbar[k]; else if (LAT.cy[k] == -1) jy = jy - fbar[k];   \
        if (LAT.cz[k] == 1) jz = jz + fbar[k]; else if (LAT.cz[k] == -1) jz = jz - fbar[k];   \
      }                                                                                       \
      const R ux = jx / rho, uy = jy / rho, uz = jz / rho;                                    \
      const R tf = (R)tau_f - (R)0.5, tc = (R)tau_c - (R)0.5;                                 \
      const R sc = tf > (R)1e-6f ? rclamp(tc / tf, (R)0.01f, (R)100.0f) : (R)1;               \
      for (int k = 0; k < 27; ++k) {                                                          \
        const R fe = feq_auto(rho, ux, uy, uz, wk<R>(k), (R)LAT.cx[k], (R)LAT.cy[k],          \
                              (R)LAT.cz[k], comp);                                            \
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
