/*
 * ol_oracle_cell.h -- the oracle's per-cell restatement of the reference's
 * device kernels (stream-collide, Bouzidi, thermal DDF, coarse-to-fine
 * interpolation), shared by the CPU loops of ol_oracle_kernels.cpp and the
 * one-thread-per-cell GPU loops of ol_oracle_gpu.cu.
 *
 * TEST INFRASTRUCTURE (see ol_oracle_kernels.cpp).  Written for g++ with
 * -ffp-contract=off; under nvcc the functions are also device functions
 * (ORC_HD), built with --fmad=false so products and sums round as written.
 */
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define ORC_HD __host__ __device__
#else
#define ORC_HD
#endif

namespace orc {

constexpr int BS = 8, NC = 512, Q = 27;

// lattice.jl:5-56 / timestep.jl:161-179 (k-order: x fastest): k = (cx+1) + 3 (cy+1) + 9 (cz+1)
ORC_HD inline int lat_cx(int k) { return k % 3 - 1; }
ORC_HD inline int lat_cy(int k) { return (k / 3) % 3 - 1; }
ORC_HD inline int lat_cz(int k) { return k / 9 - 1; }
ORC_HD inline int lat_opp(int k) { return 26 - k; }                 // -c
ORC_HD inline int lat_my(int k) { return k - 6 * lat_cy(k); }       // (cx, -cy, cz)
ORC_HD inline int lat_mz(int k) { return k - 18 * lat_cz(k); }      // (cx, cy, -cz)
ORC_HD inline int lat_d2(int k) {
  return lat_cx(k) * lat_cx(k) + lat_cy(k) * lat_cy(k) + lat_cz(k) * lat_cz(k);
}
// Float32 weights, the reference's Float32 quotients
ORC_HD inline float lat_wf(int k) {
  const int d2 = lat_d2(k);
  return d2 == 0 ? 8.0f / 27.0f : d2 == 1 ? 2.0f / 27.0f : d2 == 2 ? 1.0f / 54.0f : 1.0f / 216.0f;
}

// Weights: the Float32 quotients of the reference for float; exact quotients
// for the double (accuracy-oracle) instantiation.
template <class R> ORC_HD inline R wk(int k) { return (R)lat_wf(k); }
template <> ORC_HD inline double wk<double>(int k) {
  const int d2 = lat_d2(k);
  return d2 == 0 ? 8.0 / 27.0 : d2 == 1 ? 2.0 / 27.0 : d2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
}
// c_s^2: the reference's literal 0.333333333f0 (kernel_cumulant.jl:420); exact for double.
template <class R> ORC_HD inline R cs2_lit() { return (R)0.333333333f; }
template <> ORC_HD inline double cs2_lit<double>() { return 1.0 / 3.0; }
template <class R> ORC_HD inline R third_lit() { return (R)(1.0f / 3.0f); }
template <> ORC_HD inline double third_lit<double>() { return 1.0 / 3.0; }
template <class R> ORC_HD inline R rmax(R a, R b) { return a > b ? a : b; }
template <class R> ORC_HD inline R rmin(R a, R b) { return a < b ? a : b; }
template <class R> ORC_HD inline R rclamp(R x, R lo, R hi) { return x > hi ? hi : (x < lo ? lo : x); }

// physics_utils.jl:19-24
template <class R>
ORC_HD R feq(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz) {
  R cu = cx * ux + cy * uy + cz * uz;
  R usq = ux * ux + uy * uy + uz * uz;
  return rho * w * ((R)1 + (R)3 * cu + (R)4.5 * cu * cu - (R)1.5 * usq);
}
// physics_utils.jl:39-61
template <class R>
ORC_HD R feq_comp(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz) {
  R cu = cx * ux + cy * uy + cz * uz;
  R usq = ux * ux + uy * uy + uz * uz;
  R cu2 = cu * cu, cu3 = cu2 * cu, cu4 = cu2 * cu2, usq2 = usq * usq;
  R val = (R)1 + (R)3 * cu + (R)4.5 * cu2 - (R)1.5 * usq;
  val += (R)4.5 * cu3 - (R)4.5 * cu * usq;
  val += (R)3.375 * cu4 - (R)6.75 * cu2 * usq + (R)1.125 * usq2;
  return rho * w * val;
}
template <class R>
ORC_HD R feq_auto(R rho, R ux, R uy, R uz, R w, R cx, R cy, R cz, int comp) {
  return comp == 1 ? feq_comp(rho, ux, uy, uz, w, cx, cy, cz) : feq(rho, ux, uy, uz, w, cx, cy, cz);
}
// physics_utils.jl:78-83
template <class R>
ORC_HD R geq(R T, R ux, R uy, R uz, R w, R cx, R cy, R cz) {
  R cu = cx * ux + cy * uy + cz * uz;
  return w * T * ((R)1 + (R)3 * cu);
}
// physics_utils.jl:5-17
ORC_HD inline uint32_t gpu_hash(int32_t x) {
  uint32_t h = (uint32_t)x;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  return h ^ (h >> 16);
}
ORC_HD inline float gradient_noise(int32_t gx, int32_t gy, int32_t gz, int32_t seed) {
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
ORC_HD R interpolate(const Parent<R> &P, int fgx, int fgy, int fgz, int k, R w, R cx, R cy, R cz,
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
    if (!ok[s])
      for (int i = 0; i < 5; ++i) d[s][i] = d[0][i];
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
ORC_HD void vel_nb(const Level<R> &L, int x, int y, int z, int b, int dx, int dy, int dz, R &ux, R &uy,
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
ORC_HD inline void chim_f(R &a, R &b, R &c, R u) {
  R m0 = a + b + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = m1 - u * m0;
  c = m2 - (R)2 * u * m1 + u * u * m0;
}
template <class R>
ORC_HD inline void chim_b(R &a, R &b, R &c, R u) {
  R m0 = a, m1 = b + u * a, m2 = c + (R)2 * u * b + u * u * a;
  R fp = (m2 + m1) * (R)0.5, fm = (m2 - m1) * (R)0.5, f0 = m0 - m2;
  a = fm; b = f0; c = fp;
}

// kernel_cumulant.jl:29-627 and kernel_regularized_bgk.jl:4-325 (op == 1),
// one cell (x, y, z 1-based; b 0-based).
template <class R>
ORC_HD void cell_step(const Level<R> &L, const Parent<R> &P, const StepParams &sp, int b, int x, int y,
               int z) {
  const size_t S = (size_t)NC * L.nB;
  const size_t own = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
  const int gx = (L.mx[b] - 1) * BS + x, gy = (L.my[b] - 1) * BS + y, gz = (L.mz[b] - 1) * BS + z;
  const bool is_obs = L.obstacle[own] != 0;
  const R u_in = (R)sp.u_inlet;
  R rho = 0, jx = 0, jy = 0, jz = 0;
  R fs[27];
  for (int k = 0; k < 27; ++k) {
    int cx = lat_cx(k), cy = lat_cy(k), cz = lat_cz(k);
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
          val = L.f_in[own + lat_my(k) * S];
        } else if (sgz < 1 || sgz > sp.nz_global) {
          val = L.f_in[own + lat_mz(k) * S];
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
      R fc = fs[lat_opp(k)];
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
        R ft = feq_auto(rho_t, ux_t, (R)0, (R)0, wk<R>(k), (R)lat_cx(k), (R)lat_cy(k), (R)lat_cz(k),
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
          R fe = feq_auto(rho, uxe, uye, uze, wk<R>(k), (R)lat_cx(k), (R)lat_cy(k), (R)lat_cz(k),
                          sp.compressible_corr);
          R fn = A[k] - fe;
          if (fn < (R)0 && fe > (R)1e-15) alpha = rmin(alpha, fe / (fe - fn + (R)1e-15));
        }
        alpha = rmax(alpha, (R)0);
        for (int k = 0; k < 27; ++k) {
          R fe = feq_auto(rho, uxe, uye, uze, wk<R>(k), (R)lat_cx(k), (R)lat_cy(k), (R)lat_cz(k),
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
      R cx = (R)lat_cx(k), cy = (R)lat_cy(k), cz = (R)lat_cz(k);
      R fe = feq_auto(rho, uxe, uye, uze, wk<R>(k), cx, cy, cz, sp.compressible_corr);
      R fn = fs[k] - fe;
      Pxx += fn * cx * cx; Pyy += fn * cy * cy; Pzz += fn * cz * cz;
      Pxy += fn * cx * cy; Pyz += fn * cy * cz; Pzx += fn * cz * cx;
    }
    const R cs2p = third_lit<R>();
    for (int k = 0; k < 27; ++k) {
      R cx = (R)lat_cx(k), cy = (R)lat_cy(k), cz = (R)lat_cz(k), w = wk<R>(k);
      R fe = feq_auto(rho, uxe, uye, uze, w, cx, cy, cz, sp.compressible_corr);
      R Qxx = cx * cx - cs2p, Qyy = cy * cy - cs2p, Qzz = cz * cz - cs2p;
      R fr = w * (R)4.5 * (Pxx * Qxx + Pyy * Qyy + Pzz * Qzz + (R)2 * (Pxy * cx * cy + Pyz * cy * cz + Pzx * cz * cx));
      A[k] = fe + ((R)1 - om) * fr;
    }
  }
  // Guo forcing + store (kernel_cumulant.jl:604-623; BGK :292-321 with cu = c.u_eq)
  for (int k = 0; k < 27; ++k) {
    R cx = (R)lat_cx(k), cy = (R)lat_cy(k), cz = (R)lat_cz(k), w = wk<R>(k);
    R cu = cx * uxe + cy * uye + cz * uze;
    R ft = w * (R)3 * ((cx - ux + (R)3 * cu * cx) * Fx + (cy - uy + (R)3 * cu * cy) * Fy +
                       (cz - uz + (R)3 * cu * cz) * Fz);
    R fc = A[k] + ((R)1 - (R)0.5 * om) * ft;
    if (post) L.f_post[own + k * S] = fc;
    L.f_out[own + k * S] = fc;
  }
}

// binary16 bits -> float (IEEE round trip, exact)
ORC_HD inline float h2f(uint16_t h) {
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
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}


// bouzidi_kernel.jl:13-92, boundary cell i (reads f_post, writes f_out)
template <class R>
ORC_HD void bouzidi_cell(R *f_out, const R *f_post, const uint16_t *q, const int32_t *cb,
                         const int8_t *cxl, const int8_t *cyl, const int8_t *czl, int i,
                         const int32_t *nbr, int nB, float qmin) {
  const size_t S = (size_t)NC * nB;
  int b = cb[i] - 1, x = cxl[i], y = cyl[i], z = czl[i];
  size_t own = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
  for (int k = 0; k < 27; ++k) {
    R qv = (R)h2f(q[own + k * S]);
    if (qv > (R)qmin && qv <= (R)1) {
      int ko = lat_opp(k);
      R fk = f_post[own + k * S];
      if (qv < (R)0.5) {
        int nx = x + lat_cx(ko), ny = y + lat_cy(ko), nz = z + lat_cz(ko);
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

struct ThermalParams {  // mirrors ol_thermal_params
  float tau_g, tau_g_parent;
  int32_t is_level_1, is_symmetric, nx_global, ny_global, nz_global;
  float u_inlet, T_inlet, T_wall;
  int32_t wall_bc_adiabatic, store_post_collision;
  float temporal_weight;
  int32_t use_temporal_interp, sponge_blend_distributions;
};


// kernel_thermal.jl:14-202, one cell (x, y, z 1-based; b 0-based)
template <class R>
ORC_HD void thermal_cell(R *g_out, const R *g_in, R *g_post, R *T_out, const R *vel,
                         const uint8_t *obs, const float *sponge, const int32_t *nbr,
                         const int32_t *mx, const int32_t *my, const int32_t *mz, int nB,
                         const Parent<R> &P, const ThermalParams &tp, int b, int x, int y, int z) {
  const size_t S = (size_t)NC * nB;
  const bool post = tp.store_post_collision == 1 && g_post;
  size_t own = (size_t)b * NC + (x - 1) + BS * (y - 1) + BS * BS * (z - 1);
  int gx = (mx[b] - 1) * BS + x, gy = (my[b] - 1) * BS + y, gz = (mz[b] - 1) * BS + z;
  bool is_obs = obs[own] != 0;
  R ux = vel[own], uy = vel[own + S], uz = vel[own + 2 * S];
  R Tsum = 0;
  R gs[27];
  for (int k = 0; k < 27; ++k) {
    int cx = lat_cx(k), cy = lat_cy(k), cz = lat_cz(k);
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
          val = g_in[own + lat_my(k) * S];
        } else if (sgz < 1 || sgz > tp.nz_global) {
          val = g_in[own + lat_mz(k) * S];
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
        go = g_in[own + lat_opp(k) * S];
      } else {
        R gw = geq((R)tp.T_wall, (R)0, (R)0, (R)0, wk<R>(k), (R)cx, (R)cy, (R)cz);
        go = (R)2 * gw - g_in[own + lat_opp(k) * S];
      }
      g_out[own + k * S] = go;
      if (post) g_post[own + k * S] = go;
    } else {
      gs[k] = val;
    }
  }
  if (is_obs) {
    T_out[own] = tp.wall_bc_adiabatic == 1 ? Tsum : (R)tp.T_wall;
    return;
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
    R cx = (R)lat_cx(k), cy = (R)lat_cy(k), cz = (R)lat_cz(k);
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

}  // namespace orc
