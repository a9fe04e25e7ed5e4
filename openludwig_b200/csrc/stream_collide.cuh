// Fused pull-stream + collision for one 8^3 block per CTA (one cell per
// thread).  Cell stages follow kernel_cumulant.jl:70-627 and
// kernel_regularized_bgk.jl:43-325 in the same order:
//   pull + domain BCs -> obstacle bounce-back -> rho, u, sponge -> wall
//   model -> store u, rho -> WALE -> collision -> Guo forcing + store.
// The block's pull windows are staged in shared memory first (stage_block),
// rare paths (domain boundaries, level interfaces) fill their slots during
// that staging, and the per-cell path has no call sites and no
// address-taken arrays; the 27-direction loops are fully unrolled so every
// lattice constant folds.
#pragma once
#include "level_dev.cuh"

namespace ol {

// ---------------------------------------------------------------------------
// Coarse-to-fine ghost value (physics_interpolation.jl:4-127).
// gx, gy, gz: 1-based fine-level global source coordinates.
// ---------------------------------------------------------------------------
template <class ST>
__device__ __noinline__ float interp_parent(const LevelDev &L, int k, int gx,
                                            int gy, int gz) {
  const ol_step_params &sp = L.sp;
  const float w = w_of(k);
  const float cx = (float)cx_of(k), cy = (float)cy_of(k), cz = (float)cz_of(k);
  const float pxc = ((float)gx - 0.5f) * 0.5f;
  const float pyc = ((float)gy - 0.5f) * 0.5f;
  const float pzc = ((float)gz - 0.5f) * 0.5f;
  int px0 = (int)floorf(pxc), py0 = (int)floorf(pyc), pz0 = (int)floorf(pzc);
  const int px1 = px0 + 1, py1 = py0 + 1, pz1 = pz0 + 1;
  const float wx = pxc - (float)px0, wy = pyc - (float)py0, wz = pzc - (float)pz0;
  px0 = max(1, px0); py0 = max(1, py0); pz0 = max(1, pz0);

  const bool temporal = sp.use_temporal_interp == 1 && sp.temporal_weight < 0.99f;
  const float tw = sp.temporal_weight;
  float v[8][5];
  bool ok[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int pgx = (s & 1) ? px1 : px0;
    const int pgy = (s & 2) ? py1 : py0;
    const int pgz = (s & 4) ? pz1 : pz0;
    const int pbx = (pgx - 1) / BS + 1, pby = (pgy - 1) / BS + 1, pbz = (pgz - 1) / BS + 1;
    ok[s] = false;
    v[s][0] = w; v[s][1] = 1.0f; v[s][2] = 0.0f; v[s][3] = 0.0f; v[s][4] = 0.0f;
    if (pbx >= 1 && pbx <= L.pdim_x && pby >= 1 && pby <= L.pdim_y && pbz >= 1 &&
        pbz <= L.pdim_z) {
      const int pb = L.pptr[(pbx - 1) + L.pdim_x * ((pby - 1) + L.pdim_y * (pbz - 1))];
      if (pb > 0) {
        const int cell = (pgx - 1) % BS + BS * ((pgy - 1) % BS) + BS * BS * ((pgz - 1) % BS);
        const size_t ci = (size_t)(L.p_block_offset + pb - 1) * BCELLS + cell;
        const float fn = ST::load((const typename ST::T *)L.pf, ci + (size_t)k * L.p_dstride,
                                  k, L.p_inv_scale);
        const float rn = L.prho[ci];
        const float uxn = L.pvel[ci], uyn = L.pvel[ci + L.p_dstride],
                    uzn = L.pvel[ci + 2 * L.p_dstride];
        if (temporal) {
          const float fo = ST::load((const typename ST::T *)L.pf_old,
                                    ci + (size_t)k * L.p_dstride, k, L.p_inv_scale);
          const float ro = L.prho_old[ci];
          const float uxo = L.pvel_old[ci], uyo = L.pvel_old[ci + L.p_dstride],
                      uzo = L.pvel_old[ci + 2 * L.p_dstride];
          v[s][0] = fo * (1.0f - tw) + fn * tw;
          v[s][1] = ro * (1.0f - tw) + rn * tw;
          v[s][2] = uxo * (1.0f - tw) + uxn * tw;
          v[s][3] = uyo * (1.0f - tw) + uyn * tw;
          v[s][4] = uzo * (1.0f - tw) + uzn * tw;
        } else {
          v[s][0] = fn; v[s][1] = rn; v[s][2] = uxn; v[s][3] = uyn; v[s][4] = uzn;
        }
        ok[s] = true;
      }
    }
  }
  // Missing samples fall back to the (possibly missing) first corner.
#pragma unroll
  for (int s = 1; s < 8; ++s)
    if (!ok[s])
#pragma unroll
      for (int i = 0; i < 5; ++i) v[s][i] = v[0][i];
  float r[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const float c00 = v[0][i] * (1.0f - wx) + v[1][i] * wx;
    const float c01 = v[4][i] * (1.0f - wx) + v[5][i] * wx;
    const float c10 = v[2][i] * (1.0f - wx) + v[3][i] * wx;
    const float c11 = v[6][i] * (1.0f - wx) + v[7][i] * wx;
    const float c0 = c00 * (1.0f - wy) + c10 * wy;
    const float c1 = c01 * (1.0f - wy) + c11 * wy;
    r[i] = c0 * (1.0f - wz) + c1 * wz;
  }
  const float fe = feq_auto(r[1], r[2], r[3], r[4], w, cx, cy, cz, sp.compressible_corr);
  const float fneq = r[0] - fe;
  const float tc = sp.tau_parent - 0.5f, tf = sp.tau_molecular - 0.5f;
  const float sc = tc > 1e-6f ? fminf(fmaxf(tf / tc, 0.01f), 100.0f) : 1.0f;
  return fe + fneq * sc;
}

// ---------------------------------------------------------------------------
// Source value of a pull whose neighbour block is absent
// (kernel_cumulant.jl:117-159).  x, y, z are 0-based local coordinates.
// ---------------------------------------------------------------------------
template <class ST>
__device__ __noinline__ float pull_boundary(const LevelDev &L, int k, int b,
                                            int x, int y, int z) {
  const ol_step_params &sp = L.sp;
  const int cx = cx_of(k), cy = cy_of(k), cz = cz_of(k);
  const int gx = (L.map_x[b] - 1) * BS + x + 1;
  const int gy = (L.map_y[b] - 1) * BS + y + 1;
  const int gz = (L.map_z[b] - 1) * BS + z + 1;
  const int sgx = gx - cx, sgy = gy - cy, sgz = gz - cz;
  const float w = w_of(k);
  if (sgx < 1) {
    const float noise = sp.inlet_turbulence > 0.0f
                            ? gradient_noise(gy, gz, sp.time_step_seed, 1234) *
                                  sp.inlet_turbulence * sp.u_inlet
                            : 0.0f;
    return feq_auto(1.0f, sp.u_inlet + noise, 0.0f, 0.0f, w, (float)cx, (float)cy,
                    (float)cz, sp.compressible_corr);
  }
  if (sgx > sp.nx_global)
    return feq_auto(1.0f, sp.u_inlet, 0.0f, 0.0f, w, (float)cx, (float)cy,
                    (float)cz, sp.compressible_corr);
  const size_t ci = (size_t)(L.block_offset + b) * BCELLS + x + BS * y + BS * BS * z;
  if (sgy < 1 || sgy > sp.ny_global) {
    const int km = mirror_y_of(k);
    return ST::load((const typename ST::T *)L.f_in, ci + (size_t)km * L.dstride, km,
                    L.inv_scale);
  }
  if (sgz < 1 || sgz > sp.nz_global) {
    const int km = mirror_z_of(k);
    return ST::load((const typename ST::T *)L.f_in, ci + (size_t)km * L.dstride, km,
                    L.inv_scale);
  }
  if (sp.is_level_1 == 0) return interp_parent<ST>(L, k, sgx, sgy, sgz);
  return w;
}

// ---------------------------------------------------------------------------
// WALE eddy viscosity from vel_in central differences
// (kernel_cumulant.jl:264-305, physics_utils.jl:85-123).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void vel_neighbor(const LevelDev &L, const int *nbbase,
                                             int x, int y, int z, int dx,
                                             int dy, int dz, float &ux, float &uy,
                                             float &uz) {
  int nx = x + dx, ny = y + dy, nz = z + dz;
  const int ox = nx < 0 ? -1 : (nx > 7 ? 1 : 0);
  const int oy = ny < 0 ? -1 : (ny > 7 ? 1 : 0);
  const int oz = nz < 0 ? -1 : (nz > 7 ? 1 : 0);
  const int nb = nbbase[(ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
  size_t ci;
  if (nb >= 0) {
    ci = (size_t)nb + (nx & 7) + BS * (ny & 7) + BS * BS * (nz & 7);
  } else {
    ci = (size_t)nbbase[13] + x + BS * y + BS * BS * z;
  }
  ux = __ldg(L.vel_in + ci);
  uy = __ldg(L.vel_in + ci + L.dstride);
  uz = __ldg(L.vel_in + ci + 2 * L.dstride);
}

__device__ __forceinline__ float wale_nu(const LevelDev &L, const int *nbbase, int x, int y,
                                         int z) {
  float exx, eyx, ezx, wxx, wyx, wzx;  // E (x+1), W (x-1)
  float nxx, nyx, nzx, sxx, syx, szx;  // N (y+1), S (y-1)
  float txx, tyx, tzx, bxx, byx, bzx;  // T (z+1), B (z-1)
  vel_neighbor(L, nbbase, x, y, z, 1, 0, 0, exx, eyx, ezx);
  vel_neighbor(L, nbbase, x, y, z, -1, 0, 0, wxx, wyx, wzx);
  vel_neighbor(L, nbbase, x, y, z, 0, 1, 0, nxx, nyx, nzx);
  vel_neighbor(L, nbbase, x, y, z, 0, -1, 0, sxx, syx, szx);
  vel_neighbor(L, nbbase, x, y, z, 0, 0, 1, txx, tyx, tzx);
  vel_neighbor(L, nbbase, x, y, z, 0, 0, -1, bxx, byx, bzx);
  const float g11 = 0.5f * (exx - wxx), g12 = 0.5f * (nxx - sxx), g13 = 0.5f * (txx - bxx);
  const float g21 = 0.5f * (eyx - wyx), g22 = 0.5f * (nyx - syx), g23 = 0.5f * (tyx - byx);
  const float g31 = 0.5f * (ezx - wzx), g32 = 0.5f * (nzx - szx), g33 = 0.5f * (tzx - bzx);

  const float gsq11 = g11 * g11 + g12 * g21 + g13 * g31;
  const float gsq12 = g11 * g12 + g12 * g22 + g13 * g32;
  const float gsq13 = g11 * g13 + g12 * g23 + g13 * g33;
  const float gsq21 = g21 * g11 + g22 * g21 + g23 * g31;
  const float gsq22 = g21 * g12 + g22 * g22 + g23 * g32;
  const float gsq23 = g21 * g13 + g22 * g23 + g23 * g33;
  const float gsq31 = g31 * g11 + g32 * g21 + g33 * g31;
  const float gsq32 = g31 * g12 + g32 * g22 + g33 * g32;
  const float gsq33 = g31 * g13 + g32 * g23 + g33 * g33;
  const float tr_term = (gsq11 + gsq22 + gsq33) / 3.0f;
  const float Sd11 = gsq11 - tr_term, Sd22 = gsq22 - tr_term, Sd33 = gsq33 - tr_term;
  const float Sd12 = 0.5f * (gsq12 + gsq21), Sd13 = 0.5f * (gsq13 + gsq31),
              Sd23 = 0.5f * (gsq23 + gsq32);
  const float S12 = 0.5f * (g12 + g21), S13 = 0.5f * (g13 + g31), S23 = 0.5f * (g23 + g32);
  const float OP1 = Sd11 * Sd11 + Sd22 * Sd22 + Sd33 * Sd33 +
                    2.0f * (Sd12 * Sd12 + Sd13 * Sd13 + Sd23 * Sd23);
  const float OP2 = g11 * g11 + g22 * g22 + g33 * g33 +
                    2.0f * (S12 * S12 + S13 * S13 + S23 * S23);
  float nu = 0.0f;
  if (OP1 > 1e-12f) {
    const float op1_32 = OP1 * sqrtf(OP1);
    const float op2_52 = OP2 * OP2 * sqrtf(fmaxf(OP2, 1e-12f));
    const float den = op2_52 + OP1 * sqrtf(sqrtf(fmaxf(OP1, 1e-12f)));
    if (den > 1e-12f) nu = (L.sp.c_wale * L.sp.c_wale) * op1_32 / den;
  }
  return nu;
}

// ---------------------------------------------------------------------------
// Wall-model force (kernel_cumulant.jl:220-250).  dist is in the units the
// wall-distance array carries (metres in the reference, domain_generation.jl:421).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void wall_force(float dist, float rho, float ux, float uy,
                                           float uz, float tau_mol, float &Fx, float &Fy,
                                           float &Fz) {
  Fx = Fy = Fz = 0.0f;
  if (!(dist > 0.0f && dist < 10.0f)) return;
  const float umag = sqrtf(ux * ux + uy * uy + uz * uz);
  const float nu = (tau_mol - 0.5f) / 3.0f;
  if (!(umag > 1e-6f && nu > 1e-10f)) return;
  float ut = umag * powf(nu / (dist * umag + 1e-10f), 1.0f / 7.0f) *
             powf(2.0f * 8.3f, -1.0f / 7.0f);
  ut = fmaxf(ut, 1e-6f);
  const float yp = ut * dist / nu;
  if (yp > 11.81f) {
    const float uplus = (1.0f / 0.41f) * logf(yp) + 5.2f;
    if (uplus > 0.1f) {
      ut = ut * ((umag / ut) / uplus);
      ut = fmaxf(ut, 1e-6f);
    }
  }
  const float tw = rho * ut * ut;
  const float tr = rho * nu * (umag / dist);
  if (tw > tr) {
    const float fm = (tw - tr) / dist;
    Fx = -fm * ux / umag;
    Fy = -fm * uy / umag;
    Fz = -fm * uz / umag;
  }
}

// ---------------------------------------------------------------------------
// Chimera transforms (kernel_cumulant.jl:4-26) and the cumulant collision
// (kernel_cumulant.jl:330-559).  A holds populations on entry and on exit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void chim_fwd(float &a, float &b, float &c, float u) {
  const float m0 = a + b + c, m1 = c - a, m2 = a + c;
  a = m0;
  b = m1 - u * m0;
  c = m2 - 2.0f * u * m1 + u * u * m0;
}
__device__ __forceinline__ void chim_bwd(float &a, float &b, float &c, float u) {
  const float m0 = a, m1 = b + u * a, m2 = c + 2.0f * u * b + u * u * a;
  c = (m2 + m1) * 0.5f;
  a = (m2 - m1) * 0.5f;
  b = m0 - m2;
}

struct CumulantRates {
  float omega1, omega_bulk, omega3, omega4, omega4_diag;
  int limiter;
};

__device__ __forceinline__ void collide_cumulant(float A[27], float ux, float uy,
                                                 float uz, const CumulantRates &r) {
  // forward: x (consecutive triples), then y (stride 3), then z (stride 9)
#pragma unroll
  for (int i = 0; i < 9; ++i) chim_fwd(A[3 * i], A[3 * i + 1], A[3 * i + 2], ux);
#pragma unroll
  for (int zz = 0; zz < 3; ++zz)
#pragma unroll
    for (int a = 0; a < 3; ++a)
      chim_fwd(A[a + 9 * zz], A[a + 3 + 9 * zz], A[a + 6 + 9 * zz], uy);
#pragma unroll
  for (int i = 0; i < 9; ++i) chim_fwd(A[i], A[i + 9], A[i + 18], uz);

  const float k000 = A[0];
  const float inv_r = 1.0f / fmaxf(k000, 0.01f);
  // index of central moment (a,b,c) = a + 3b + 9c
  const float c200 = A[2] * inv_r, c020 = A[6] * inv_r, c002 = A[18] * inv_r;
  const float c110 = A[4] * inv_r, c101 = A[10] * inv_r, c011 = A[12] * inv_r;
  const float c210 = A[5] * inv_r, c120 = A[7] * inv_r, c201 = A[11] * inv_r;
  const float c021 = A[15] * inv_r, c102 = A[19] * inv_r, c012 = A[21] * inv_r;
  const float c111 = A[13] * inv_r;
  const float c220n = A[8] * inv_r, c202n = A[20] * inv_r, c022n = A[24] * inv_r;
  const float c211n = A[14] * inv_r, c121n = A[16] * inv_r, c112n = A[22] * inv_r;

  const float C220 = c220n - c200 * c020 - 2.0f * c110 * c110;
  const float C202 = c202n - c200 * c002 - 2.0f * c101 * c101;
  const float C022 = c022n - c020 * c002 - 2.0f * c011 * c011;
  const float C211 = c211n - c200 * c011 - 2.0f * c110 * c101;
  const float C121 = c121n - c020 * c101 - 2.0f * c110 * c011;
  const float C112 = c112n - c002 * c110 - 2.0f * c101 * c011;

  const float cs2 = 0.333333333f;
  const float om1 = r.omega1, omb = r.omega_bulk;
  const float Dtr = c200 + c020 + c002;
  const float Dtr_s = (1.0f - omb) * Dtr + omb * (3.0f * cs2);
  const float D1s = (1.0f - om1) * (c200 - c020);
  const float D2s = (1.0f - om1) * (c200 - c002);
  const float c200s = (Dtr_s + D1s + D2s) / 3.0f;
  const float c020s = (Dtr_s - 2.0f * D1s + D2s) / 3.0f;
  const float c002s = (Dtr_s + D1s - 2.0f * D2s) / 3.0f;
  float c110s = (1.0f - om1) * c110;
  float c101s = (1.0f - om1) * c101;
  float c011s = (1.0f - om1) * c011;
  if (r.limiter == OL_LIMITER_FACTORED) {
    const float b110 = sqrtf(fmaxf(c200s * c020s, 0.0f));
    const float b101 = sqrtf(fmaxf(c200s * c002s, 0.0f));
    const float b011 = sqrtf(fmaxf(c020s * c002s, 0.0f));
    c110s = fminf(fmaxf(c110s, -b110), b110);
    c101s = fminf(fmaxf(c101s, -b101), b101);
    c011s = fminf(fmaxf(c011s, -b011), b011);
  }
  const float o3 = 1.0f - r.omega3;
  const float c210s = o3 * c210, c120s = o3 * c120, c201s = o3 * c201;
  const float c021s = o3 * c021, c102s = o3 * c102, c012s = o3 * c012;
  const float c111s = o3 * c111;
  const float o4d = 1.0f - r.omega4_diag, o4 = 1.0f - r.omega4;
  const float C220s = o4d * C220, C202s = o4d * C202, C022s = o4d * C022;
  const float C211s = o4 * C211, C121s = o4 * C121, C112s = o4 * C112;

  const float c220s = C220s + c200s * c020s + 2.0f * c110s * c110s;
  const float c202s = C202s + c200s * c002s + 2.0f * c101s * c101s;
  const float c022s = C022s + c020s * c002s + 2.0f * c011s * c011s;
  const float c211s = C211s + c200s * c011s + 2.0f * c110s * c101s;
  const float c121s = C121s + c020s * c101s + 2.0f * c110s * c011s;
  const float c112s = C112s + c002s * c110s + 2.0f * c101s * c011s;
  const float c221s = c200s * c021s + c020s * c201s + 4.0f * c110s * c111s +
                      2.0f * c101s * c120s + 2.0f * c011s * c210s;
  const float c212s = c200s * c012s + c002s * c210s + 2.0f * c110s * c102s +
                      4.0f * c101s * c111s + 2.0f * c011s * c201s;
  const float c122s = c020s * c102s + c002s * c120s + 2.0f * c110s * c012s +
                      4.0f * c011s * c111s + 2.0f * c101s * c021s;
  float c222s = c200s * C022s + c020s * C202s + c002s * C220s +
                4.0f * (c110s * C112s + c101s * C121s + c011s * C211s);
  c222s += 2.0f * (c210s * c012s + c201s * c021s + c120s * c102s) + 4.0f * c111s * c111s;
  c222s += c200s * c020s * c002s +
           2.0f * (c200s * c011s * c011s + c020s * c101s * c101s + c002s * c110s * c110s) +
           8.0f * c110s * c101s * c011s;

  const float rr = k000;
  A[0] = rr;
  A[1] = 0.0f; A[3] = 0.0f; A[9] = 0.0f;
  A[2] = rr * c200s; A[6] = rr * c020s; A[18] = rr * c002s;
  A[4] = rr * c110s; A[10] = rr * c101s; A[12] = rr * c011s;
  A[5] = rr * c210s; A[7] = rr * c120s; A[11] = rr * c201s;
  A[15] = rr * c021s; A[19] = rr * c102s; A[21] = rr * c012s;
  A[13] = rr * c111s;
  A[8] = rr * c220s; A[20] = rr * c202s; A[24] = rr * c022s;
  A[14] = rr * c211s; A[16] = rr * c121s; A[22] = rr * c112s;
  A[17] = rr * c221s; A[23] = rr * c212s; A[25] = rr * c122s;
  A[26] = rr * c222s;

  // backward: z, then y, then x
#pragma unroll
  for (int i = 0; i < 9; ++i) chim_bwd(A[i], A[i + 9], A[i + 18], uz);
#pragma unroll
  for (int zz = 0; zz < 3; ++zz)
#pragma unroll
    for (int a = 0; a < 3; ++a)
      chim_bwd(A[a + 9 * zz], A[a + 3 + 9 * zz], A[a + 6 + 9 * zz], uy);
#pragma unroll
  for (int i = 0; i < 9; ++i) chim_bwd(A[3 * i], A[3 * i + 1], A[3 * i + 2], ux);
}

// Positivity limiter (kernel_cumulant.jl:564-599).
__device__ __forceinline__ void positivity_limit(float (&A)[27], float rho, float ux, float uy,
                                              float uz, int comp) {
  float alpha = 1.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const float fe = feq_auto(rho, ux, uy, uz, w_of(k), (float)cx_of(k), (float)cy_of(k),
                              (float)cz_of(k), comp);
    const float fn = A[k] - fe;
    if (fn < 0.0f && fe > 1e-15f) alpha = fminf(alpha, fe / (fe - fn + 1e-15f));
  }
  alpha = fmaxf(alpha, 0.0f);
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const float fe = feq_auto(rho, ux, uy, uz, w_of(k), (float)cx_of(k), (float)cy_of(k),
                              (float)cz_of(k), comp);
    A[k] = fe + alpha * (A[k] - fe);
  }
}

// ---------------------------------------------------------------------------
// One cell of one block.  OP = OL_OP_*; WALE = gradients evaluated (c_wale
// != 0; with c_wale == 0 the reference's nu_eddy is exactly 0).
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Shared-memory staging of a block's 27 pull windows.
//
// E holds one halo-extended 10^3 plane per direction (E[k*1000 + (x+1) +
// 10(y+1) + 100(z+1)] for x, y, z in -1..8), so the pull of cell (x, y, z)
// in direction k is a single shared load at a compile-time offset from the
// cell's base.  The own block's 27 planes are copied with 16-byte loads; the
// 3176 out-of-block sources of the block (the slab each direction needs
// from its up to 7 neighbours) come from a per-device table of packed
// (k, neighbour direction, source cell, destination slot) entries; sources
// whose neighbour block is absent get their boundary value (inlet/outlet
// equilibrium, free-slip mirror, parent interpolation) right there.
// nbbase[dir] = element offset of neighbour `dir` within a direction plane,
// or -1 when it is absent.
// ---------------------------------------------------------------------------
constexpr int EPL = 1000;                 // floats per staged direction plane
constexpr int kStageBytes = 27 * EPL * 4;  // dynamic shared memory per CTA
constexpr int kHaloEntries = 3176;

__host__ __device__ constexpr int e_index(int x, int y, int z) {
  return (x + 1) + 10 * (y + 1) + 100 * (z + 1);
}

template <class ST, class BC>
__device__ __forceinline__ void stage_block(const void *f_in_v, int64_t dstride, float inv_scale,
                                            const int *nbbase, int t, float *E,
                                            const uint32_t *__restrict__ tab, BC bc) {
  using T = typename ST::T;
  const T *__restrict__ fin = (const T *)f_in_v;
  const int own = nbbase[13];
  if (ST::kBytes == 4) {
    const int c0 = (t & 127) * 4;
    const int dst = e_index(c0 & 7, (c0 >> 3) & 7, c0 >> 6);
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      const int k = (t >> 7) + 4 * j;
      if (k < 27) {
        const float4 v = __ldg((const float4 *)((const float *)fin + (size_t)k * dstride + own + c0));
        float *e = E + k * EPL + dst;
        e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w;
      }
    }
  } else {
    const int c0 = (t & 63) * 8;
    const int dst = e_index(0, (c0 >> 3) & 7, c0 >> 6);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = (t >> 6) + 8 * j;
      if (k < 27) {
        const uint4 raw = __ldg((const uint4 *)((const __half *)fin + (size_t)k * dstride + own + c0));
        const __half2 *h = (const __half2 *)&raw;
        const float w = w_of(k), sc = w * inv_scale;
        float *e = E + k * EPL + dst;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float2 f2 = __half22float2(h[i]);
          e[2 * i] = fmaf(f2.x, sc, w);
          e[2 * i + 1] = fmaf(f2.y, sc, w);
        }
      }
    }
  }
#pragma unroll 1
  for (int i = t; i < kHaloEntries; i += BCELLS) {
    const uint32_t te = __ldg(tab + i);
    const int k = te & 31, dir = (te >> 5) & 31, src = (te >> 10) & 511, dst = te >> 19;
    const int nb = nbbase[dir];
    float v;
    if (nb >= 0) {
      v = ST::load(fin, (size_t)k * dstride + nb + src, k, inv_scale);
    } else {
      const int sx = dst % 10 - 1, sy = (dst / 10) % 10 - 1, sz = dst / 100 - 1;
      v = bc(k, sx + cx_of(k), sy + cy_of(k), sz + cz_of(k));
    }
    E[k * EPL + dst] = v;
  }
}

// Neighbour-table row -> element offsets of the 27 neighbour blocks.
__device__ __forceinline__ void load_nbbase(const int32_t *nbr, int64_t nbr_stride,
                                            int64_t block_offset, int b, int t, int *nbbase) {
  if (t < 27) {
    const int nb = nbr[b + nbr_stride * t];
    nbbase[t] = nb > 0 ? (int)((block_offset + nb - 1) * BCELLS) : -1;
  }
}

// Stage the flow populations of block b of level L.
template <class ST>
__device__ __forceinline__ void stage_flow(const LevelDev &L, const int *nbbase, int b, int t,
                                           float *E) {
  stage_block<ST>(L.f_in, L.dstride, L.inv_scale, nbbase, t, E, L.halo_tab,
                  [&](int k, int x, int y, int z) { return pull_boundary<ST>(L, k, b, x, y, z); });
}

template <int OP, class ST, bool WALE>
__device__ __forceinline__ void stream_collide_cell(const LevelDev &L, const int *nbbase,
                                                    const float *E, int b, int t) {
  using T = typename ST::T;
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const ol_step_params &sp = L.sp;
  const size_t own = (size_t)nbbase[13] + t;
  T *__restrict__ fout = (T *)L.f_out;

  float A[27];
  const int eb = e_index(x, y, z);
#pragma unroll
  for (int k = 0; k < 27; ++k)
    A[k] = E[k * EPL + eb - (cx_of(k) + 10 * cy_of(k) + 100 * cz_of(k))];
  float rho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    rho += A[k];
    if (cx_of(k) == 1) jx += A[k]; else if (cx_of(k) == -1) jx -= A[k];
    if (cy_of(k) == 1) jy += A[k]; else if (cy_of(k) == -1) jy -= A[k];
    if (cz_of(k) == 1) jz += A[k]; else if (cz_of(k) == -1) jz -= A[k];
  }
  // Note: jx += v*cx in the reference equals jx +/- v exactly for cx = +/-1.
  if (L.status) {  // device watchdog (native path): report, never trap
    if (!(fabsf(rho) < 1e30f)) atomicOr(L.status, 1);
    else if (rho < 0.01f) atomicOr(L.status, 2);
  }

  float *fpost = (sp.store_post_collision && L.f_post) ? L.f_post : nullptr;
  if (L.obstacle[own]) {
    L.vel_out[own] = 0.0f;
    L.vel_out[own + L.dstride] = 0.0f;
    L.vel_out[own + 2 * L.dstride] = 0.0f;
    L.rho_out[own] = 1.0f;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      ST::store(fout, own + (size_t)k * L.dstride, k, L.scale, A[opp_of(k)]);
      if (fpost) fpost[own + (size_t)k * L.dstride] = A[opp_of(k)];
    }
    return;
  }
  rho = fmaxf(rho, 0.01f);
  const float inv_rho = 1.0f / rho;
  float ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const float spg = L.sponge[own];
  if (spg > 0.0f) {
    rho = rho * (1.0f - spg) + 1.0f * spg;
    ux = ux * (1.0f - spg) + sp.u_inlet * spg;
    uy = uy * (1.0f - spg);
    uz = uz * (1.0f - spg);
    if (sp.sponge_blend_distributions == 1) {
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const float ft = feq_auto(1.0f, sp.u_inlet, 0.0f, 0.0f, w_of(k), (float)cx_of(k),
                                  (float)cy_of(k), (float)cz_of(k), sp.compressible_corr);
        A[k] = A[k] * (1.0f - spg) + ft * spg;
      }
    }
  }
  float Fx = 0.0f, Fy = 0.0f, Fz = 0.0f;
  if (sp.wall_model_active == 1 && L.wall_dist)
    wall_force(L.wall_dist[own], rho, ux, uy, uz, sp.tau_molecular, Fx, Fy, Fz);
  const bool forced = (Fx != 0.0f) | (Fy != 0.0f) | (Fz != 0.0f);
  const float uxe = ux + 0.5f * Fx * inv_rho;
  const float uye = uy + 0.5f * Fy * inv_rho;
  const float uze = uz + 0.5f * Fz * inv_rho;

  L.vel_out[own] = ux;
  L.vel_out[own + L.dstride] = uy;
  L.vel_out[own + 2 * L.dstride] = uz;
  L.rho_out[own] = rho;

  float nu_eddy = 0.0f;
  if (WALE) nu_eddy = wale_nu(L, nbbase, x, y, z);
  nu_eddy = fmaxf(nu_eddy, sp.nu_sgs_background);

  float omega;  // omega_1 (cumulant) or omega (BGK)
  if (OP == OL_OP_CUMULANT) {
    const float nu_mol = (sp.tau_molecular - 0.5f) / 3.0f;
    const float tau_eff = 0.5f + 3.0f * (nu_mol + nu_eddy);
    omega = 1.0f / fmaxf(tau_eff, 0.500001f);
    CumulantRates r;
    r.omega1 = omega;
    r.omega_bulk = sp.omega_bulk;
    r.omega3 = sp.omega_3;
    r.omega4 = sp.omega_4;
    r.omega4_diag = sp.omega_4;
    if (sp.adaptive_omega4 == 1) {
      const float om1m2 = omega - 2.0f;
      const float Av = -(om1m2 * om1m2) / (sp.lambda_param * omega + 1e-10f);
      r.omega4_diag = fminf(fmaxf(Av, 0.01f), 2.0f);
    }
    r.limiter = sp.limiter_type;
    collide_cumulant(A, uxe, uye, uze, r);
    if (sp.limiter_type == OL_LIMITER_POSITIVITY) {
      float fmin = A[0];
#pragma unroll
      for (int k = 1; k < 27; ++k) fmin = fminf(fmin, A[k]);
      if (fmin < 0.0f) positivity_limit(A, rho, uxe, uye, uze, sp.compressible_corr);
    }
  } else {
    // Regularized BGK (kernel_regularized_bgk.jl:270-316); the Guo term uses
    // c.u_eq, as kernel_cumulant.jl:610 does (the reference line 302 names
    // an undefined `cu`).
    const float tau_turb = sp.tau_molecular + nu_eddy * 3.0f;
    omega = 1.0f / fmaxf(tau_turb, 0.500001f);
    float Pxx = 0.f, Pyy = 0.f, Pzz = 0.f, Pxy = 0.f, Pyz = 0.f, Pzx = 0.f;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      const float cxf = (float)cx_of(k), cyf = (float)cy_of(k), czf = (float)cz_of(k);
      const float fn = A[k] - feq_auto(rho, uxe, uye, uze, w_of(k), cxf, cyf, czf,
                                       sp.compressible_corr);
      Pxx += fn * cxf * cxf; Pyy += fn * cyf * cyf; Pzz += fn * czf * czf;
      Pxy += fn * cxf * cyf; Pyz += fn * cyf * czf; Pzx += fn * czf * cxf;
    }
    const float cs2p = 1.0f / 3.0f;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      const float cxf = (float)cx_of(k), cyf = (float)cy_of(k), czf = (float)cz_of(k);
      const float w = w_of(k);
      const float fe = feq_auto(rho, uxe, uye, uze, w, cxf, cyf, czf, sp.compressible_corr);
      const float fr = w * 4.5f *
                       (Pxx * (cxf * cxf - cs2p) + Pyy * (cyf * cyf - cs2p) +
                        Pzz * (czf * czf - cs2p) +
                        2.0f * (Pxy * cxf * cyf + Pyz * cyf * czf + Pzx * czf * cxf));
      A[k] = fe + (1.0f - omega) * fr;
    }
  }
  if (forced) {
    const float g = 1.0f - 0.5f * omega;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      const float cxf = (float)cx_of(k), cyf = (float)cy_of(k), czf = (float)cz_of(k);
      const float cu = cxf * uxe + cyf * uye + czf * uze;
      const float ft = w_of(k) * 3.0f *
                       ((cxf - ux + 3.0f * cu * cxf) * Fx +
                        (cyf - uy + 3.0f * cu * cyf) * Fy +
                        (czf - uz + 3.0f * cu * czf) * Fz);
      A[k] = A[k] + g * ft;
    }
  }
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    ST::store(fout, own + (size_t)k * L.dstride, k, L.scale, A[k]);
    if (fpost) fpost[own + (size_t)k * L.dstride] = A[k];
  }
}

}  // namespace ol
