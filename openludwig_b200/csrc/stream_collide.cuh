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
#include <type_traits>

#include "level_dev.cuh"

namespace ol {

// ---------------------------------------------------------------------------
// Coarse-to-fine ghost values (physics_interpolation.jl:4-127), split into
// what a ghost position shares across directions (the parent stencil and the
// blended, interpolated rho and u) and the per-direction population.
// gx, gy, gz: 1-based fine-level global source coordinates.
// ---------------------------------------------------------------------------
// Parent cell indices fit 32 bits (every launch checks that a level's cells
// do); gathers add them to per-plane base pointers.
struct ParentStencil {
  int32_t ci[8];     // parent cell of each trilinear corner, -1 when absent
  float wx, wy, wz;  // trilinear weights
};

// Trilinear weights of the fine cell (gx, gy, gz) in the parent grid and the
// parent cell of corner s (bit 0: x + 1, bit 1: y + 1, bit 2: z + 1), or -1
// when that parent cell does not exist.
template <class DEV>
__device__ __forceinline__ int32_t parent_corner(const DEV &L, int gx, int gy, int gz, int s,
                                                 float &wx, float &wy, float &wz) {
  const float pxc = ((float)gx - 0.5f) * 0.5f;
  const float pyc = ((float)gy - 0.5f) * 0.5f;
  const float pzc = ((float)gz - 0.5f) * 0.5f;
  const int px0 = (int)floorf(pxc), py0 = (int)floorf(pyc), pz0 = (int)floorf(pzc);
  wx = pxc - (float)px0;
  wy = pyc - (float)py0;
  wz = pzc - (float)pz0;
  const int pgx = (s & 1) ? px0 + 1 : max(1, px0);
  const int pgy = (s & 2) ? py0 + 1 : max(1, py0);
  const int pgz = (s & 4) ? pz0 + 1 : max(1, pz0);
  const int pbx = (pgx - 1) / BS + 1, pby = (pgy - 1) / BS + 1, pbz = (pgz - 1) / BS + 1;
  if (pbx >= 1 && pbx <= L.pdim_x && pby >= 1 && pby <= L.pdim_y && pbz >= 1 &&
      pbz <= L.pdim_z) {
    const int pb = L.pptr[(pbx - 1) + L.pdim_x * ((pby - 1) + L.pdim_y * (pbz - 1))];
    if (pb > 0)
      return (int32_t)((L.p_block_offset + pb - 1) * BCELLS) + (pgx - 1) % BS +
             BS * ((pgy - 1) % BS) + BS * BS * ((pgz - 1) % BS);
  }
  return -1;
}

template <class DEV>
__device__ __forceinline__ void parent_stencil(const DEV &L, int gx, int gy, int gz,
                                               ParentStencil &P) {
#pragma unroll
  for (int s = 0; s < 8; ++s) P.ci[s] = parent_corner(L, gx, gy, gz, s, P.wx, P.wy, P.wz);
}

// a * (1 - w) + b * w, each product and the sum rounded on its own (as the
// reference's Float32 expression; the same bits wherever it is evaluated)
__device__ __forceinline__ float lerp_rn(float a, float b, float w) {
  return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, w)), __fmul_rn(b, w));
}

__device__ __forceinline__ float trilerp(const float (&v)[8], float wx, float wy, float wz) {
  const float c00 = lerp_rn(v[0], v[1], wx);
  const float c01 = lerp_rn(v[4], v[5], wx);
  const float c10 = lerp_rn(v[2], v[3], wx);
  const float c11 = lerp_rn(v[6], v[7], wx);
  const float c0 = lerp_rn(c00, c10, wy);
  const float c1 = lerp_rn(c01, c11, wy);
  return lerp_rn(c0, c1, wz);
}

// Temporal blend of a parent value: lerp_rn(old, new, tw), or new alone
// without temporal interpolation.  At tw = 0 (the first child sub-step of a
// parent step) (1 - 0) * old + 0 * new rounds to old for every finite new, so
// `new` is not read there: half the parent gathers of that sub-step.
template <class NEW>
__device__ __forceinline__ float blend_parent(bool temporal, float tw, float old_v, NEW new_v) {
  if (!temporal) return new_v();
  if (tw == 0.0f) return old_v;
  return lerp_rn(old_v, new_v(), tw);
}

// Blended parent moments (rho, ux, uy, uz) of the present parent cell c at
// temporal weight tw.
__device__ __forceinline__ void corner_moments(const LevelDev &L, uint32_t c, float tw,
                                               float (&m)[4]) {
  const bool temporal = L.sp.use_temporal_interp == 1 && tw < 0.99f;
  const int64_t S = L.p_dstride;
  const float *vo = L.pvel_old, *vn = L.pvel;
  if (temporal && tw == 0.0f) {
    m[0] = L.prho_old[c]; m[1] = vo[c];
    m[2] = (vo + S)[c]; m[3] = (vo + 2 * S)[c];
    return;
  }
  const float rn = L.prho[c], uxn = vn[c], uyn = (vn + S)[c], uzn = (vn + 2 * S)[c];
  if (temporal) {
    m[0] = lerp_rn(L.prho_old[c], rn, tw);
    m[1] = lerp_rn(vo[c], uxn, tw);
    m[2] = lerp_rn((vo + S)[c], uyn, tw);
    m[3] = lerp_rn((vo + 2 * S)[c], uzn, tw);
  } else {
    m[0] = rn; m[1] = uxn; m[2] = uyn; m[3] = uzn;
  }
}

// Blended parent population k of the present parent cell c at weight tw.
template <class ST>
__device__ __forceinline__ float corner_population(const LevelDev &L, uint32_t c, int k,
                                                   float tw) {
  const bool temporal = L.sp.use_temporal_interp == 1 && tw < 0.99f;
  using T = typename ST::T;
  const T *po = (const T *)L.pf_old + (size_t)k * L.p_dstride;   // plane k
  const T *pn = (const T *)L.pf + (size_t)k * L.p_dstride;
  const float fo = temporal ? ST::load(po, c, k, L.p_inv_scale) : 0.0f;
  return blend_parent(temporal, tw, fo, [&] { return ST::load(pn, c, k, L.p_inv_scale); });
}

// Parent rho, ux, uy, uz at the ghost position: each corner blended between
// the parent's old and new state, missing corners replaced by the (possibly
// missing, then rho = 1, u = 0) first corner, then trilinear.
__device__ __forceinline__ void interp_moments(const LevelDev &L, const ParentStencil &P,
                                               float tw, float (&r)[4]) {
  float v[4][8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    float m[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    if (P.ci[s] >= 0) corner_moments(L, (uint32_t)P.ci[s], tw, m);
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i][s] = m[i];
  }
#pragma unroll
  for (int s = 1; s < 8; ++s)
    if (P.ci[s] < 0)
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i][s] = v[i][0];
#pragma unroll
  for (int i = 0; i < 4; ++i) r[i] = trilerp(v[i], P.wx, P.wy, P.wz);
}

// From the 8 corner values of f_k (absent corners already replaced): the
// interpolated f_k split into equilibrium (from the interpolated moments r)
// and non-equilibrium part, the latter rescaled by (tau_f - 1/2) /
// (tau_c - 1/2) clamped to [0.01, 100].
__device__ __forceinline__ float finish_population(const LevelDev &L, int k, const float (&v)[8],
                                                   float wx, float wy, float wz,
                                                   const float (&r)[4]) {
  const ol_step_params &sp = L.sp;
  const float fi = trilerp(v, wx, wy, wz);
  const float fe = feq_auto(r[0], r[1], r[2], r[3], w_of(k), (float)cx_of(k), (float)cy_of(k),
                            (float)cz_of(k), sp.compressible_corr);
  const float fneq = fi - fe;
  const float tc = sp.tau_parent - 0.5f, tf = sp.tau_molecular - 0.5f;
  const float sc = tc > 1e-6f ? fminf(fmaxf(tf / tc, 0.01f), 100.0f) : 1.0f;
  return __fadd_rn(fe, __fmul_rn(fneq, sc));
}

// Ghost population k at a position with stencil P and moments r (weight tw).
template <class ST>
__device__ __forceinline__ float interp_population(const LevelDev &L, int k,
                                                   const ParentStencil &P, const float (&r)[4],
                                                   float tw) {
  float v[8];
#pragma unroll
  for (int s = 0; s < 8; ++s)
    v[s] = P.ci[s] >= 0 ? corner_population<ST>(L, (uint32_t)P.ci[s], k, tw) : w_of(k);
#pragma unroll
  for (int s = 1; s < 8; ++s)
    if (P.ci[s] < 0) v[s] = v[0];
  return finish_population(L, k, v, P.wx, P.wy, P.wz, r);
}

// The same population for both child sub-steps of a parent step from one
// read of the parent's old and new state: g0 at weight 0 (the old state),
// g1 at kSecondSubstepWeight; r0 / r1 are the moments at those weights.
// Bitwise what interp_population gives at each weight.
template <class ST>
__device__ __forceinline__ void interp_population_pair(const LevelDev &L, int k,
                                                       const ParentStencil &P,
                                                       const float (&r0)[4],
                                                       const float (&r1)[4], float &g0,
                                                       float &g1) {
  const bool temporal = L.sp.use_temporal_interp == 1;
  using T = typename ST::T;
  const T *po = (const T *)L.pf_old + (size_t)k * L.p_dstride;   // plane k
  const T *pn = (const T *)L.pf + (size_t)k * L.p_dstride;
  float v0[8], v1[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    v0[s] = v1[s] = w_of(k);
    if (P.ci[s] >= 0) {
      const uint32_t c = (uint32_t)P.ci[s];
      const float fn = ST::load(pn, c, k, L.p_inv_scale);
      const float fo = temporal ? ST::load(po, c, k, L.p_inv_scale) : fn;
      v0[s] = fo;
      v1[s] = temporal ? lerp_rn(fo, fn, kSecondSubstepWeight) : fn;
    }
  }
#pragma unroll
  for (int s = 1; s < 8; ++s)
    if (P.ci[s] < 0) { v0[s] = v0[0]; v1[s] = v1[0]; }
  g0 = finish_population(L, k, v0, P.wx, P.wy, P.wz, r0);
  g1 = finish_population(L, k, v1, P.wx, P.wy, P.wz, r1);
}

// ---------------------------------------------------------------------------
// Source value of a pull whose neighbour block is absent and whose source
// lies outside the domain or on level 1 (kernel_cumulant.jl:117-159); the
// fine-level interface case (:153-155) is interp_population, filled by
// fill_missing_flow.  x, y, z are 0-based local coordinates.
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
  return w;
}

// ---------------------------------------------------------------------------
// WALE eddy viscosity from vel_in central differences
// (kernel_cumulant.jl:264-305, physics_utils.jl:85-123).
// ---------------------------------------------------------------------------
// Cell index of a face neighbour of the cell at local index `own` (element
// offset, own block at nbbase[13]) one step along an axis: inside the block
// `own + step`; across the face, the same cell of the face neighbour `dir`
// (`own + wrap - nbbase[13] + nbbase[dir]`); with no neighbour there, the cell
// itself (the zero-gradient fallback of physics_utils.jl:85-123).
__device__ __forceinline__ int vel_neighbor(const int *nbbase, int own, bool inside, int step,
                                            int dir, int wrap) {
  if (inside) return own + step;
  const int nb = nbbase[dir];
  return nb >= 0 ? own - nbbase[13] + nb + wrap : own;
}

// The 18 neighbour velocities the WALE gradients need (E, W, N, S, T, B
// neighbour, x/y/z component each), read from vel_in.
struct WaleVel {
  float e[3], w[3], n[3], s[3], t[3], b[3];
};

__device__ __forceinline__ void wale_load(const LevelDev &L, const int *nbbase, int x, int y, int z,
                                          WaleVel &V) {
  // the three velocity components are planes dstride apart
  const float *__restrict__ v0 = L.vel_in;
  const float *__restrict__ v1 = v0 + L.dstride;
  const float *__restrict__ v2 = v1 + L.dstride;
  const int own = nbbase[13] + x + BS * y + BS * BS * z;
  // E (x+1), W (x-1), N (y+1), S (y-1), T (z+1), B (z-1)
  const int ce = vel_neighbor(nbbase, own, x < BS - 1, 1, 14, -(BS - 1));
  const int cw = vel_neighbor(nbbase, own, x > 0, -1, 12, BS - 1);
  const int cn = vel_neighbor(nbbase, own, y < BS - 1, BS, 16, -BS * (BS - 1));
  const int cs = vel_neighbor(nbbase, own, y > 0, -BS, 10, BS * (BS - 1));
  const int ct = vel_neighbor(nbbase, own, z < BS - 1, BS * BS, 22, -BS * BS * (BS - 1));
  const int cb = vel_neighbor(nbbase, own, z > 0, -BS * BS, 4, BS * BS * (BS - 1));
  V.e[0] = __ldg(v0 + ce); V.e[1] = __ldg(v1 + ce); V.e[2] = __ldg(v2 + ce);
  V.w[0] = __ldg(v0 + cw); V.w[1] = __ldg(v1 + cw); V.w[2] = __ldg(v2 + cw);
  V.n[0] = __ldg(v0 + cn); V.n[1] = __ldg(v1 + cn); V.n[2] = __ldg(v2 + cn);
  V.s[0] = __ldg(v0 + cs); V.s[1] = __ldg(v1 + cs); V.s[2] = __ldg(v2 + cs);
  V.t[0] = __ldg(v0 + ct); V.t[1] = __ldg(v1 + ct); V.t[2] = __ldg(v2 + ct);
  V.b[0] = __ldg(v0 + cb); V.b[1] = __ldg(v1 + cb); V.b[2] = __ldg(v2 + cb);
}

__device__ __forceinline__ float wale_from(const WaleVel &V, float c_wale) {
  const float exx = V.e[0], eyx = V.e[1], ezx = V.e[2];
  const float wxx = V.w[0], wyx = V.w[1], wzx = V.w[2];
  const float nxx = V.n[0], nyx = V.n[1], nzx = V.n[2];
  const float sxx = V.s[0], syx = V.s[1], szx = V.s[2];
  const float txx = V.t[0], tyx = V.t[1], tzx = V.t[2];
  const float bxx = V.b[0], byx = V.b[1], bzx = V.b[2];
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
    if (den > 1e-12f) nu = (c_wale * c_wale) * op1_32 / den;
  }
  return nu;
}

__device__ __forceinline__ float wale_nu(const LevelDev &L, const int *nbbase, int x, int y,
                                         int z) {
  WaleVel V;
  wale_load(L, nbbase, x, y, z, V);
  return wale_from(V, L.sp.c_wale);
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
// (m2 +- m1) / 2 as fma(+-1/2, m1, m2 / 2): the same bits (halving is exact
// at these magnitudes, so both round the same exact value once), one
// instruction fewer.
__device__ __forceinline__ void chim_bwd(float &a, float &b, float &c, float u) {
  const float m0 = a, m1 = b + u * a, m2 = c + 2.0f * u * b + u * u * a;
  const float h = 0.5f * m2;
  c = fmaf(0.5f, m1, h);
  a = fmaf(-0.5f, m1, h);
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

// Boundary values of the staging slots whose neighbour block is absent.  One
// call per thread, made only by CTAs whose block has an absent neighbour, so
// the call and its register save/restore stay off the bulk path.
template <class BC>
__device__ __noinline__ void fill_missing_slots(const int *nbbase, int t, float *E,
                                                const uint32_t *__restrict__ tab, BC bc) {
  for (int i = t; i < kHaloEntries; i += BCELLS) {
    const uint32_t te = __ldg(tab + i);
    const int k = te & 31, dir = (te >> 5) & 31, dst = te >> 19;
    if (nbbase[dir] >= 0) continue;
    const int sx = dst % 10 - 1, sy = (dst / 10) % 10 - 1, sz = dst / 100 - 1;
    E[k * EPL + dst] = bc(k, sx + cx_of(k), sy + cy_of(k), sz + cz_of(k));
  }
}

// Ring positions of the staging plane (the 488 slots of the 10^3 plane
// outside the 8^3 block), listed in the staging table after its halo entries.
constexpr int kRingEntries = 1000 - 512;
// Staging table layout: kHaloEntries packed entries, the kRingEntries ring
// slots of the 10^3 plane, then per halo entry the ring index of its slot.
constexpr int kRingIndexOffset = kHaloEntries + kRingEntries;
constexpr int kHaloTableSize = kRingIndexOffset + kHaloEntries;

// Staging planes whose slot p is never read, for a ring position p with
// outward offsets (ox, oy, oz): a direction k with c_a = o_a on the first
// axis a where o_a != 0 would pull slot p into a cell at -2 or 9 on that
// axis, outside the block.  Four of these (i = 0..3) hold the interpolated
// rho, ux, uy, uz of an interface position between the two fill phases.
__device__ __forceinline__ int stash_plane(int ox, int oy, int oz, int i) {
  const int u = (i & 1) + 1, v = (i >> 1) + 1;
  if (ox != 0) return (ox + 1) + 3 * u + 9 * v;
  if (oy != 0) return u + 3 * (oy + 1) + 9 * v;
  return u + 3 * v + 9 * (oz + 1);
}

// Boundary values of the flow staging slots whose neighbour block is absent.
// Domain boundaries (inlet, outlet, free-slip mirrors) and level-1 gaps are
// evaluated per slot by pull_boundary.  A fine-level interface slot needs the
// parent's rho and u interpolated at its source position, which every
// direction pulling from that position shares: phase 1 computes them once
// per ring position (one thread each) into stash slots, phase 2 spreads the
// (direction, slot) entries over all threads and interpolates only f_k.
template <class ST>
__device__ __noinline__ void fill_missing_flow(const LevelDev &L, const int *nbbase, int b, int t,
                                               float *E) {
  const ol_step_params &sp = L.sp;
  const uint32_t *__restrict__ tab = L.halo_tab;
  const bool fine = sp.is_level_1 == 0;
  const int gx0 = (L.map_x[b] - 1) * BS + 1, gy0 = (L.map_y[b] - 1) * BS + 1,
            gz0 = (L.map_z[b] - 1) * BS + 1;
  if (fine) {
    if (t < kRingEntries) {
      const int p = (int)__ldg(tab + kHaloEntries + t);
      const int sx = p % 10 - 1, sy = (p / 10) % 10 - 1, sz = p / 100 - 1;
      const int ox = sx < 0 ? -1 : (sx > 7 ? 1 : 0);
      const int oy = sy < 0 ? -1 : (sy > 7 ? 1 : 0);
      const int oz = sz < 0 ? -1 : (sz > 7 ? 1 : 0);
      const int sgx = gx0 + sx, sgy = gy0 + sy, sgz = gz0 + sz;
      if (nbbase[(ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)] < 0 && sgx >= 1 &&
          sgx <= sp.nx_global && sgy >= 1 && sgy <= sp.ny_global && sgz >= 1 &&
          sgz <= sp.nz_global) {
        ParentStencil P;
        parent_stencil(L, sgx, sgy, sgz, P);
        float r[4];
        interp_moments(L, P, sp.temporal_weight, r);
#pragma unroll
        for (int i = 0; i < 4; ++i) E[stash_plane(ox, oy, oz, i) * EPL + p] = r[i];
      }
    }
    __syncthreads();
  }
  for (int i = t; i < kHaloEntries; i += BCELLS) {
    const uint32_t te = __ldg(tab + i);
    const int k = te & 31, dir = (te >> 5) & 31, p = te >> 19;
    if (nbbase[dir] >= 0) continue;
    const int sx = p % 10 - 1, sy = (p / 10) % 10 - 1, sz = p / 100 - 1;
    const int sgx = gx0 + sx, sgy = gy0 + sy, sgz = gz0 + sz;
    float v;
    if (fine && sgx >= 1 && sgx <= sp.nx_global && sgy >= 1 && sgy <= sp.ny_global &&
        sgz >= 1 && sgz <= sp.nz_global) {
      const int ox = sx < 0 ? -1 : (sx > 7 ? 1 : 0);
      const int oy = sy < 0 ? -1 : (sy > 7 ? 1 : 0);
      const int oz = sz < 0 ? -1 : (sz > 7 ? 1 : 0);
      float r[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) r[j] = E[stash_plane(ox, oy, oz, j) * EPL + p];
      ParentStencil P;
      parent_stencil(L, sgx, sgy, sgz, P);
      v = interp_population<ST>(L, k, P, r, sp.temporal_weight);
    } else {
      v = pull_boundary<ST>(L, k, b, sx + cx_of(k), sy + cy_of(k), sz + cz_of(k));
    }
    E[k * EPL + p] = v;
  }
}

// Separate pass over the blocks of a level: the absent-neighbour pull sources
// of block b, in staging-table order, into L.ghost[b * kHaloEntries + i].
// Same values as fill_missing_flow; here the CTA is small, leaves the SM's
// L1 to the parent gathers (a parent cell serves ~20 ghost slots), keeps the
// whole parent stencil of each ring position in shared memory, and spreads
// only the slots that need a value over its threads (compacted lists), so no
// stream-collide CTA waits at a barrier while a few of its threads
// interpolate.  Parent cell indices are kept as int32 (the launch checks
// that the parent's cells fit).
constexpr int kGhostThreads = 256;
constexpr int kGhostMinBlocks = 4;  // resident CTAs per SM (64 registers per thread)
constexpr int kGhostScan = (kHaloEntries + kGhostThreads - 1) / kGhostThreads;  // 13

// Warp-aggregated append of `value` to a shared list when `flag` is set;
// every lane of the warp makes the call.
__device__ __forceinline__ void append_if(bool flag, int value, int *count, int16_t *list) {
  const unsigned m = __ballot_sync(0xffffffffu, flag);
  if (m == 0) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (flag) list[base + __popc(m & ((1u << lane) - 1u))] = (int16_t)value;
}

// Row of block b in the ghost scratch of level L (null when the block has
// no row: no scratch, or no absent neighbour under a compact index).  DEV is
// the flow (LevelDev) or thermal (ThermalDev) level.
template <class DEV>
__device__ __forceinline__ float *ghost_row_of(const DEV &L, int b) {
  if (!L.ghost) return nullptr;
  const int r = L.gidx ? L.gidx[b] : b;
  return r >= 0 ? L.ghost + (size_t)r * kHaloEntries : nullptr;
}
// The same row of ghost_next (written by the first sub-step of a pair).
template <class DEV>
__device__ __forceinline__ float *ghost_next_row_of(const DEV &L, int b) {
  if (L.ghost_mode != kGhostPairFirst || !L.ghost_next) return nullptr;
  const int r = L.gidx ? L.gidx[b] : b;
  return r >= 0 ? L.ghost_next + (size_t)r * kHaloEntries : nullptr;
}

// What the ghost pass needs to know of a flow level; the thermal DDF
// provides the same functions for its populations (thermal.cuh).
__device__ __forceinline__ const ol_step_params &ghost_params(const LevelDev &L) { return L.sp; }
__device__ __forceinline__ void ghost_corner_moments(const LevelDev &L, uint32_t c, float tw,
                                                     float (&m)[4]) {
  corner_moments(L, c, tw, m);
}
__device__ __forceinline__ void ghost_moments(const LevelDev &L, const ParentStencil &P, float tw,
                                              float (&r)[4]) {
  interp_moments(L, P, tw, r);
}
template <class ST>
__device__ __forceinline__ float ghost_population(const LevelDev &L, int k, const ParentStencil &P,
                                                  const float (&r)[4], float tw, ST) {
  return interp_population<ST>(L, k, P, r, tw);
}
template <class ST>
__device__ __forceinline__ void ghost_population_pair(const LevelDev &L, int k,
                                                      const ParentStencil &P,
                                                      const float (&r0)[4], const float (&r1)[4],
                                                      ST, float &g0, float &g1) {
  interp_population_pair<ST>(L, k, P, r0, r1, g0, g1);
}
template <class ST>
__device__ __forceinline__ float ghost_boundary(const LevelDev &L, int k, int b, int x, int y,
                                                int z, ST) {
  return pull_boundary<ST>(L, k, b, x, y, z);
}

// One CTA of kGhostThreads threads evaluates block b's row G.  With
// L.ghost_mode == kGhostPairFirst it also writes into G2 the coarse-to-fine
// slots of the pair's second sub-step (the parent does not step in between),
// reading each parent value once for both; with kGhostPairSecond those slots
// of G are already set and only the domain-boundary slots are evaluated.
template <class ST, class DEV>
__device__ __forceinline__ void ghost_fill_block(const DEV &L, int b, float *G, float *G2) {
  __shared__ int nbbase[27];
  __shared__ int n_pos, n_slot;
  __shared__ float rs[4][kRingEntries];     // interpolated rho, ux, uy, uz
  __shared__ float rs2[4][kRingEntries];    // the same at the second sub-step's weight
  __shared__ int32_t cs[8][kRingEntries];   // parent stencil cells
  __shared__ float ws[3][kRingEntries];     // trilinear weights
  __shared__ uint8_t iface_of[kRingEntries];  // ring position takes coarse-to-fine values
  __shared__ int16_t pos_list[kRingEntries];
  __shared__ int16_t slot_list[kHaloEntries];
  const int t = threadIdx.x;
  const auto &sp = ghost_params(L);
  const bool precomputed = L.ghost_mode == kGhostPairSecond;
  const int mx = L.map_x[b], my = L.map_y[b], mz = L.map_z[b];
  int missing = 0;
  if (t < 27) {
    const int nb = L.nbr[b + L.nbr_stride * t];
    nbbase[t] = nb > 0 ? (int)((L.block_offset + nb - 1) * BCELLS) : -1;
    missing = nb <= 0;
    if (missing && precomputed) {
      // the second sub-step of a pair only revisits absent neighbours that are
      // not wholly inside the domain (all others are coarse-to-fine, set)
      const int nbx = mx + t % 3 - 1, nby = my + (t / 3) % 3 - 1, nbz = mz + t / 9 - 1;
      missing = !(nbx >= 1 && nbx * BS <= sp.nx_global && nby >= 1 &&
                  nby * BS <= sp.ny_global && nbz >= 1 && nbz * BS <= sp.nz_global);
    }
  }
  if (t == 0) { n_pos = 0; n_slot = 0; }
  if (!__syncthreads_or(missing)) return;
  const uint32_t *__restrict__ tab = L.halo_tab;
  const bool fine = sp.is_level_1 == 0;
  const bool pair = G2 != nullptr;                         // first sub-step of a pair
  const bool interp = fine && !precomputed;                // this pass interpolates
  const float tw = sp.temporal_weight;
  const int gx0 = (mx - 1) * BS + 1, gy0 = (my - 1) * BS + 1, gz0 = (mz - 1) * BS + 1;
  auto in_domain = [&](int gx, int gy, int gz) {
    return gx >= 1 && gx <= sp.nx_global && gy >= 1 && gy <= sp.ny_global && gz >= 1 &&
           gz <= sp.nz_global;
  };
  // lists: interface ring positions and slots whose neighbour is absent
  uint32_t te[kGhostScan];
#pragma unroll
  for (int j = 0; j < kGhostScan; ++j) {
    const int i = t + j * kGhostThreads;
    te[j] = i < kHaloEntries ? __ldg(tab + i) : 0u;
  }
  if (fine) {
    for (int j = 0; j < (kRingEntries + kGhostThreads - 1) / kGhostThreads; ++j) {
      const int q = t + j * kGhostThreads;
      bool want = false;
      if (q < kRingEntries) {
        const int p = (int)__ldg(tab + kHaloEntries + q);
        const int sx = p % 10 - 1, sy = (p / 10) % 10 - 1, sz = p / 100 - 1;
        const int ox = sx < 0 ? -1 : (sx > 7 ? 1 : 0);
        const int oy = sy < 0 ? -1 : (sy > 7 ? 1 : 0);
        const int oz = sz < 0 ? -1 : (sz > 7 ? 1 : 0);
        want = nbbase[(ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)] < 0 &&
               in_domain(gx0 + sx, gy0 + sy, gz0 + sz);
        iface_of[q] = want;
      }
      append_if(interp && want, q, &n_pos, pos_list);
    }
  }
#pragma unroll
  for (int j = 0; j < kGhostScan; ++j) {
    const int i = t + j * kGhostThreads;
    append_if(i < kHaloEntries && nbbase[(te[j] >> 5) & 31] < 0, i, &n_slot, slot_list);
  }
  __syncthreads();
  if (interp) {
    for (int j = t; j < n_pos; j += kGhostThreads) {
      const int q = pos_list[j];
      const int p = (int)__ldg(tab + kHaloEntries + q);
      const int sx = p % 10 - 1, sy = (p / 10) % 10 - 1, sz = p / 100 - 1;
      ParentStencil P;
      parent_stencil(L, gx0 + sx, gy0 + sy, gz0 + sz, P);
      float r[4];
      ghost_moments(L, P, tw, r);
#pragma unroll
      for (int i = 0; i < 4; ++i) rs[i][q] = r[i];
      if (pair) {
        ghost_moments(L, P, kSecondSubstepWeight, r);
#pragma unroll
        for (int i = 0; i < 4; ++i) rs2[i][q] = r[i];
      }
#pragma unroll
      for (int s = 0; s < 8; ++s) cs[s][q] = P.ci[s];
      ws[0][q] = P.wx; ws[1][q] = P.wy; ws[2][q] = P.wz;
    }
    __syncthreads();
  }
  for (int j = t; j < n_slot; j += kGhostThreads) {
    const int i = slot_list[j];
    const uint32_t e = __ldg(tab + i);
    const int k = e & 31;
    const int q = fine ? (int)__ldg(tab + kRingIndexOffset + i) : 0;
    if (fine && iface_of[q]) {
      if (precomputed) continue;
      ParentStencil P;
#pragma unroll
      for (int s = 0; s < 8; ++s) P.ci[s] = cs[s][q];
      P.wx = ws[0][q]; P.wy = ws[1][q]; P.wz = ws[2][q];
      const float r[4] = {rs[0][q], rs[1][q], rs[2][q], rs[3][q]};
      if (pair) {
        const float r2[4] = {rs2[0][q], rs2[1][q], rs2[2][q], rs2[3][q]};
        float g0, g1;
        ghost_population_pair(L, k, P, r, r2, ST{}, g0, g1);
        G[i] = g0;
        G2[i] = g1;
      } else {
        G[i] = ghost_population(L, k, P, r, tw, ST{});
      }
    } else {
      const int p = e >> 19;
      const int sx = p % 10 - 1, sy = (p / 10) % 10 - 1, sz = p / 100 - 1;
      G[i] = ghost_boundary(L, k, b, sx + cx_of(k), sy + cy_of(k), sz + cz_of(k), ST{});
    }
  }
}

// Drop-in: one CTA per block of the level (rows indexed by block).
template <class ST>
__global__ void __launch_bounds__(kGhostThreads, kGhostMinBlocks)
    k_ghost_fill(const __grid_constant__ LevelDev L) {
  pdl_wait();  // the parent's new state and this level's f_in
  const int b = L.gblocks ? L.gblocks[blockIdx.x] : (int)blockIdx.x;
  ghost_fill_block<ST>(L, b, ghost_row_of(L, b), ghost_next_row_of(L, b));
}

constexpr int kHaloPerThread = (kHaloEntries + BCELLS - 1) / BCELLS;  // 7

// Asks L2 for the per-cell arrays of block nb (local index) of level L: its
// 27 population planes, velocity (WALE reads it), sponge, mask and wall
// distance, one bulk prefetch per thread t < 33.  The stream-collide launch
// issues this for the block its CTA slot takes one wave later, so that
// block's staging loads find their data in L2 (no registers, no shared
// memory, nothing to wait for).  Every run is whole and 16-byte aligned:
// blocks are 512 cells and the arrays' planes are whole blocks.
template <class ST>
__device__ __forceinline__ void prefetch_block_l2(const LevelDev &L, int nb, int t) {
  if (nb >= L.n_blocks || t >= 33) return;
  using T = typename ST::T;
  const int64_t o = (L.block_offset + nb) * BCELLS;
  const void *src = nullptr;
  unsigned bytes = BCELLS * sizeof(float);
  if (t < 27) {
    src = (const T *)L.f_in + o + (int64_t)t * L.dstride;
    bytes = BCELLS * sizeof(T);
  } else if (t < 30) {
    if (L.vel_in) src = L.vel_in + o + (int64_t)(t - 27) * L.dstride;
  } else if (t == 30) {
    src = L.sponge + o;
  } else if (t == 31) {
    src = L.obstacle + o;
    bytes = BCELLS;
  } else if (L.wall_dist) {
    src = L.wall_dist + o;
  }
  if (src) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes)
                        : "memory");
}

// The own block's 27 planes, loaded into registers with 16-byte loads
// (FP32: 7 float4 per thread; FP16: 4 x 8 halves).  The loads depend only on
// the block's own offset, so a kernel can issue them before it has read the
// neighbour table.
template <class ST> struct OwnRegs;
template <> struct OwnRegs<StoreF32> { float4 v[7]; };
template <> struct OwnRegs<StoreF16S> { uint4 v[4]; };

__device__ __forceinline__ void own_load(const void *f_in_v, int64_t dstride, int64_t own, int t,
                                         OwnRegs<StoreF32> &r) {
  const float *fin = (const float *)f_in_v;
  const int c0 = (t & 127) * 4;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const int k = (t >> 7) + 4 * j;
    if (k < 27) r.v[j] = __ldg((const float4 *)(fin + (size_t)k * dstride + own + c0));
  }
}
__device__ __forceinline__ void own_load(const void *f_in_v, int64_t dstride, int64_t own, int t,
                                         OwnRegs<StoreF16S> &r) {
  const __half *fin = (const __half *)f_in_v;
  const int c0 = (t & 63) * 8;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = (t >> 6) + 8 * j;
    if (k < 27) r.v[j] = __ldg((const uint4 *)(fin + (size_t)k * dstride + own + c0));
  }
}
// Odd lanes (x = 4..7 of a row) write their four cells rotated by one, so each
// store instruction of a warp touches every bank at most twice (three times
// in x order).
__device__ __forceinline__ void own_store(const OwnRegs<StoreF32> &r, float, int t, float *E) {
  const int c0 = (t & 127) * 4;
  const int dst = e_index(c0 & 7, (c0 >> 3) & 7, c0 >> 6);
  const bool odd = t & 1;
  const int o0 = odd ? 1 : 0, o1 = odd ? 2 : 1, o2 = odd ? 3 : 2, o3 = odd ? 0 : 3;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const int k = (t >> 7) + 4 * j;
    if (k < 27) {
      float *e = E + k * EPL + dst;
      const float4 v = r.v[j];
      e[o0] = odd ? v.y : v.x;
      e[o1] = odd ? v.z : v.y;
      e[o2] = odd ? v.w : v.z;
      e[o3] = odd ? v.x : v.w;
    }
  }
}
__device__ __forceinline__ void own_store(const OwnRegs<StoreF16S> &r, float inv_scale, int t,
                                          float *E) {
  const int c0 = (t & 63) * 8;
  const int dst = e_index(0, (c0 >> 3) & 7, c0 >> 6);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = (t >> 6) + 8 * j;
    if (k < 27) {
      const __half2 *h = (const __half2 *)&r.v[j];
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

// Halo part of the staging, then the own block's registers into E.
// ghost_row: this block's precomputed absent-neighbour values in table order
// (kHaloEntries floats), or null to compute them here with `fill`.
template <class ST, class FILL>
__device__ __forceinline__ void stage_halo(const void *f_in_v, int64_t dstride, float inv_scale,
                                           const int *nbbase, int t, float *E,
                                           const uint32_t *__restrict__ tab, bool any_missing,
                                           const float *__restrict__ ghost_row,
                                           const OwnRegs<ST> &own_regs, FILL fill) {
  using T = typename ST::T;
  const T *__restrict__ fin = (const T *)f_in_v;
  // halo sources: all table entries and source values of this thread in flight at once
  uint32_t te[kHaloPerThread];
#pragma unroll
  for (int j = 0; j < kHaloPerThread; ++j) {
    const int i = t + j * BCELLS;
    te[j] = i < kHaloEntries ? __ldg(tab + i) : 0xFFFFFFFFu;
  }
  float hv[kHaloPerThread];
  int hd[kHaloPerThread];
#pragma unroll
  for (int j = 0; j < kHaloPerThread; ++j) {
    hd[j] = -1;
    hv[j] = 0.0f;
    if (te[j] != 0xFFFFFFFFu) {
      const int k = te[j] & 31, dir = (te[j] >> 5) & 31, src = (te[j] >> 10) & 511;
      const int nb = nbbase[dir];
      if (nb >= 0) {
        hd[j] = k * EPL + (int)(te[j] >> 19);
        hv[j] = ST::load(fin, (size_t)k * dstride + nb + src, k, inv_scale);
      } else if (ghost_row) {
        hd[j] = k * EPL + (int)(te[j] >> 19);
        hv[j] = ghost_row[t + j * BCELLS];
      }
    }
  }
  own_store(own_regs, inv_scale, t, E);
#pragma unroll
  for (int j = 0; j < kHaloPerThread; ++j)
    if (hd[j] >= 0) E[hd[j]] = hv[j];
  if (any_missing && !ghost_row) fill();
}

template <class ST, class FILL>
__device__ __forceinline__ void stage_block(const void *f_in_v, int64_t dstride, float inv_scale,
                                            const int *nbbase, int t, float *E,
                                            const uint32_t *__restrict__ tab, bool any_missing,
                                            const float *__restrict__ ghost_row, FILL fill) {
  OwnRegs<ST> r;
  own_load(f_in_v, dstride, nbbase[13], t, r);
  stage_halo<ST>(f_in_v, dstride, inv_scale, nbbase, t, E, tab, any_missing, ghost_row, r, fill);
}

// Neighbour-table row -> element offsets of the 27 neighbour blocks, then a
// barrier; returns whether any neighbour of the block is absent.
__device__ __forceinline__ bool load_nbbase_sync(const int32_t *nbr, int64_t nbr_stride,
                                                 int64_t block_offset, int b, int t, int *nbbase) {
  int missing = 0;
  if (t < 27) {
    const int nb = nbr[b + nbr_stride * t];
    nbbase[t] = nb > 0 ? (int)((block_offset + nb - 1) * BCELLS) : -1;
    missing = nb <= 0;
  }
  return __syncthreads_or(missing) != 0;
}

// Stage the flow populations of block b of level L.
template <class ST>
__device__ __forceinline__ void stage_flow(const LevelDev &L, const int *nbbase, int b, int t,
                                           float *E, bool any_missing) {
  const float *ghost_row = ghost_row_of(L, b);
  stage_block<ST>(L.f_in, L.dstride, L.inv_scale, nbbase, t, E, L.halo_tab, any_missing,
                  ghost_row, [&]() { fill_missing_flow<ST>(L, nbbase, b, t, E); });
}

// The same with the own block already in registers (own_load issued before
// the neighbour table was read).
template <class ST>
__device__ __forceinline__ void stage_flow(const LevelDev &L, const int *nbbase, int b, int t,
                                           float *E, bool any_missing, const OwnRegs<ST> &r) {
  const float *ghost_row = ghost_row_of(L, b);
  stage_halo<ST>(L.f_in, L.dstride, L.inv_scale, nbbase, t, E, L.halo_tab, any_missing,
                 ghost_row, r, [&]() { fill_missing_flow<ST>(L, nbbase, b, t, E); });
}

// obs / spg: this cell's obstacle flag and sponge weight, loaded by the
// caller before staging so that their latency overlaps it.
// The 27 pulls of cell t from the staged windows.
__device__ __forceinline__ void load_pulls(const float *E, int t, float (&A)[27]) {
  const int eb = e_index(t & 7, (t >> 3) & 7, t >> 6);
#pragma unroll
  for (int k = 0; k < 27; ++k)
    A[k] = E[k * EPL + eb - (cx_of(k) + 10 * cy_of(k) + 100 * cz_of(k))];
}

// Per-cell inputs a caller may have read ahead of the collision (the
// warp-specialised kernel issues them before its shared-memory pulls):
// the wall distance and the WALE neighbour velocities.
struct CellAux {
  float wall_dist;
  WaleVel wale;
};

// collide_cell's stores: populations (and the optional post-collision copy)
// and rho, u, straight to the level's arrays.
template <class ST>
struct GlobalOut {
  const LevelDev &L;
  size_t own;
  float *fpost;
  __device__ __forceinline__ GlobalOut(const LevelDev &L_, size_t own_)
      : L(L_), own(own_), fpost((L_.sp.store_post_collision && L_.f_post) ? L_.f_post : nullptr) {}
  __device__ __forceinline__ void macro(float rho, float ux, float uy, float uz) const {
    L.vel_out[own] = ux;
    L.vel_out[own + L.dstride] = uy;
    L.vel_out[own + 2 * L.dstride] = uz;
    L.rho_out[own] = rho;
  }
  // all 27 populations, A[k] (OPP = false) or the bounce-back A[opp(k)]
  template <bool OPP>
  __device__ __forceinline__ void f_all(const float (&A)[27]) const {
    typename ST::T *fout = (typename ST::T *)L.f_out;
    if (fpost) {
#pragma unroll
      for (int k = 0; k < 27; ++k) {
        const float v = A[OPP ? opp_of(k) : k];
        ST::store(fout, own + (size_t)k * L.dstride, k, L.scale, v);
        fpost[own + (size_t)k * L.dstride] = v;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 27; ++k)
        ST::store(fout, own + (size_t)k * L.dstride, k, L.scale, A[OPP ? opp_of(k) : k]);
    }
  }
};

template <int OP, class ST, bool WALE>
__device__ __forceinline__ void collide_cell(const LevelDev &L, const int *nbbase, float (&A)[27],
                                             int b, int t, bool obs, float spg,
                                             const CellAux *aux = nullptr);

template <int OP, class ST, bool WALE>
__device__ __forceinline__ void stream_collide_cell(const LevelDev &L, const int *nbbase,
                                                    const float *E, int b, int t, bool obs,
                                                    float spg) {
  float A[27];
  load_pulls(E, t, A);
  collide_cell<OP, ST, WALE>(L, nbbase, A, b, t, obs, spg);
}

// Everything after the pull: bounce-back, moments, sponge, wall model,
// WALE, collision, forcing and the stores of cell t of block b.
template <int OP, class ST, bool WALE>
__device__ __forceinline__ void collide_cell(const LevelDev &L, const int *nbbase, float (&A)[27],
                                             int b, int t, bool obs, float spg,
                                             const CellAux *aux) {
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const ol_step_params &sp = L.sp;
  const size_t own = (size_t)nbbase[13] + t;
  const GlobalOut<ST> out(L, own);

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

  if (obs) {
    out.macro(1.0f, 0.0f, 0.0f, 0.0f);
    out.template f_all<true>(A);
    return;
  }
  rho = fmaxf(rho, 0.01f);
  const float inv_rho = 1.0f / rho;
  float ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
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
    wall_force(aux ? aux->wall_dist : L.wall_dist[own], rho, ux, uy, uz, sp.tau_molecular, Fx,
               Fy, Fz);
  const bool forced = (Fx != 0.0f) | (Fy != 0.0f) | (Fz != 0.0f);
  const float uxe = ux + 0.5f * Fx * inv_rho;
  const float uye = uy + 0.5f * Fy * inv_rho;
  const float uze = uz + 0.5f * Fz * inv_rho;

  out.macro(rho, ux, uy, uz);

  float nu_eddy = 0.0f;
  if (WALE) nu_eddy = aux ? wale_from(aux->wale, sp.c_wale) : wale_nu(L, nbbase, x, y, z);
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
  out.template f_all<false>(A);
}

}  // namespace ol
