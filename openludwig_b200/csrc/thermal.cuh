// Thermal double-distribution stream-collide (kernel_thermal.jl:14-202):
// passive-scalar BGK for 27 populations g driven by this sub-step's flow
// velocity.  One CTA per block, one thread per cell, pull windows staged in
// shared memory exactly as for the flow populations.
#pragma once
#include "stream_collide.cuh"

namespace ol {

struct ThermalDev {
  const void *g_in;  void *g_out;  float *g_post;
  float *T_out;  const float *vel;  const uint8_t *obstacle;  const float *sponge;
  const int32_t *nbr;  const int32_t *map_x, *map_y, *map_z;
  int32_t n_blocks;
  int64_t block_offset, dstride, nbr_stride;
  float scale, inv_scale;
  const void *pg;  const float *pT, *pvel;  const void *pg_old;  const float *pT_old, *pvel_old;
  const int32_t *pptr;  int32_t pdim_x, pdim_y, pdim_z;
  int64_t p_block_offset, p_dstride;
  float p_inv_scale;
  ol_thermal_params tp;
  const uint32_t *halo_tab;
  float *ghost;            // absent-neighbour pull sources, kHaloEntries per row, or null
  const int32_t *gidx;     // block -> ghost row (-1: none); null = row b for block b
  float *ghost_next;       // as LevelDev::ghost_next / ghost_mode
  int32_t ghost_mode;
  const int32_t *gblocks;  // as LevelDev::gblocks / n_gblocks
  int32_t n_gblocks;
};

// Coarse-to-fine thermal ghost (physics_interpolation.jl:135-247), in the
// parts the ghost pass shares with the flow (stream_collide.cuh): blended
// corner moments (T, u), the blended corner population g_k, trilinear
// weights, then g = g_eq(T, u) + (g - g_eq) * clamp((tau_g - 1/2) /
// (tau_g,parent - 1/2), 0.01, 100).
__device__ __forceinline__ const ol_thermal_params &ghost_params(const ThermalDev &D) {
  return D.tp;
}
// Blended parent T, ux, uy, uz of the present parent cell c at weight tw.
__device__ __forceinline__ void ghost_corner_moments(const ThermalDev &D, uint32_t c, float tw,
                                                     float (&m)[4]) {
  const bool temporal = D.tp.use_temporal_interp == 1 && tw < 0.99f;
  const int64_t S = D.p_dstride;
  const float *vo = D.pvel_old, *vn = D.pvel;
  if (temporal && tw == 0.0f) {   // old state alone (blend_parent)
    m[0] = D.pT_old[c]; m[1] = vo[c]; m[2] = (vo + S)[c]; m[3] = (vo + 2 * S)[c];
    return;
  }
  const float Tn = D.pT[c], uxn = vn[c], uyn = (vn + S)[c], uzn = (vn + 2 * S)[c];
  if (temporal) {
    m[0] = lerp_rn(D.pT_old[c], Tn, tw);
    m[1] = lerp_rn(vo[c], uxn, tw);
    m[2] = lerp_rn((vo + S)[c], uyn, tw);
    m[3] = lerp_rn((vo + 2 * S)[c], uzn, tw);
  } else {
    m[0] = Tn; m[1] = uxn; m[2] = uyn; m[3] = uzn;
  }
}

__device__ __forceinline__ void ghost_moments(const ThermalDev &D, const ParentStencil &P,
                                              float tw, float (&r)[4]) {
  float v[4][8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    float m[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    if (P.ci[s] >= 0) ghost_corner_moments(D, (uint32_t)P.ci[s], tw, m);
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

// g_eq(T, u) + (g - g_eq) * clamp(...) from the 8 corner values of g_k.
__device__ __forceinline__ float finish_thermal(const ThermalDev &D, int k, const float (&v)[8],
                                                const ParentStencil &P, const float (&r)[4]) {
  const ol_thermal_params &tp = D.tp;
  const float gi = trilerp(v, P.wx, P.wy, P.wz);
  const float ge = geq(r[0], r[1], r[2], r[3], w_of(k), (float)cx_of(k), (float)cy_of(k),
                       (float)cz_of(k));
  const float gneq = gi - ge;
  const float tc = tp.tau_g_parent - 0.5f, tf = tp.tau_g - 0.5f;
  const float sc = tc > 1e-6f ? fminf(fmaxf(tf / tc, 0.01f), 100.0f) : 1.0f;
  return __fadd_rn(ge, __fmul_rn(gneq, sc));
}

template <class ST>
__device__ __forceinline__ float ghost_population(const ThermalDev &D, int k,
                                                  const ParentStencil &P, const float (&r)[4],
                                                  float tw, ST) {
  const bool temporal = D.tp.use_temporal_interp == 1 && tw < 0.99f;
  using T = typename ST::T;
  const T *po = (const T *)D.pg_old + (size_t)k * D.p_dstride;   // plane k
  const T *pn = (const T *)D.pg + (size_t)k * D.p_dstride;
  float v[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    v[s] = w_of(k);
    if (P.ci[s] >= 0) {
      const uint32_t c = (uint32_t)P.ci[s];
      const float go = temporal ? ST::load(po, c, k, D.p_inv_scale) : 0.0f;
      v[s] = blend_parent(temporal, tw, go, [&] { return ST::load(pn, c, k, D.p_inv_scale); });
    }
  }
#pragma unroll
  for (int s = 1; s < 8; ++s)
    if (P.ci[s] < 0) v[s] = v[0];
  return finish_thermal(D, k, v, P, r);
}

// Both child sub-steps of a parent step from one read of the parent's old
// and new g (as interp_population_pair for the flow).
template <class ST>
__device__ __forceinline__ void ghost_population_pair(const ThermalDev &D, int k,
                                                      const ParentStencil &P,
                                                      const float (&r0)[4], const float (&r1)[4],
                                                      ST, float &g0, float &g1) {
  const bool temporal = D.tp.use_temporal_interp == 1;
  using T = typename ST::T;
  const T *po = (const T *)D.pg_old + (size_t)k * D.p_dstride;   // plane k
  const T *pn = (const T *)D.pg + (size_t)k * D.p_dstride;
  float v0[8], v1[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    v0[s] = v1[s] = w_of(k);
    if (P.ci[s] >= 0) {
      const uint32_t c = (uint32_t)P.ci[s];
      const float gn = ST::load(pn, c, k, D.p_inv_scale);
      const float go = temporal ? ST::load(po, c, k, D.p_inv_scale) : gn;
      v0[s] = go;
      v1[s] = temporal ? lerp_rn(go, gn, kSecondSubstepWeight) : gn;
    }
  }
#pragma unroll
  for (int s = 1; s < 8; ++s)
    if (P.ci[s] < 0) { v0[s] = v0[0]; v1[s] = v1[0]; }
  g0 = finish_thermal(D, k, v0, P, r0);
  g1 = finish_thermal(D, k, v1, P, r1);
}

template <class ST>
__device__ __noinline__ float interp_parent_thermal(const ThermalDev &D, int k, int gx,
                                                    int gy, int gz) {
  ParentStencil P;
  parent_stencil(D, gx, gy, gz, P);
  float r[4];
  ghost_moments(D, P, D.tp.temporal_weight, r);
  return ghost_population(D, k, P, r, D.tp.temporal_weight, ST{});
}

// kernel_thermal.jl:90-130
template <class ST>
__device__ __noinline__ float pull_boundary_thermal(const ThermalDev &D, int k, int b, int x,
                                                    int y, int z) {
  const ol_thermal_params &tp = D.tp;
  const int cx = cx_of(k), cy = cy_of(k), cz = cz_of(k);
  const int gx = (D.map_x[b] - 1) * BS + x + 1;
  const int gy = (D.map_y[b] - 1) * BS + y + 1;
  const int gz = (D.map_z[b] - 1) * BS + z + 1;
  const int sgx = gx - cx, sgy = gy - cy, sgz = gz - cz;
  const float w = w_of(k);
  if (sgx < 1 || sgx > tp.nx_global)
    return geq(tp.T_inlet, tp.u_inlet, 0.0f, 0.0f, w, (float)cx, (float)cy, (float)cz);
  const size_t ci = (size_t)(D.block_offset + b) * BCELLS + x + BS * y + BS * BS * z;
  if (sgy < 1 || sgy > tp.ny_global) {
    const int km = mirror_y_of(k);
    return ST::load((const typename ST::T *)D.g_in, ci + (size_t)km * D.dstride, km,
                    D.inv_scale);
  }
  if (sgz < 1 || sgz > tp.nz_global) {
    const int km = mirror_z_of(k);
    return ST::load((const typename ST::T *)D.g_in, ci + (size_t)km * D.dstride, km,
                    D.inv_scale);
  }
  if (tp.is_level_1 == 0) return interp_parent_thermal<ST>(D, k, sgx, sgy, sgz);
  return w * tp.T_inlet;
}

template <class ST>
__device__ __forceinline__ float ghost_boundary(const ThermalDev &D, int k, int b, int x, int y,
                                                int z, ST) {
  return pull_boundary_thermal<ST>(D, k, b, x, y, z);
}

// Stage the thermal populations of block b (same layout as the flow).
template <class ST>
__device__ __forceinline__ void stage_thermal(const ThermalDev &D, const int *nbbase, int b, int t,
                                              float *E, const uint32_t *tab, bool any_missing) {
  const ThermalDev *Dp = &D;
  stage_block<ST>(D.g_in, D.dstride, D.inv_scale, nbbase, t, E, tab, any_missing,
                  ghost_row_of(D, b), [&]() {
    fill_missing_slots(nbbase, t, E, tab, [Dp, b](int k, int x, int y, int z) {
      return pull_boundary_thermal<ST>(*Dp, k, b, x, y, z);
    });
  });
}

template <class ST>
__device__ __forceinline__ void thermal_cell(const ThermalDev &D, const int *nbbase,
                                             const float *E, int b, int t) {
  using T = typename ST::T;
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const ol_thermal_params &tp = D.tp;
  const size_t own = (size_t)nbbase[13] + t;
  T *__restrict__ gout = (T *)D.g_out;
  float ux = D.vel[own], uy = D.vel[own + D.dstride], uz = D.vel[own + 2 * D.dstride];
  const int eb = e_index(x, y, z);
  float G[27];
  float Tsum = 0.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    G[k] = E[k * EPL + eb - (cx_of(k) + 10 * cy_of(k) + 100 * cz_of(k))];
    Tsum += G[k];
  }
  float *gpost = (tp.store_post_collision && D.g_post) ? D.g_post : nullptr;
  if (D.obstacle[own]) {
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      const float gopp = E[opp_of(k) * EPL + eb];  // g_in at this cell, opposite link
      float v;
      if (tp.wall_bc_adiabatic == 1) {
        v = gopp;
      } else {
        const float gw = geq(tp.T_wall, 0.0f, 0.0f, 0.0f, w_of(k), (float)cx_of(k),
                             (float)cy_of(k), (float)cz_of(k));
        v = 2.0f * gw - gopp;
      }
      ST::store(gout, own + (size_t)k * D.dstride, k, D.scale, v);
      if (gpost) gpost[own + (size_t)k * D.dstride] = v;
    }
    D.T_out[own] = tp.wall_bc_adiabatic == 1 ? Tsum : tp.T_wall;
    return;
  }
  float Tl = fmaxf(Tsum, 0.01f);
  const float spg = D.sponge[own];
  if (spg > 0.0f) {
    Tl = Tl * (1.0f - spg) + tp.T_inlet * spg;
    ux = ux * (1.0f - spg) + tp.u_inlet * spg;
    uy = uy * (1.0f - spg);
    uz = uz * (1.0f - spg);
  }
  D.T_out[own] = Tl;
  const float og = 1.0f / fmaxf(tp.tau_g, 0.500001f);
  const bool blend = spg > 0.0f && tp.sponge_blend_distributions == 1;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const float w = w_of(k);
    const float cxf = (float)cx_of(k), cyf = (float)cy_of(k), czf = (float)cz_of(k);
    float gs = G[k];
    if (blend) {
      const float gt = geq(tp.T_inlet, tp.u_inlet, 0.0f, 0.0f, w, cxf, cyf, czf);
      gs = gs * (1.0f - spg) + gt * spg;
    }
    const float ge = geq(Tl, ux, uy, uz, w, cxf, cyf, czf);
    const float gc = gs - og * (gs - ge);
    ST::store(gout, own + (size_t)k * D.dstride, k, D.scale, gc);
    if (gpost) gpost[own + (size_t)k * D.dstride] = gc;
  }
}

void launch_thermal(const ThermalDev &D, bool f16, cudaStream_t s);

}  // namespace ol
