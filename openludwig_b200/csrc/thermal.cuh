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
};

// Coarse-to-fine thermal ghost (physics_interpolation.jl:135-247).
template <class ST>
__device__ __noinline__ float interp_parent_thermal(const ThermalDev &D, int k, int gx,
                                                    int gy, int gz) {
  const ol_thermal_params &tp = D.tp;
  const float w = w_of(k);
  const float cx = (float)cx_of(k), cy = (float)cy_of(k), cz = (float)cz_of(k);
  const float pxc = ((float)gx - 0.5f) * 0.5f;
  const float pyc = ((float)gy - 0.5f) * 0.5f;
  const float pzc = ((float)gz - 0.5f) * 0.5f;
  int px0 = (int)floorf(pxc), py0 = (int)floorf(pyc), pz0 = (int)floorf(pzc);
  const int px1 = px0 + 1, py1 = py0 + 1, pz1 = pz0 + 1;
  const float wx = pxc - (float)px0, wy = pyc - (float)py0, wz = pzc - (float)pz0;
  px0 = max(1, px0); py0 = max(1, py0); pz0 = max(1, pz0);
  const bool temporal = tp.use_temporal_interp == 1 && tp.temporal_weight < 0.99f;
  const float tw = tp.temporal_weight;
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
    if (pbx >= 1 && pbx <= D.pdim_x && pby >= 1 && pby <= D.pdim_y && pbz >= 1 &&
        pbz <= D.pdim_z) {
      const int pb = D.pptr[(pbx - 1) + D.pdim_x * ((pby - 1) + D.pdim_y * (pbz - 1))];
      if (pb > 0) {
        const int cell = (pgx - 1) % BS + BS * ((pgy - 1) % BS) + BS * BS * ((pgz - 1) % BS);
        const size_t ci = (size_t)(D.p_block_offset + pb - 1) * BCELLS + cell;
        const float gn = ST::load((const typename ST::T *)D.pg, ci + (size_t)k * D.p_dstride, k,
                                  D.p_inv_scale);
        const float Tn = D.pT[ci];
        const float uxn = D.pvel[ci], uyn = D.pvel[ci + D.p_dstride],
                    uzn = D.pvel[ci + 2 * D.p_dstride];
        if (temporal) {
          const float go = ST::load((const typename ST::T *)D.pg_old,
                                    ci + (size_t)k * D.p_dstride, k, D.p_inv_scale);
          const float To = D.pT_old[ci];
          const float uxo = D.pvel_old[ci], uyo = D.pvel_old[ci + D.p_dstride],
                      uzo = D.pvel_old[ci + 2 * D.p_dstride];
          v[s][0] = go * (1.0f - tw) + gn * tw;
          v[s][1] = To * (1.0f - tw) + Tn * tw;
          v[s][2] = uxo * (1.0f - tw) + uxn * tw;
          v[s][3] = uyo * (1.0f - tw) + uyn * tw;
          v[s][4] = uzo * (1.0f - tw) + uzn * tw;
        } else {
          v[s][0] = gn; v[s][1] = Tn; v[s][2] = uxn; v[s][3] = uyn; v[s][4] = uzn;
        }
        ok[s] = true;
      }
    }
  }
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
  const float ge = geq(r[1], r[2], r[3], r[4], w, cx, cy, cz);
  const float gneq = r[0] - ge;
  const float tc = tp.tau_g_parent - 0.5f, tf = tp.tau_g - 0.5f;
  const float sc = tc > 1e-6f ? fminf(fmaxf(tf / tc, 0.01f), 100.0f) : 1.0f;
  return ge + gneq * sc;
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

// Stage the thermal populations of block b (same layout as the flow).
template <class ST>
__device__ __forceinline__ void stage_thermal(const ThermalDev &D, const int *nbbase, int b, int t,
                                              float *E, const uint32_t *tab, bool any_missing) {
  const ThermalDev *Dp = &D;
  stage_block<ST>(D.g_in, D.dstride, D.inv_scale, nbbase, t, E, tab, any_missing, nullptr, [&]() {
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
