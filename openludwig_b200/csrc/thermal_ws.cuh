// Warp-specialised persistent kernel for the thermal populations
// (kernel_thermal.jl:14-202), FP32 storage, drop-in levels.
//
// The same structure as k_sc_ws (ws.cuh): one CTA per SM walks a static share
// of the level's blocks; one producer warp bulk-copies each block's 27 g
// planes straight into the compute stage at their pull shifts (slot
// k * kSPlane + kSPad + t - c_x holds the value cell t pulls in direction k),
// and its flow velocity (this sub-step's u), sponge weight and solid mask
// beside it; 16 consumer warps write the out-of-block pull sources they
// loaded one block earlier (a neighbour's g, the precomputed ghost value, or
// pull_boundary_thermal) into the slots of the cells that pull them, pull,
// release the stage to the next copies and run the passive-scalar BGK update.
// The update is light (about 990 instructions per cell), too short to hide a
// block's copies behind the previous block's update, so there are two stages:
// block j+1 lands while block j is pulled and updated.  The one-CTA-per-block
// kernel stages through registers instead.
// A solid cell bounces its own unstreamed g back (adiabatic or isothermal
// wall); the stage does not keep a cell's own values once the out-of-block
// sources are written, so a solid cell reads them from global memory.
#pragma once
#include "thermal.cuh"
#include "ws.cuh"

namespace ol {

// Dynamic shared memory (bytes): two buffers, so that two blocks are in
// flight per SM (the update is too short to hide one block's copies), each
// a stage with the velocity, sponge and mask beside it; then the table.
constexpr int kTwS = 0;                                // float [27][kSPlane]
constexpr int kTwLdV = kTwS + 27 * kSPlane * 4;        // float [3][512] flow velocity
constexpr int kTwLdSP = kTwLdV + 3 * BCELLS * 4;       // float [512]
constexpr int kTwLdOB = kTwLdSP + BCELLS * 4;          // uint8 [512]
constexpr int kTwBuf = kTwLdOB + BCELLS;               // bytes per buffer (79,552)
constexpr int kTwTab = 2 * kTwBuf;                     // uint32 [kWsTableTotal]
constexpr int kTwBytes = kTwTab + kWsTableTotal * 4;   // 186,048
constexpr int kTwRing = 8;                             // descriptor slots (block j uses j & 7)
static_assert(kTwLdV % 16 == 0 && kTwLdSP % 16 == 0 && kTwLdOB % 16 == 0 && kTwBuf % 16 == 0,
              "bulk-copy destinations stay 16-byte aligned");

// The producer's bulk copies of block b into the stage (lane 0 announces the
// bytes, then arrives).
__device__ __forceinline__ void tws_produce(const ThermalDev &D, int b, int lane,
                                            unsigned char *sm, uint64_t *bar) {
  constexpr uint32_t kPlane = BCELLS * 4;
  const int64_t own0 = (D.block_offset + b) * BCELLS;
  const float *gin = (const float *)D.g_in;
  if (lane == 0) mbar_expect_tx(bar, 27 * kPlane + 3 * kPlane + kPlane + BCELLS);
  __syncwarp();
  const int c = lane;  // 32 copies, one per lane
  if (c < 27) {
    bulk_copy(sm + kTwS + (c * kSPlane + kSPad + 8 * cy_of(c) + 64 * cz_of(c)) * 4,
              gin + (size_t)c * D.dstride + own0, kPlane, bar);
  } else if (c < 30) {
    bulk_copy(sm + kTwLdV + (c - 27) * kPlane, D.vel + (size_t)(c - 27) * D.dstride + own0,
              kPlane, bar);
  } else if (c == 30) {
    bulk_copy(sm + kTwLdSP, D.sponge + own0, kPlane, bar);
  } else {
    bulk_copy(sm + kTwLdOB, D.obstacle + own0, BCELLS, bar);
  }
}

// Out-of-block pull sources of consumer thread t (loader-table entries
// t + 512 m) for block b, into registers.
__device__ __forceinline__ void tws_halo_load(const ThermalDev &D, int b, const int *nbbase,
                                              int t, const uint32_t *tabs,
                                              float (&h)[kWsHaloPerConsumer]) {
  const float *gin = (const float *)D.g_in;
  const float *ghost_row = ghost_row_of(D, b);
#pragma unroll
  for (int m = 0; m < kWsHaloPerConsumer; ++m) {
    const int i = t + BCELLS * m;
    h[m] = 0.0f;
    if (i >= kHaloEntries) continue;
    const uint32_t e = tabs[i];
    const int k = e & 31, dir = (e >> 5) & 31, src = (e >> 10) & 511;
    const int nb = nbbase[dir];
    if (nb >= 0) h[m] = __ldg(gin + (size_t)k * D.dstride + nb + src);
    else if (ghost_row) h[m] = ghost_row[i];
  }
}

// The BGK update of cell t from its 27 pulled values A (thermal_cell's
// arithmetic, in its order), velocity u, sponge weight and solid flag.
__device__ __forceinline__ void tws_cell(const ThermalDev &D, size_t own, const float (&A)[27],
                                         float ux, float uy, float uz, float spg, bool obs) {
  const ol_thermal_params &tp = D.tp;
  float *__restrict__ gout = (float *)D.g_out;
  float *gpost = (tp.store_post_collision && D.g_post) ? D.g_post : nullptr;
  float Tsum = 0.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) Tsum += A[k];
  if (obs) {
    const float *gin = (const float *)D.g_in;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      const float gopp = __ldg(gin + own + (size_t)opp_of(k) * D.dstride);  // own cell, unstreamed
      float v;
      if (tp.wall_bc_adiabatic == 1) {
        v = gopp;
      } else {
        const float gw = geq(tp.T_wall, 0.0f, 0.0f, 0.0f, w_of(k), (float)cx_of(k),
                             (float)cy_of(k), (float)cz_of(k));
        v = 2.0f * gw - gopp;
      }
      gout[own + (size_t)k * D.dstride] = v;
      if (gpost) gpost[own + (size_t)k * D.dstride] = v;
    }
    D.T_out[own] = tp.wall_bc_adiabatic == 1 ? Tsum : tp.T_wall;
    return;
  }
  float Tl = fmaxf(Tsum, 0.01f);
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
    float gs = A[k];
    if (blend) {
      const float gt = geq(tp.T_inlet, tp.u_inlet, 0.0f, 0.0f, w, cxf, cyf, czf);
      gs = gs * (1.0f - spg) + gt * spg;
    }
    const float ge = geq(Tl, ux, uy, uz, w, cxf, cyf, czf);
    const float gc = gs - og * (gs - ge);
    gout[own + (size_t)k * D.dstride] = gc;
    if (gpost) gpost[own + (size_t)k * D.dstride] = gc;
  }
}

__global__ void __launch_bounds__(kWsThreads, 1)
    k_thermal_ws(const __grid_constant__ ThermalDev D, const uint32_t *__restrict__ tab,
                 int *fault) {
  extern __shared__ __align__(16) unsigned char tw_smem[];
  // neighbour offsets and block of block p in slot p & (kTwRing - 1): the
  // producer fetches block j+1 before waiting for buffer j & 1, while the
  // consumers may still be finishing block j-3
  __shared__ int nbb[kTwRing][27];
  __shared__ int blk[kTwRing];
  // per buffer: "landed" (bulk bytes plus the producer's arrival), "free"
  // (one arrival per consumer warp); block j uses buffer j & 1, and its
  // (j >> 1)-th phase of each
  __shared__ __align__(8) uint64_t bars[4];
  uint64_t *const landed = &bars[0], *const lfree = &bars[2];
  uint32_t *const tabs = (uint32_t *)(tw_smem + kTwTab);
  const int t = threadIdx.x;
  const int n = D.n_blocks;
  const int first = blockIdx.x;
  const int cnt = first < n ? (n - 1 - first) / (int)gridDim.x + 1 : 0;
  if (t == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(landed + i, 1);
      mbar_init(lfree + i, BCELLS / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = t; i < kWsTableTotal; i += kWsThreads) tabs[i] = __ldg(tab + i);
  __syncthreads();

  if (t >= BCELLS) {
    // ------------------------------------------------------------ producer
    const int lane = t - BCELLS;
    auto fetch = [&](int p) {
      const int r = p & (kTwRing - 1);
      const int b = first + p * (int)gridDim.x;
      if (lane < 27) {
        const int nb = D.nbr[b + D.nbr_stride * lane];
        nbb[r][lane] = nb > 0 ? (int)((D.block_offset + nb - 1) * BCELLS) : -1;
      }
      if (lane == 0) blk[r] = b;
      __syncwarp();
    };
    fetch(0);
    if (cnt > 1) fetch(1);
    int j = 0;
    for (; j < cnt; ++j) {
      const int r = j & (kTwRing - 1), bi = j & 1;
      if (j >= 1 && j + 1 < cnt) fetch(j + 1);
      // buffer bi is free once the consumers have pulled block j-2
      const bool ok =
          j < 2 || mbar_wait(lfree + bi, ((j - 2) >> 1) & 1, fault, kWsFaultLoaderWait);
      if (!__all_sync(0xffffffffu, ok)) break;
      if (j >= 2) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tws_produce(D, blk[r], lane, tw_smem + bi * kTwBuf, landed + bi);
    }
    // bulk copies still in flight (a loop left early) land before the CTA exits
    if (j < cnt)
      for (int i = j >= 2 ? j - 2 : 0; i < j; ++i)
        mbar_wait(landed + (i & 1), (i >> 1) & 1, nullptr, 0);
    return;
  }

  // -------------------------------------------------------------- consumers
  float h[kWsHaloPerConsumer];
  for (int j = 0; j < cnt; ++j) {
    const int r = j & (kTwRing - 1), bi = j & 1;
    unsigned char *const buf = tw_smem + bi * kTwBuf;
    float *const F = (float *)(buf + kTwS);
    const bool ok = mbar_wait(landed + bi, (j >> 1) & 1, fault, kWsFaultConsumerWait);
    if (!consumer_sync_and(ok)) break;  // also: every consumer is done pulling block j-1
    const int *nbase = nbb[r];
    const int b = blk[r];
    if (j == 0) tws_halo_load(D, b, nbase, t, tabs, h);
    const bool ghost = ghost_row_of(D, b) != nullptr;
#pragma unroll
    for (int m = 0; m < kWsHaloPerConsumer; ++m) {
      const int i = t + BCELLS * m;
      if (i >= kHaloEntries) continue;
      const uint32_t e = tabs[i];
      const int k = e & 31, dir = (e >> 5) & 31, d = e >> 19;
      const float v = (nbase[dir] >= 0 || ghost)
                          ? h[m]
                          : pull_boundary_thermal<StoreF32>(D, k, b, d & 7, (d >> 3) & 7, d >> 6);
      F[tabs[kWsSlotOffset + i]] = v;
    }
    const float *const lv = (const float *)(buf + kTwLdV);
    const float ux = lv[t], uy = lv[BCELLS + t], uz = lv[2 * BCELLS + t];
    const float spg = ((const float *)(buf + kTwLdSP))[t];
    const bool obs = buf[kTwLdOB + t] != 0;
    consumer_sync();  // the stage holds block j
    float A[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) A[k] = F[k * kSPlane + kSPad + t - cx_of(k)];
    // the buffer is read: order these accesses before its next bulk copies
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if ((t & 31) == 0) mbar_arrive(lfree + bi);
    if (j + 1 < cnt) {
      const int r1 = (j + 1) & (kTwRing - 1);
      tws_halo_load(D, blk[r1], nbb[r1], t, tabs, h);
    }
    tws_cell(D, (size_t)nbase[13] + t, A, ux, uy, uz, spg, obs);
  }
}

}  // namespace ol
