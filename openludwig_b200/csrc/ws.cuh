// Warp-specialised persistent stream-collide (cumulant operator).
//
// One CTA per SM walks a static share of the work items (blocks of one level
// for the drop-in entry point, (descriptor, block) items for the block pool).
// Its 544 threads have two roles:
//   * 1 producer warp only starts copies.  While the consumers work on item
//     j it reads the neighbour-table row of item j+2 and, once the landing
//     buffer is free again, starts the TMA bulk copies (cp.async.bulk,
//     completion counted in bytes on an mbarrier) of item j+1's contiguous
//     arrays: 27 population planes, 3 velocity planes, sponge, obstacle, wall
//     distance -- 66 KB in FP32, moved without registers or request slots.
//   * 16 consumer warps, one cell per thread, per item: complete the compute
//     stage -- with FP32 storage the population planes landed in it already,
//     each shifted so that every pull is one conflict-free shared load at a
//     compile-time offset (WsLayout); with FP16 storage they decode the
//     landed block into a "pre-streamed" stage (the value cell d pulls in
//     direction k at F[k][d]) -- by writing the out-of-block pull sources
//     each thread loaded for this item one item earlier (a neighbour's value,
//     the precomputed ghost value, or, without a ghost row, pull_boundary as
//     in the one-CTA-per-block kernel) into the slots of the cells that pull
//     them, and the velocities into 10^3 slots per component with a one-cell
//     face halo (a face without neighbour repeats the cell beside it, the
//     zero-gradient fallback of the WALE gradients); then pull, release the
//     buffer the next bulk copies land in, issue the out-of-block loads of
//     item j+1 into registers, collide and store straight to global memory.
//     The next item's bulk copies and out-of-block loads land while they
//     collide.
// Why this split (measured on B200): a block is 66 KB, and an SM has to keep
// ~60-90 KB in flight to draw its share of HBM bandwidth.  Loader warps that
// moved everything themselves -- 4-byte cp.async of every value (too few in
// flight, 128 bytes each), 16-byte loads through their registers (too few
// bytes per round trip), bulk copies they then redistributed (four warps
// cannot hide their own latency), or 4-byte cp.async of just the 3176
// scattered out-of-block values (still ~15k cycles per block) -- all left
// the consumers waiting for data more than half the time.
// Hand-over uses mbarriers ("landed": bulk bytes plus the producer's
// arrival; "free": one arrival per consumer warp) and a named barrier among
// the consumers around the stage.  Every mbarrier wait is bounded in time: a
// wait that runs out sets a bit in the fault word, and the warps give up
// together (consumers through the same named barriers, the producer after
// its copies in flight have landed), so no thread is left at a barrier and
// the kernel always ends.  The staged values are the ones the
// one-CTA-per-block kernel pulls, and the cell update is the same code.
#pragma once
#include "stream_collide.cuh"

namespace ol {

constexpr int kWsProducers = 32;                   // 1 producer warp
constexpr int kWsThreads = BCELLS + kWsProducers;  // 544
constexpr int kWsRing = 4;  // descriptor / neighbour-offset slots (item j uses j & 3)
// Table of the warp-specialised kernel: the kHaloEntries out-of-block pulls
// in the order of the staging table (k | dir << 5 | source cell << 10 |
// destination cell << 19), then the kWsVelEntries face-halo velocity slots
// (face dir | own cell beside the slot << 5).
constexpr int kWsVelEntries = 6 * 64;
constexpr int kWsTableSize = kHaloEntries + kWsVelEntries;
// ... then, per out-of-block pull i, the index of the FP32 compute-stage slot
// it is written to (k * kSPlane + kSPad + destination cell - c_x(k); below)
constexpr int kWsSlotOffset = kWsTableSize;
constexpr int kWsTableTotal = kWsTableSize + kHaloEntries;
// Dynamic shared memory (byte offsets).
// FP32 storage ("direct"): the bulk copies land each population plane k
// straight into the compute stage, shifted by 8 c_y + 64 c_z cells, so the
// value cell t pulls in direction k sits at S[k][t - c_x]: no spread of the
// landed block, one conflict-free shared load per pull.  A plane of the stage
// holds 72 + 512 + 72 slots (the shifts reach 72 cells either way; every
// landing address stays 32-byte aligned); the slots whose source lies
// outside the block are then overwritten with the out-of-block values.  The
// stage is the landing buffer, so it is free for the next item once the
// consumers have pulled.  Velocity, sponge, wall distance and mask land
// beside it.
// FP16-shifted storage: the planes land in a buffer of their own and the
// consumers decode them into a pre-streamed stage F[k][d] (the value cell d
// pulls in direction k), releasing the buffer before they pull.
constexpr int kSPad = 72;                         // stage slots before cell 0 (and after 511)
constexpr int kSPlane = kSPad + BCELLS + kSPad;   // 656 floats = 2624 bytes
template <class ST> struct WsLayout;
template <> struct WsLayout<StoreF32> {
  static constexpr bool kDirect = true;
  static constexpr int kS = 0;                                  // float [27][kSPlane]
  static constexpr int kV = kS + 27 * kSPlane * 4;              // float [3][1000]
  static constexpr int kLdV = kV + 3 * EPL * 4;                 // float [3][512]
  static constexpr int kLdSP = kLdV + 3 * BCELLS * 4;           // float [512]
  static constexpr int kLdWD = kLdSP + BCELLS * 4;              // float [512]
  static constexpr int kLdOB = kLdWD + BCELLS * 4;              // uint8 [512]
  static constexpr int kTab = kLdOB + BCELLS;                   // uint32 [kWsTableTotal]
  static constexpr int kBytes = kTab + kWsTableTotal * 4;       // 120,544
  static constexpr int kLdF = 0, kF = 0;                        // (unused)
};
template <> struct WsLayout<StoreF16S> {
  static constexpr bool kDirect = false;
  static constexpr int kLdF = 0;                                // half [27][512]
  static constexpr int kLdV = kLdF + 27 * BCELLS * 4;           // float [3][512]
  static constexpr int kLdSP = kLdV + 3 * BCELLS * 4;           // float [512]
  static constexpr int kLdWD = kLdSP + BCELLS * 4;              // float [512]
  static constexpr int kLdOB = kLdWD + BCELLS * 4;              // uint8 [512]
  static constexpr int kF = kLdOB + BCELLS;                     // float [27][512], pre-streamed
  static constexpr int kV = kF + 27 * BCELLS * 4;               // float [3][1000]
  static constexpr int kTab = kV + 3 * EPL * 4;                 // uint32 [kWsTableTotal]
  static constexpr int kBytes = kTab + kWsTableTotal * 4;       // 160,288
  static constexpr int kS = 0;                                  // (unused)
};
static_assert(WsLayout<StoreF32>::kV % 16 == 0 && WsLayout<StoreF32>::kLdV % 16 == 0 &&
                  WsLayout<StoreF32>::kLdOB % 16 == 0 && (kSPlane * 4) % 32 == 0 &&
                  (kSPad * 4) % 32 == 0,
              "bulk-copy destinations stay 16-byte aligned");
static_assert(WsLayout<StoreF16S>::kF % 16 == 0 && WsLayout<StoreF16S>::kV % 16 == 0,
              "alignment");
template <class ST>
constexpr int ws_smem_bytes() { return WsLayout<ST>::kBytes; }
constexpr int kWsHaloPerConsumer = (kHaloEntries + BCELLS - 1) / BCELLS;  // 7
// A wait that has not completed after this long (ns) is treated as lost.
constexpr unsigned long long kWsWaitNs = 2000000000ull;
// Bits of the fault word.
constexpr int kWsFaultConsumerWait = 1, kWsFaultLoaderWait = 2;

// Per-device loader table (built once; null on failure).
const uint32_t *ws_table_device();

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(
                   smem_addr(bar))
               : "memory");
}
// One arrival once every cp.async this thread has issued so far has landed
// (.noinc: the arrival is part of the barrier's expected count).
__device__ __forceinline__ void mbar_arrive_cp_async(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
      "selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the completion of the phase of `bar` with parity `parity`,
// bounded by kWsWaitNs of wall time and 2^26 polls; false (and `code` set in
// *fault) when the bound runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *fault, int code) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t i = 0; i < (1u << 26); ++i) {
    if (mbar_test(bar, parity)) return true;
    if ((i & 63) == 63 && global_ns() - t0 > kWsWaitNs) break;
  }
  if (fault) atomicOr(fault, code);
  return false;
}

__device__ __forceinline__ void cp_async_4(uint32_t dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_4_if(bool p, uint32_t dst, const void *src) {
  if (p) cp_async_4(dst, src);
}
__device__ __forceinline__ void cp_async_16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Barrier of the 512 consumer threads only (named barrier 1); the AND form
// returns whether all of them passed a non-zero predicate.
__device__ __forceinline__ void consumer_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(BCELLS) : "memory");
}
__device__ __forceinline__ bool consumer_sync_and(int pred) {
  int r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.s32 p, %1, 0; bar.red.and.pred q, 1, %2, p; "
      "selp.s32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"(pred), "n"(BCELLS)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(
                   smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// TMA bulk copy global -> shared (no multicast), completion counted on bar.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// The producer warp's bulk copies of one item into the landing buffer ld
// (lane 0 announces the bytes, then arrives; the bytes complete the phase).
template <class ST, bool WALE>
__device__ __forceinline__ void ws_produce(const LevelDev &L, int b, int lane, unsigned char *ld,
                                           uint64_t *bar) {
  using T = typename ST::T;
  using Lay = WsLayout<ST>;
  constexpr uint32_t kPlane = BCELLS * sizeof(T);
  const int64_t own0 = (L.block_offset + b) * BCELLS;
  const bool wd = L.sp.wall_model_active == 1 && L.wall_dist;
  const T *fin = (const T *)L.f_in;
  const uint32_t bytes = 27 * kPlane + (WALE ? 3 * BCELLS * 4 : 0) + BCELLS * 4 + BCELLS +
                         (wd ? BCELLS * 4 : 0);
  if (lane == 0) mbar_expect_tx(bar, bytes);
  __syncwarp();
  for (int c = lane; c < 33; c += 32) {
    if (c < 27) {
      // direct: plane c shifted by 8 c_y + 64 c_z slots (a multiple of 8)
      unsigned char *dst =
          Lay::kDirect
              ? ld + Lay::kS + (c * kSPlane + kSPad + 8 * cy_of(c) + 64 * cz_of(c)) * 4
              : ld + Lay::kLdF + c * kPlane;
      bulk_copy(dst, fin + (size_t)c * L.dstride + own0, kPlane, bar);
    } else if (c < 30) {
      if (WALE)
        bulk_copy(ld + Lay::kLdV + (c - 27) * BCELLS * 4,
                  L.vel_in + (size_t)(c - 27) * L.dstride + own0, BCELLS * 4, bar);
    } else if (c == 30) {
      bulk_copy(ld + Lay::kLdSP, L.sponge + own0, BCELLS * 4, bar);
    } else if (c == 31) {
      bulk_copy(ld + Lay::kLdOB, L.obstacle + own0, BCELLS, bar);
    } else if (wd) {
      bulk_copy(ld + Lay::kLdWD, L.wall_dist + own0, BCELLS * 4, bar);
    }
  }
}

// Out-of-block pull sources of consumer thread t (table entries t + 512 m)
// and its face-halo velocities (entry t < 384), loaded into registers.
struct HaloRegs {
  float f[kWsHaloPerConsumer];
  float v[3];
};
template <class ST, bool WALE>
__device__ __forceinline__ void ws_halo_load(const LevelDev &L, int b, const int *nbbase, int t,
                                             const uint32_t *tabs, HaloRegs &h) {
  using T = typename ST::T;
  const T *fin = (const T *)L.f_in;
  const float *ghost_row = ghost_row_of(L, b);
#pragma unroll
  for (int m = 0; m < kWsHaloPerConsumer; ++m) {
    const int i = t + BCELLS * m;
    h.f[m] = 0.0f;
    if (i >= kHaloEntries) continue;
    const uint32_t e = tabs[i];
    const int k = e & 31, dir = (e >> 5) & 31, src = (e >> 10) & 511;
    const int nb = nbbase[dir];
    if (nb >= 0) h.f[m] = ST::load(fin, (size_t)k * L.dstride + nb + src, k, L.inv_scale);
    else if (ghost_row) h.f[m] = ghost_row[i];
  }
  if (WALE && t < kWsVelEntries) {
    const uint32_t e = tabs[kHaloEntries + t];
    const int dir = e & 31, oc = (int)(e >> 5);
    const int dx = dir % 3 - 1, dy = (dir / 3) % 3 - 1, dz = dir / 9 - 1;
    const int nb = nbbase[dir];
    const int64_t src = nb >= 0 ? (int64_t)nb + oc - (7 * dx + 56 * dy + 448 * dz)
                                : (L.block_offset + b) * BCELLS + oc;
#pragma unroll
    for (int c = 0; c < 3; ++c) h.v[c] = __ldg(L.vel_in + (size_t)c * L.dstride + src);
  }
}

// Whether the pull of direction k by cell t + c_k stays in the block.
struct CellMask {
  bool xlo, xhi, ylo, yhi, zlo, zhi;  // x > 0, x < 7, y > 0, y < 7, z > 0, z < 7
};
__device__ __forceinline__ bool pull_inside(const CellMask &m, int k) {
  const int cx = cx_of(k), cy = cy_of(k), cz = cz_of(k);
  return (cx == 0 || (cx > 0 ? m.xhi : m.xlo)) && (cy == 0 || (cy > 0 ? m.yhi : m.ylo)) &&
         (cz == 0 || (cz > 0 ? m.zhi : m.zlo));
}
__device__ __forceinline__ float land_value(const unsigned char *ld, int k, int c, float inv_scale,
                                            StoreF16S) {
  const float w = w_of(k);
  return fmaf(__half2float(((const __half *)(ld + WsLayout<StoreF16S>::kLdF))[k * BCELLS + c]),
              w * inv_scale, w);
}
__device__ __forceinline__ float land_value(const unsigned char *, int, int, float, StoreF32) {
  return 0.0f;  // (direct layout: no spread)
}
template <int OP, class ST, bool WALE, bool BATCHED>
__global__ void __launch_bounds__(kWsThreads, 1)
    k_sc_ws(const __grid_constant__ LevelDev L0, const LevelDev *__restrict__ descs,
            const WorkItem *__restrict__ items, int n_items, const uint32_t *__restrict__ tab,
            int *fault) {
  extern __shared__ __align__(16) unsigned char ws_smem[];
  __shared__ __align__(16) LevelDev Ls[BATCHED ? kWsRing : 1];
  __shared__ int nbb[kWsRing][27];
  __shared__ int blk[kWsRing];
  __shared__ __align__(8) uint64_t bars[2];  // landed, free
  uint64_t *const landed = &bars[0], *const lfree = &bars[1];
  unsigned char *const ld = ws_smem;
  using Lay = WsLayout<ST>;
  uint32_t *const tabs = (uint32_t *)(ws_smem + Lay::kTab);
  const int t = threadIdx.x;
  const int n = BATCHED ? n_items : L0.n_blocks;
  const int first = blockIdx.x;
  const int cnt = first < n ? (n - 1 - first) / (int)gridDim.x + 1 : 0;
  if (t == 0) {
    mbar_init(landed, 1);          // the producer's expect_tx arrival + the bulk bytes
    mbar_init(lfree, BCELLS / 32);  // one arrival per consumer warp
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = t; i < kWsTableTotal; i += kWsThreads) tabs[i] = __ldg(tab + i);
  __syncthreads();
  pdl_wait();  // f_in, vel_in, ghost rows: written by the launches before this one

  if (t >= BCELLS) {
    // ------------------------------------------------------------ producer
    const int lane = t - BCELLS;
    // descriptor and neighbour offsets of item p into ring slot p & 3
    auto fetch = [&](int p) {
      const int r = p & (kWsRing - 1);
      const int it = first + p * (int)gridDim.x;
      int b = it;
      if (BATCHED) {
        const WorkItem w = items[it];
        static_assert(sizeof(LevelDev) % 4 == 0, "descriptor copy");
        for (int q = lane; q < (int)(sizeof(LevelDev) / 4); q += 32)
          ((uint32_t *)&Ls[r])[q] = ((const uint32_t *)(descs + w.desc))[q];
        b = w.block;
        __syncwarp();
      }
      const LevelDev &L = BATCHED ? Ls[r] : L0;
      if (lane < 27) {
        const int nb = L.nbr[b + L.nbr_stride * lane];
        nbb[r][lane] = nb > 0 ? (int)((L.block_offset + nb - 1) * BCELLS) : -1;
      }
      if (lane == 0) blk[r] = b;
      __syncwarp();
    };
    // item 0's and item 1's offsets are published with item 0's copies;
    // item j+1's with item j's, so consumers can load ahead
    fetch(0);
    if (cnt > 1) fetch(1);
    int j = 0;
    for (; j < cnt; ++j) {
      const int r = j & (kWsRing - 1);
      if (j >= 1 && j + 1 < cnt) fetch(j + 1);
      // the landing buffer is free once the consumers have spread item j-1
      const bool ok = j == 0 || mbar_wait(lfree, (j - 1) & 1, fault, kWsFaultLoaderWait);
      if (!__all_sync(0xffffffffu, ok)) break;
      if (j > 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const LevelDev &L = BATCHED ? Ls[r] : L0;
      ws_produce<ST, WALE>(L, blk[r], lane, ld, landed);
    }
    // bulk copies still in flight (a loop left early) land before the CTA exits
    if (j > 0 && j < cnt) mbar_wait(landed, (j - 1) & 1, nullptr, 0);
    return;
  }

  // -------------------------------------------------------------- consumers
  float *const F = (float *)(ws_smem + (Lay::kDirect ? Lay::kS : Lay::kF));
  float *const V = (float *)(ws_smem + Lay::kV);
  const int x = t & 7, y = (t >> 3) & 7, z = t >> 6;
  const CellMask cm{x > 0, x < 7, y > 0, y < 7, z > 0, z < 7};
  const int eo = e_index(x, y, z);
  HaloRegs h;
  for (int j = 0; j < cnt; ++j) {
    const int r = j & (kWsRing - 1);
    const bool ok = mbar_wait(landed, j & 1, fault, kWsFaultConsumerWait);
    if (!consumer_sync_and(ok)) break;  // also: every consumer is done pulling item j-1
    const LevelDev &L = BATCHED ? Ls[r] : L0;
    const int *nbase = nbb[r];
    const int b = blk[r];
    if (j == 0) ws_halo_load<ST, WALE>(L, b, nbase, t, tabs, h);
    if constexpr (!Lay::kDirect) {
      // spread the landed block into the pre-streamed stage
#pragma unroll
      for (int k = 0; k < 27; ++k)
        if (pull_inside(cm, k))
          F[k * BCELLS + t + cx_of(k) + 8 * cy_of(k) + 64 * cz_of(k)] =
              land_value(ld, k, t, L.inv_scale, ST{});
    }
    // this thread's out-of-block values into the slots of the cells that pull them
    const bool ghost = ghost_row_of(L, b) != nullptr;
#pragma unroll
    for (int m = 0; m < kWsHaloPerConsumer; ++m) {
      const int i = t + BCELLS * m;
      if (i >= kHaloEntries) continue;
      const uint32_t e = tabs[i];
      const int k = e & 31, dir = (e >> 5) & 31, d = e >> 19;
      const float v = (nbase[dir] >= 0 || ghost)
                          ? h.f[m]
                          : pull_boundary<ST>(L, k, b, d & 7, (d >> 3) & 7, d >> 6);
      if constexpr (Lay::kDirect) F[tabs[kWsSlotOffset + i]] = v;
      else F[k * BCELLS + d] = v;
    }
    if (WALE) {
      const float *lv = (const float *)(ld + Lay::kLdV);
#pragma unroll
      for (int c = 0; c < 3; ++c) V[c * EPL + eo] = lv[c * BCELLS + t];
      if (t < kWsVelEntries) {
        const uint32_t e = tabs[kHaloEntries + t];
        const int dir = e & 31, oc = (int)(e >> 5);
        const int dx = dir % 3 - 1, dy = (dir / 3) % 3 - 1, dz = dir / 9 - 1;
        const int slot = e_index(oc & 7, (oc >> 3) & 7, oc >> 6) + dx + 10 * dy + 100 * dz;
#pragma unroll
        for (int c = 0; c < 3; ++c) V[c * EPL + slot] = h.v[c];
      }
    }
    CellAux aux;
    aux.wall_dist = ((const float *)(ld + Lay::kLdWD))[t];
    const float spg = ((const float *)(ld + Lay::kLdSP))[t];
    const bool obs = ld[Lay::kLdOB + t] != 0;
    if constexpr (!Lay::kDirect) {
      // the landing buffer is read: the producer may fill it with item j+1
      if (j + 1 < cnt) {
        __syncwarp();
        if ((t & 31) == 0) mbar_arrive(lfree);
      }
    }
    consumer_sync();  // the stage holds item j
    float A[27];
    if constexpr (Lay::kDirect) {
#pragma unroll
      for (int k = 0; k < 27; ++k) A[k] = F[k * kSPlane + kSPad + t - cx_of(k)];
      // the stage (also the landing buffer) is read: order these shared-memory
      // accesses before the bulk copies of item j+1, then release it
      if (j + 1 < cnt) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if ((t & 31) == 0) mbar_arrive(lfree);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 27; ++k) A[k] = F[k * BCELLS + t];
    }
    // item j+1's out-of-block values, in flight while item j collides
    if (j + 1 < cnt) {
      const int r1 = (j + 1) & (kWsRing - 1);
      ws_halo_load<ST, WALE>(BATCHED ? Ls[r1] : L0, blk[r1], nbb[r1], t, tabs, h);
    }
    if (WALE) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        aux.wale.e[c] = V[c * EPL + eo + 1];
        aux.wale.w[c] = V[c * EPL + eo - 1];
        aux.wale.n[c] = V[c * EPL + eo + 10];
        aux.wale.s[c] = V[c * EPL + eo - 10];
        aux.wale.t[c] = V[c * EPL + eo + 100];
        aux.wale.b[c] = V[c * EPL + eo - 100];
      }
    }
    collide_cell<OP, ST, WALE>(L, nbase, A, b, t, obs, spg, &aux);
  }
}

}  // namespace ol
