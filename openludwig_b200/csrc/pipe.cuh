// Software-pipelined stream-collide: one persistent 512-thread CTA per SM
// walks its share of the blocks with two staging buffers.  While block i is
// being collided out of buffer i&1, the asynchronous copies (cp.async) of
// block i+1's 27 pull windows are in flight into the other buffer, and the
// boundary values of block i+1's absent neighbours are computed.  One CTA
// per SM leaves 128 registers per thread for the cell update (no spills)
// and 2 x 105 KB of shared memory for the two buffers.
#pragma once
#include "stream_collide.cuh"

namespace ol {

constexpr int kPipeBytes = 2 * kStageBytes;

__device__ __forceinline__ void cp_async4(float *dst_smem, const float *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issue the asynchronous copies of block b's pull windows into E and fill
// the slots of absent neighbours with their boundary values (FP32 storage).
__device__ __forceinline__ void issue_stage_f32(const LevelDev &L, const int *nbbase, int b, int t,
                                                float *E, bool any_missing) {
  const float *fin = (const float *)L.f_in;
  const int own = nbbase[13];
  const int eb = e_index(t & 7, (t >> 3) & 7, t >> 6);
  const float *src = fin + own + t;
  const uint32_t *tab = L.halo_tab;
  uint32_t te[kHaloPerThread];
#pragma unroll
  for (int j = 0; j < kHaloPerThread; ++j) {
    const int i = t + j * BCELLS;
    te[j] = i < kHaloEntries ? __ldg(tab + i) : 0xFFFFFFFFu;
  }
#pragma unroll
  for (int k = 0; k < 27; ++k) cp_async4(E + k * EPL + eb, src + (size_t)k * L.dstride);
  const float *ghost_row = L.ghost ? L.ghost + (size_t)b * kHaloEntries : nullptr;
#pragma unroll
  for (int j = 0; j < kHaloPerThread; ++j) {
    if (te[j] == 0xFFFFFFFFu) continue;
    const int k = te[j] & 31, dir = (te[j] >> 5) & 31, s = (te[j] >> 10) & 511, dst = te[j] >> 19;
    const int nb = nbbase[dir];
    if (nb >= 0) cp_async4(E + k * EPL + dst, fin + (size_t)k * L.dstride + nb + s);
    else if (ghost_row) cp_async4(E + k * EPL + dst, ghost_row + t + j * BCELLS);
  }
  cp_async_commit();
  if (any_missing && !ghost_row) fill_missing_flow<StoreF32>(L, nbbase, b, t, E);
}

template <class DEV>
__device__ __forceinline__ void copy_words(DEV *dst, const DEV *src, int t) {
  static_assert(sizeof(DEV) % 4 == 0, "descriptor size");
  const uint32_t *s = (const uint32_t *)src;
  uint32_t *d = (uint32_t *)dst;
  for (int i = t; i < (int)(sizeof(DEV) / 4); i += blockDim.x) d[i] = s[i];
}

// BATCHED = false: the blocks 0..n_blocks-1 of the level L0 (drop-in).
// BATCHED = true : work items (descriptor, block) from `items`.
template <int OP, bool WALE, bool BATCHED>
__global__ void __launch_bounds__(512, 1)
    k_sc_pipe(const __grid_constant__ LevelDev L0, const LevelDev *__restrict__ descs,
              const WorkItem *__restrict__ items, int n_items) {
  extern __shared__ float smem[];
  __shared__ __align__(16) LevelDev Ls[BATCHED ? 2 : 1];
  __shared__ int nbb[2][27];
  const int t = threadIdx.x;
  const int n = BATCHED ? n_items : L0.n_blocks;
  int it = blockIdx.x;
  if (it >= n) return;
  auto prepare = [&](int buf, int item) -> int {
    int blk = item;
    if (BATCHED) {
      const WorkItem w = items[item];
      copy_words(&Ls[buf], descs + w.desc, t);
      blk = w.block;
      __syncthreads();
    }
    const LevelDev &L = BATCHED ? Ls[buf] : L0;
    const bool miss = load_nbbase_sync(L.nbr, L.nbr_stride, L.block_offset, blk, t, nbb[buf]);
    issue_stage_f32(L, nbb[buf], blk, t, smem + buf * 27 * EPL, miss);
    return blk;
  };
  int blk = prepare(0, it);
  for (int i = 0;; ++i) {
    const int cur = i & 1;
    const int nxt = it + gridDim.x;
    int nblk = -1;
    const LevelDev &Lc = BATCHED ? Ls[cur] : L0;
    const size_t own = (size_t)nbb[cur][13] + t;
    const bool obs = Lc.obstacle[own] != 0;
    const float spg = Lc.sponge[own];
    if (nxt < n) {
      nblk = prepare(cur ^ 1, nxt);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    stream_collide_cell<OP, StoreF32, WALE>(Lc, nbb[cur], smem + cur * 27 * EPL, blk, t, obs,
                                            spg);
    __syncthreads();
    if (nxt >= n) break;
    it = nxt;
    blk = nblk;
  }
}

}  // namespace ol
