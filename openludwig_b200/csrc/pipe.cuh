// Software-pipelined stream-collide: persistent 512-thread CTAs (two per SM
// for the cumulant operator) each walk a share of the blocks with ONE
// staging buffer.  A cell's 27 pulls are read from the buffer into registers
// first; once every thread has them the buffer is free, so the asynchronous
// copies (cp.async) of the next block's pull windows -- and the boundary
// values of its absent neighbours -- are issued before the current block's
// collision and land while it computes.  The memory latency of block i+1
// hides behind the arithmetic of block i without a second buffer, so two
// CTAs (2 x 105 KB) still fit per SM.
#pragma once
#include "stream_collide.cuh"

namespace ol {

constexpr int kPipeBytes = kStageBytes;

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

// Issue the asynchronous copies of block b's pull windows into E (FP32
// storage).  Returns whether the slots of absent neighbours still need their
// boundary values (fill_missing_flow): the caller runs that fill where no
// cell's pulls are live in registers, since it is a call.
__device__ __forceinline__ bool issue_stage_f32(const LevelDev &L, const int *nbbase, int b, int t,
                                                float *E, bool any_missing) {
  const float *fin = (const float *)L.f_in;
  const int own = nbbase[13];
  const int eb = e_index(t & 7, (t >> 3) & 7, t >> 6);
  const float *src = fin + own + t;
  const uint32_t *tab = L.halo_tab;
#pragma unroll
  for (int k = 0; k < 27; ++k) cp_async4(E + k * EPL + eb, src + (size_t)k * L.dstride);
  const float *ghost_row = ghost_row_of(L, b);
  // one table entry at a time: this runs while a cell's pulls are held in
  // registers, so it keeps its own register footprint small
#pragma unroll 1
  for (int i = t; i < kHaloEntries; i += BCELLS) {
    const uint32_t te = __ldg(tab + i);
    const int k = te & 31, dir = (te >> 5) & 31, s = (te >> 10) & 511, dst = te >> 19;
    const int nb = nbbase[dir];
    if (nb >= 0) cp_async4(E + k * EPL + dst, fin + (size_t)k * L.dstride + nb + s);
    else if (ghost_row) cp_async4(E + k * EPL + dst, ghost_row + i);
  }
  cp_async_commit();
  return any_missing && !ghost_row;
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
// The per-item descriptor and neighbour offsets rotate through three slots:
// the slot fetched in iteration i was last read by the collision of
// iteration i-2, which every thread finished before iteration i-1's barriers.
template <int OP, bool WALE, bool BATCHED>
__global__ void __launch_bounds__(512, OP == OL_OP_CUMULANT ? 2 : 1)
    k_sc_pipe(const __grid_constant__ LevelDev L0, const LevelDev *__restrict__ descs,
              const WorkItem *__restrict__ items, int n_items) {
  extern __shared__ float E[];
  __shared__ __align__(16) LevelDev Ls[BATCHED ? 3 : 1];
  __shared__ int nbb[3][27];
  const int t = threadIdx.x;
  const int n = BATCHED ? n_items : L0.n_blocks;
  int it = blockIdx.x;
  if (it >= n) return;
  // descriptor + neighbour offsets of `item` into slot s (ends with a barrier)
  auto fetch = [&](int s, int item, int &blk) -> bool {
    blk = item;
    if (BATCHED) {
      const WorkItem w = items[item];
      copy_words(&Ls[s], descs + w.desc, t);
      blk = w.block;
      __syncthreads();
    }
    const LevelDev &L = BATCHED ? Ls[s] : L0;
    return load_nbbase_sync(L.nbr, L.nbr_stride, L.block_offset, blk, t, nbb[s]);
  };
  int cur = 0, blk = 0;
  const bool miss0 = fetch(0, it, blk);
  if (issue_stage_f32(BATCHED ? Ls[0] : L0, nbb[0], blk, t, E, miss0))
    fill_missing_flow<StoreF32>(BATCHED ? Ls[0] : L0, nbb[0], blk, t, E);
  for (;;) {
    const LevelDev &Lc = BATCHED ? Ls[cur] : L0;
    const size_t own = (size_t)nbb[cur][13] + t;
    const bool obs = Lc.obstacle[own] != 0;
    const float spg = Lc.sponge[own];
    const int nxt = it + gridDim.x;
    const int sn = cur == 2 ? 0 : cur + 1;
    int nblk = -1;
    bool nmiss = false;
    if (nxt < n) nmiss = fetch(sn, nxt, nblk);
    cp_async_wait<0>();
    __syncthreads();  // block blk staged
    float A[27];
    load_pulls(E, t, A);
    __syncthreads();  // staging buffer free
    bool fill = false;
    if (nxt < n) fill = issue_stage_f32(BATCHED ? Ls[sn] : L0, nbb[sn], nblk, t, E, nmiss);
    collide_cell<OP, StoreF32, WALE>(Lc, nbb[cur], A, blk, t, obs, spg);
    if (nxt >= n) break;
    if (fill) fill_missing_flow<StoreF32>(BATCHED ? Ls[sn] : L0, nbb[sn], nblk, t, E);
    it = nxt;
    blk = nblk;
    cur = sn;
  }
}

}  // namespace ol
