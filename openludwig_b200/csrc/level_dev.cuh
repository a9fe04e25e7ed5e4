// Device-side description of one level sub-step and the population storage
// formats.  Both the drop-in entry points (caller-owned buffers in the
// reference layout) and the batched block-pool executor fill a LevelDev, so a
// single set of cell kernels serves both.
#pragma once
#include "lattice.cuh"
#include "../../include/openludwig_b200.h"

namespace ol {

// Storage of populations.  F32 is the reference format.  F16S stores the
// binary16 value of (f_k - w_k) * (scale / w_k): the shifted, direction-
// normalised deviation, so every direction uses the same range and a
// per-level power-of-two `scale` keeps small deviations out of subnormals.
// All arithmetic stays FP32; only the stored bytes shrink.
struct StoreF32 {
  using T = float;
  static constexpr int kBytes = 4;
  __device__ __forceinline__ static float load(const T *p, size_t i, int /*k*/,
                                               float /*scale*/) {
    return __ldg(p + i);
  }
  __device__ __forceinline__ static void store(T *p, size_t i, int /*k*/,
                                               float /*scale*/, float v) {
    p[i] = v;
  }
};

struct StoreF16S {
  using T = __half;
  static constexpr int kBytes = 2;
  __device__ __forceinline__ static float load(const T *p, size_t i, int k,
                                               float inv_scale) {
    const float w = w_of(k);
    return fmaf(__half2float(__ldg(p + i)), w * inv_scale, w);
  }
  __device__ __forceinline__ static void store(T *p, size_t i, int k,
                                               float scale, float v) {
    // scale * (1/w) with the reciprocal folded at compile time: the same
    // bits as scale / w for the power-of-two scales the layer uses
    const float w = w_of(k);
    p[i] = __float2half_rn((v - w) * (scale * (1.0f / w)));
  }
};

// One level sub-step.  Every per-cell array of the level is addressed as
// base[(block_offset + b) * 512 + cell + c * dstride] for 0-based local block
// b; neighbour tables and block pointers hold 1-based local ids (0 = none).
struct LevelDev {
  const void *f_in;  void *f_out;  float *f_post;
  float *rho_out;  float *vel_out;  const float *vel_in;
  const uint8_t *obstacle;  const float *sponge;  const float *wall_dist;
  const int32_t *nbr;  const int32_t *map_x, *map_y, *map_z;
  int32_t n_blocks;
  int64_t block_offset;   // first block of this level in its arrays
  int64_t dstride;        // elements between consecutive directions/components
  int64_t nbr_stride;     // rows of the neighbour table (nB of its allocation)
  float scale, inv_scale; // FP16 shift scale of this level

  // parent level (coarse-to-fine interpolation)
  const void *pf;  const float *prho;  const float *pvel;
  const void *pf_old;  const float *prho_old;  const float *pvel_old;
  const int32_t *pptr;  int32_t pdim_x, pdim_y, pdim_z;
  int64_t p_block_offset, p_dstride;
  float p_inv_scale;

  ol_step_params sp;
  int32_t *status;        // device watchdog word (may be null)
  const uint32_t *halo_tab;  // staging table (stream_collide.cuh)
  float *ghost;           // absent-neighbour pull sources, kHaloEntries per row, or null
  const int32_t *gidx;    // block -> ghost row (-1: none); null = row b for block b
  // Pairing of the two child sub-steps of one parent step (kGhost* below):
  // 1 = this first sub-step also writes the second one's coarse-to-fine
  // values into ghost_next (same row layout); 2 = ghost already holds them
  // and only the domain-boundary slots are evaluated; 0 = no pairing.
  float *ghost_next;
  int32_t ghost_mode;
  const int32_t *gblocks;  // blocks the drop-in ghost pass visits (null = all)
  int32_t n_gblocks;
  int32_t prefetch_ahead;  // stream-collide: L2-prefetch block b + this (0 = off)
};

constexpr int kGhostUnpaired = 0, kGhostPairFirst = 1, kGhostPairSecond = 2;
// temporal weight of the second child sub-step (solver_control.jl:65-97)
constexpr float kSecondSubstepWeight = 0.5f;

// One unit of batched work: block `block` of the level described by
// descriptor `desc`.
struct WorkItem {
  int32_t desc;
  int32_t block;
};

// Per-device staging table of the 3176 out-of-block pull sources of a block
// (built once on first use; see stage_block).
const uint32_t *halo_table_device();
// Per-device fault word of the warp-specialised kernels (null on failure).
int *fault_word_device();
// Current ol_set_stream_collide_kernel choice (OL_SC_KERNEL_*).
int stream_collide_kernel_choice();
// Grid of a warp-specialised launch over n_items work items.
int ws_grid(int64_t n_items, int n_sm);

}  // namespace ol
