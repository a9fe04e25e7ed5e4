// Bouzidi interpolated bounce-back on the sparse boundary-cell list
// (bouzidi_kernel.jl:13-92), one thread per (boundary cell, direction),
// direction-major so that a warp reads neighbouring cells of one plane.
//
// For each link k of a boundary cell x with q in (q_min, 1]:
//   q <  1/2 : f_out[x, opp k] = 2q f*[x,k] + (1-2q) f*[x + c_opp k, k]
//   q >= 1/2 : f_out[x, opp k] = f*[x,k]/(2q) + (2q-1)/(2q) f*[x, opp k]
// where f* is the post-collision state; a missing x + c_opp k falls back to
// f*[x,k].  The written slot is post-collision / pre-stream, exactly as in
// the reference.
#pragma once
#include "common.cuh"
#include "level_dev.cuh"

namespace ol {

struct BouzDev {
  void *f;              // populations corrected in place (f_out)
  const void *src;      // post-collision source: f_post, or == f (two-phase)
  const uint16_t *q;    // dense [cells*27] (drop-in) or sparse [n_boundary*27]
  int dense_q;
  const int32_t *cell_block;  // 1-based level-local block ids
  const int8_t *cell_x, *cell_y, *cell_z;  // 1-based
  int32_t n_boundary;
  const int32_t *nbr;  int64_t nbr_stride;
  int64_t block_offset, dstride;
  float q_min, scale, inv_scale;
  float *scratch;       // [n_boundary*27] gathered values (two-phase)
  int32_t desc;         // batched: owning level descriptor (f = its f_out / g_out)
  int32_t thermal;      // batched: correct the thermal populations instead
  int64_t scratch_off;  // batched: first scratch slot of this list
  const ol_bouzidi_link *links;  // batched: the level's cut links (level-local cells)
};

__device__ __forceinline__ float half_bits_to_float(uint16_t h) {
  return __half2float(__ushort_as_half(h));
}

// The corrected value from the link's own post-collision f_k and, for
// q < 1/2, f_k of the cell one link further in (fff), else f_opp(k) of the
// cell itself (bouzidi_kernel.jl:60-87).
__device__ __forceinline__ float bouzidi_value(float q, float fk, float fother) {
  if (q < 0.5f) {
    const float c1 = 2.0f * q;
    return c1 * fk + (1.0f - c1) * fother;
  }
  const float inv2q = 1.0f / (2.0f * q);
  const float c2 = (2.0f * q - 1.0f) * inv2q;
  return inv2q * fk + c2 * fother;
}

template <class ST>
__device__ __forceinline__ bool bouzidi_link(const BouzDev &B, int64_t i, int k, size_t &own,
                                             float &val) {
  using T = typename ST::T;
  const int b = B.cell_block[i] - 1;
  const int x = B.cell_x[i] - 1, y = B.cell_y[i] - 1, z = B.cell_z[i] - 1;
  own = (size_t)(B.block_offset + b) * BCELLS + x + BS * y + BS * BS * z;
  const float q = half_bits_to_float(B.dense_q ? B.q[own - (size_t)B.block_offset * BCELLS +
                                                     (size_t)k * B.dstride]
                                               : B.q[i * 27 + k]);
  if (!(q > B.q_min && q <= 1.0f)) return false;
  const int ko = opp_of(k);
  const T *src = (const T *)B.src;
  const float fk = ST::load(src, own + (size_t)k * B.dstride, k, B.inv_scale);
  if (q < 0.5f) {
    // x_ff = x + c_opp(k) = x - c_k
    const int nx = x - cx_of(k), ny = y - cy_of(k), nz = z - cz_of(k);
    float fff = fk;
    if (nx >= 0 && nx < BS && ny >= 0 && ny < BS && nz >= 0 && nz < BS) {
      fff = ST::load(src, (size_t)(B.block_offset + b) * BCELLS + nx + BS * ny + BS * BS * nz +
                              (size_t)k * B.dstride,
                     k, B.inv_scale);
    } else {
      const int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0);
      const int oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0);
      const int oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
      const int nb = B.nbr[b + B.nbr_stride * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))];
      if (nb > 0)
        fff = ST::load(src, (size_t)(B.block_offset + nb - 1) * BCELLS + (nx & 7) +
                                BS * (ny & 7) + BS * BS * (nz & 7) + (size_t)k * B.dstride,
                       k, B.inv_scale);
    }
    val = bouzidi_value(q, fk, fff);
  } else {
    val = bouzidi_value(q, fk, ST::load(src, own + (size_t)ko * B.dstride, ko, B.inv_scale));
  }
  return true;
}

// ---------------------------------------------------------------------------
// Link lists: the (cell, direction) pairs whose q lies in (q_min, 1] are
// static for a level, so they are compacted once (k_bouzidi_build_links)
// and each step touches only them: a gather over the links into scratch,
// then a scatter, with the same arithmetic as above.  Cells are level-local
// (block_offset * 512 is added when the list is applied); far_cell is the
// cell x - c_k for q < 1/2, -1 when that neighbour block is absent (the
// value then falls back to f_k) or when q >= 1/2.
// ---------------------------------------------------------------------------
template <class ST>
__global__ void k_bouzidi_links_gather(const void *f_v, const ol_bouzidi_link *__restrict__ links,
                                       int32_t n_links, int64_t cell0, int64_t dstride,
                                       float inv_scale, float *__restrict__ scratch) {
  pdl_wait();  // f: written by the stream-collide launch before
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n_links) return;
  using T = typename ST::T;
  const T *f = (const T *)f_v;
  const ol_bouzidi_link L = links[l];
  const int k = L.k;
  const size_t own = (size_t)(cell0 + L.cell);
  const float fk = ST::load(f, own + (size_t)k * dstride, k, inv_scale);
  float fother;
  if (L.q < 0.5f)
    fother = L.far_cell >= 0 ? ST::load(f, (size_t)(cell0 + L.far_cell) + (size_t)k * dstride, k,
                                        inv_scale)
                             : fk;
  else
    fother = ST::load(f, own + (size_t)opp_of(k) * dstride, opp_of(k), inv_scale);
  scratch[l] = bouzidi_value(L.q, fk, fother);
}

template <class ST>
__global__ void k_bouzidi_links_scatter(void *f_v, const ol_bouzidi_link *__restrict__ links,
                                        int32_t n_links, int64_t cell0, int64_t dstride,
                                        float scale, const float *__restrict__ scratch) {
  pdl_wait();  // scratch: filled by the gather launch before
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n_links) return;
  const ol_bouzidi_link L = links[l];
  const int ko = opp_of(L.k);
  ST::store((typename ST::T *)f_v, (size_t)(cell0 + L.cell) + (size_t)ko * dstride, ko, scale,
            scratch[l]);
}

// Single phase: src != f (reference semantics with a post-collision copy).
template <class ST>
__global__ void k_bouzidi_direct(const __grid_constant__ BouzDev B) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int64_t)B.n_boundary * 27) return;
  const int k = (int)(j / B.n_boundary);  // direction-major: neighbouring threads
  const int64_t i = j - (int64_t)k * B.n_boundary;  // take neighbouring cells
  size_t own;
  float v;
  if (bouzidi_link<ST>(B, i, k, own, v))
    ST::store((typename ST::T *)B.f, own + (size_t)opp_of(k) * B.dstride, opp_of(k), B.scale, v);
}

// Two phases on one buffer: gather every corrected value first ...
template <class ST>
__global__ void k_bouzidi_gather(const __grid_constant__ BouzDev B) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int64_t)B.n_boundary * 27) return;
  const int k = (int)(j / B.n_boundary);  // direction-major: neighbouring threads
  const int64_t i = j - (int64_t)k * B.n_boundary;  // take neighbouring cells
  size_t own;
  float v;
  if (bouzidi_link<ST>(B, i, k, own, v)) B.scratch[j] = v;
}

// ... then scatter them, so no link reads a slot another link replaced.
template <class ST>
__global__ void k_bouzidi_scatter(const __grid_constant__ BouzDev B) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int64_t)B.n_boundary * 27) return;
  const int k = (int)(j / B.n_boundary);  // direction-major: neighbouring threads
  const int64_t i = j - (int64_t)k * B.n_boundary;  // take neighbouring cells
  const int b = B.cell_block[i] - 1;
  const int x = B.cell_x[i] - 1, y = B.cell_y[i] - 1, z = B.cell_z[i] - 1;
  const size_t own = (size_t)(B.block_offset + b) * BCELLS + x + BS * y + BS * BS * z;
  const float q = half_bits_to_float(B.dense_q ? B.q[own - (size_t)B.block_offset * BCELLS +
                                                     (size_t)k * B.dstride]
                                               : B.q[i * 27 + k]);
  if (!(q > B.q_min && q <= 1.0f)) return;
  ST::store((typename ST::T *)B.f, own + (size_t)opp_of(k) * B.dstride, opp_of(k), B.scale,
            B.scratch[j]);
}

void launch_bouzidi(const BouzDev &B, bool f16, cudaStream_t s);

}  // namespace ol
