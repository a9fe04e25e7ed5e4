// Bouzidi launches and their C ABI (apply_bouzidi_correction!,
// bouzidi_kernel.jl:99-122).
#include "bouzidi.cuh"
#include "common.cuh"

namespace ol {

void launch_bouzidi(const BouzDev &B, bool f16, cudaStream_t s) {
  const int64_t n = (int64_t)B.n_boundary * 27;
  if (n == 0) return;
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (B.src != B.f) {
    if (f16) k_bouzidi_direct<StoreF16S><<<grid, 256, 0, s>>>(B);
    else k_bouzidi_direct<StoreF32><<<grid, 256, 0, s>>>(B);
  } else {
    if (f16) {
      k_bouzidi_gather<StoreF16S><<<grid, 256, 0, s>>>(B);
      k_bouzidi_scatter<StoreF16S><<<grid, 256, 0, s>>>(B);
    } else {
      k_bouzidi_gather<StoreF32><<<grid, 256, 0, s>>>(B);
      k_bouzidi_scatter<StoreF32><<<grid, 256, 0, s>>>(B);
    }
  }
}

static int fill_dropin(BouzDev &B, float *f_out, const uint16_t *q_map, const int32_t *cell_block,
                       const int8_t *cx, const int8_t *cy, const int8_t *cz, int32_t n_boundary,
                       const int32_t *nbr, int32_t n_blocks, float q_min) {
  OL_CHECK_ARG(n_boundary >= 0 && n_blocks >= 0, "bouzidi: negative size");
  OL_CHECK_ARG(f_out && q_map && cell_block && cx && cy && cz && nbr,
               "bouzidi: null device pointer");
  B = BouzDev{};
  B.f = f_out;
  B.q = q_map;
  B.dense_q = 1;
  B.cell_block = cell_block; B.cell_x = cx; B.cell_y = cy; B.cell_z = cz;
  B.n_boundary = n_boundary;
  B.nbr = nbr; B.nbr_stride = n_blocks;
  B.block_offset = 0;
  B.dstride = (int64_t)BCELLS * n_blocks;
  B.q_min = q_min; B.scale = 1.0f; B.inv_scale = 1.0f;
  return OL_OK;
}

}  // namespace ol

using namespace ol;

extern "C" int ol_bouzidi(float *f_out, const float *f_post, const uint16_t *q_map,
                          const int32_t *cell_block, const int8_t *cell_x, const int8_t *cell_y,
                          const int8_t *cell_z, int32_t n_boundary, const int32_t *neighbor_table,
                          int32_t n_blocks, float q_min_threshold, void *stream) {
  if (n_boundary == 0) return OL_OK;
  BouzDev B;
  int rc = fill_dropin(B, f_out, q_map, cell_block, cell_x, cell_y, cell_z, n_boundary,
                       neighbor_table, n_blocks, q_min_threshold);
  if (rc) return rc;
  OL_CHECK_ARG(f_post && f_post != f_out, "ol_bouzidi: f_post must be a separate buffer");
  B.src = f_post;
  launch_bouzidi(B, false, (cudaStream_t)stream);
  OL_LAUNCHED("ol_bouzidi");
  return OL_OK;
}

extern "C" int ol_bouzidi_sparse(float *f_out, const uint16_t *q_map, const int32_t *cell_block,
                                 const int8_t *cell_x, const int8_t *cell_y, const int8_t *cell_z,
                                 int32_t n_boundary, const int32_t *neighbor_table,
                                 int32_t n_blocks, float q_min_threshold, float *scratch,
                                 void *stream) {
  if (n_boundary == 0) return OL_OK;
  BouzDev B;
  int rc = fill_dropin(B, f_out, q_map, cell_block, cell_x, cell_y, cell_z, n_boundary,
                       neighbor_table, n_blocks, q_min_threshold);
  if (rc) return rc;
  OL_CHECK_ARG(scratch, "ol_bouzidi_sparse: null scratch");
  B.src = f_out;
  B.scratch = scratch;
  launch_bouzidi(B, false, (cudaStream_t)stream);
  OL_LAUNCHED("ol_bouzidi_sparse");
  return OL_OK;
}

namespace ol {

// One thread per (direction, boundary cell), direction-major; the valid links
// are appended with warp-aggregated atomics (their order does not change any
// result: each link reads post-collision values and writes its own slot).
__global__ void k_bouzidi_build_links(const uint16_t *__restrict__ q_map,
                                      const int32_t *__restrict__ cell_block,
                                      const int8_t *__restrict__ cx, const int8_t *__restrict__ cy,
                                      const int8_t *__restrict__ cz, int32_t n_boundary,
                                      const int32_t *__restrict__ nbr, int32_t n_blocks,
                                      float q_min, ol_bouzidi_link *__restrict__ out,
                                      int32_t *__restrict__ count) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool valid = false;
  ol_bouzidi_link L = {};
  if (j < (int64_t)n_boundary * 27) {
    const int k = (int)(j / n_boundary);
    const int64_t i = j - (int64_t)k * n_boundary;
    const int b = cell_block[i] - 1;
    const int x = cx[i] - 1, y = cy[i] - 1, z = cz[i] - 1;
    const int own = b * BCELLS + x + BS * y + BS * BS * z;
    const float q = half_bits_to_float(q_map[(size_t)own + (size_t)k * BCELLS * n_blocks]);
    if (q > q_min && q <= 1.0f) {
      valid = true;
      L.cell = own;
      L.q = q;
      L.k = k;
      L.far_cell = -1;
      if (q < 0.5f) {
        const int nx = x - cx_of(k), ny = y - cy_of(k), nz = z - cz_of(k);
        if (nx >= 0 && nx < BS && ny >= 0 && ny < BS && nz >= 0 && nz < BS) {
          L.far_cell = b * BCELLS + nx + BS * ny + BS * BS * nz;
        } else {
          const int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0);
          const int oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0);
          const int oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
          const int nb = nbr[b + (int64_t)n_blocks * ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))];
          if (nb > 0) L.far_cell = (nb - 1) * BCELLS + (nx & 7) + BS * (ny & 7) + BS * BS * (nz & 7);
        }
      }
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, valid);
  if (m == 0) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (valid) out[base + __popc(m & ((1u << lane) - 1u))] = L;
}

void launch_bouzidi_links(void *f, const ol_bouzidi_link *links, int32_t n_links, int64_t cell0,
                          int64_t dstride, float scale, float *scratch, bool f16, cudaStream_t s) {
  if (n_links <= 0) return;
  const int grid = (n_links + 255) / 256;
  const void *fc = f;
  const float *sc = scratch;
  if (f16) {
    launch_pdl(k_bouzidi_links_gather<StoreF16S>, grid, 256, 0, s, fc, links, n_links, cell0,
               dstride, 1.0f / scale, scratch);
    launch_pdl(k_bouzidi_links_scatter<StoreF16S>, grid, 256, 0, s, f, links, n_links, cell0,
               dstride, scale, sc);
  } else {
    launch_pdl(k_bouzidi_links_gather<StoreF32>, grid, 256, 0, s, fc, links, n_links, cell0,
               dstride, 1.0f, scratch);
    launch_pdl(k_bouzidi_links_scatter<StoreF32>, grid, 256, 0, s, f, links, n_links, cell0,
               dstride, 1.0f, sc);
  }
}

}  // namespace ol

extern "C" int ol_bouzidi_build_links(const uint16_t *q_map, const int32_t *cell_block,
                                      const int8_t *cell_x, const int8_t *cell_y,
                                      const int8_t *cell_z, int32_t n_boundary,
                                      const int32_t *neighbor_table, int32_t n_blocks,
                                      float q_min_threshold, ol_bouzidi_link *links,
                                      int32_t *n_links_dev, void *stream) {
  OL_CHECK_ARG(n_boundary >= 0 && n_blocks > 0 && n_links_dev,
               "ol_bouzidi_build_links: bad argument");
  OL_CHECK_ARG((int64_t)n_boundary * 27 < (1LL << 31) && (int64_t)n_blocks * BCELLS < (1LL << 31),
               "ol_bouzidi_build_links: level too large");
  cudaStream_t s = (cudaStream_t)stream;
  OL_CUDA(cudaMemsetAsync(n_links_dev, 0, sizeof(int32_t), s));
  if (n_boundary == 0) return OL_OK;
  OL_CHECK_ARG(q_map && cell_block && cell_x && cell_y && cell_z && neighbor_table && links,
               "ol_bouzidi_build_links: null device pointer");
  const int64_t n = (int64_t)n_boundary * 27;
  k_bouzidi_build_links<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      q_map, cell_block, cell_x, cell_y, cell_z, n_boundary, neighbor_table, n_blocks,
      q_min_threshold, links, n_links_dev);
  OL_LAUNCHED("ol_bouzidi_build_links");
  return OL_OK;
}

extern "C" int ol_bouzidi_apply_links(float *f_out, const ol_bouzidi_link *links, int32_t n_links,
                                      int32_t n_blocks, float *scratch, void *stream) {
  OL_CHECK_ARG(n_links >= 0 && n_blocks > 0, "ol_bouzidi_apply_links: bad sizes");
  if (n_links == 0) return OL_OK;
  OL_CHECK_ARG(f_out && links && scratch, "ol_bouzidi_apply_links: null device pointer");
  OL_CHECK_ARG((int64_t)n_blocks * BCELLS < (1LL << 31),
               "ol_bouzidi_apply_links: n_blocks too large");
  launch_bouzidi_links(f_out, links, n_links, 0, (int64_t)BCELLS * n_blocks, 1.0f, scratch, false,
                       (cudaStream_t)stream);
  OL_LAUNCHED("ol_bouzidi_apply_links");
  return OL_OK;
}
