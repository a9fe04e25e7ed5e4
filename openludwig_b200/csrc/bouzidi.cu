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
