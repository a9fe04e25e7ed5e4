// Merged flow output, the device part of export_merged_mesh_sync
// (io_vtk.jl:6-129): the exported blocks of every level (those not covered
// by all 8 children) packed level after level, in list order, into the
// contiguous arrays the VTK unstructured grid is written from -- points,
// density, velocity, velocity magnitude, obstacle flag, level and
// temperature -- with NaN and +-Inf replaced by 0 (io_vtk.jl:111-115).
// One CTA of 512 threads per exported block, one thread per cell; the
// arrays leave the device in one copy each instead of a full level copy
// per field followed by a host-side gather.
#include "common.cuh"
#include "lattice.cuh"

namespace ol {

constexpr int kMaxOutputLevels = 16;
constexpr int kPointsPerBlock = (BS + 1) * (BS + 1) * (BS + 1);  // 729

struct OutputPlan {
  ol_output_level lv[kMaxOutputLevels];
  int64_t first[kMaxOutputLevels + 1];  // exported-block offset of each level
  int32_t n_levels;
};

__device__ __forceinline__ float finite_or_zero(float v) { return isfinite(v) ? v : 0.0f; }

__global__ void __launch_bounds__(BCELLS)
    k_pack_merged(const __grid_constant__ OutputPlan P, const __grid_constant__ ol_output_fields O) {
  const int64_t i = blockIdx.x;  // exported block, over all levels
  int l = 0;
  while (l + 1 < P.n_levels && i >= P.first[l + 1]) ++l;
  const ol_output_level &V = P.lv[l];
  const int b = V.blocks[i - P.first[l]];
  const int t = threadIdx.x;
  const int64_t S = (int64_t)BCELLS * V.n_blocks;
  const int64_t src = (int64_t)b * BCELLS + t;
  const int64_t dst = i * BCELLS + t;
  if (O.rho) O.rho[dst] = finite_or_zero(V.rho[src]);
  if (O.vel || O.vel_mag) {
    const float ux = finite_or_zero(V.vel[src]), uy = finite_or_zero(V.vel[src + S]),
                uz = finite_or_zero(V.vel[src + 2 * S]);
    if (O.vel) {
      O.vel[3 * dst] = ux;
      O.vel[3 * dst + 1] = uy;
      O.vel[3 * dst + 2] = uz;
    }
    // sqrt.(vx.^2 .+ vy.^2 .+ vz.^2) in Float32, each operation rounded
    if (O.vel_mag)
      O.vel_mag[dst] = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ux, ux), __fmul_rn(uy, uy)),
                                            __fmul_rn(uz, uz)));
  }
  if (O.obstacle) O.obstacle[dst] = V.obstacle[src] ? 1 : 0;
  if (O.level) O.level[dst] = V.level_id;
  if (O.temperature) O.temperature[dst] = V.temperature ? finite_or_zero(V.temperature[src]) : 0.0f;
  if (O.points) {
    // (Float32((b - 1) * 8) + p) * dx per axis, points x fastest (io_vtk.jl:74-79)
    const int ox = (V.map_x[b] - 1) * BS, oy = (V.map_y[b] - 1) * BS, oz = (V.map_z[b] - 1) * BS;
    for (int p = t; p < kPointsPerBlock; p += BCELLS) {
      const int px = p % (BS + 1), py = (p / (BS + 1)) % (BS + 1), pz = p / ((BS + 1) * (BS + 1));
      float *q = O.points + 3 * (i * kPointsPerBlock + p);
      q[0] = __fmul_rn((float)(ox + px), V.dx);
      q[1] = __fmul_rn((float)(oy + py), V.dx);
      q[2] = __fmul_rn((float)(oz + pz), V.dx);
    }
  }
}

}  // namespace ol

using namespace ol;

extern "C" int ol_pack_merged_fields(const ol_output_level *levels, int32_t n_levels,
                                     const ol_output_fields *out, void *stream) {
  OL_CHECK_ARG(levels && out, "ol_pack_merged_fields: null argument");
  OL_CHECK_ARG(n_levels >= 1 && n_levels <= kMaxOutputLevels,
               "ol_pack_merged_fields: n_levels must be 1..%d", kMaxOutputLevels);
  OutputPlan P = {};
  P.n_levels = n_levels;
  int64_t total = 0;
  for (int l = 0; l < n_levels; ++l) {
    const ol_output_level &V = levels[l];
    OL_CHECK_ARG(V.n_export >= 0 && V.n_export <= V.n_blocks && V.n_blocks >= 0,
                 "ol_pack_merged_fields: level %d: bad sizes", l + 1);
    OL_CHECK_ARG((int64_t)V.n_blocks * BCELLS < (1LL << 31),
                 "ol_pack_merged_fields: level %d: too many cells", l + 1);
    if (V.n_export > 0)
      OL_CHECK_ARG(V.rho && V.vel && V.obstacle && V.map_x && V.map_y && V.map_z && V.blocks,
                   "ol_pack_merged_fields: level %d: null device pointer", l + 1);
    P.lv[l] = V;
    P.first[l] = total;
    total += V.n_export;
  }
  P.first[n_levels] = total;
  if (total == 0) return OL_OK;
  OL_CHECK_ARG(total < (1LL << 31) / kPointsPerBlock, "ol_pack_merged_fields: output too large");
  k_pack_merged<<<(unsigned)total, BCELLS, 0, (cudaStream_t)stream>>>(P, *out);
  OL_LAUNCHED("ol_pack_merged_fields");
  return OL_OK;
}
