// Surface-force and flow-statistics device descriptors and launchers
// (forces.cu), shared by the drop-in entry points and the native context.
#pragma once
#include "lattice.cuh"
#include "../../include/openludwig_b200.h"

namespace ol {

struct ForceDev {
  ol_surface_mesh mesh;
  const float *rho, *vel;
  const uint8_t *obstacle;
  const int32_t *bptr;
  int64_t block_offset, dstride;
  ol_force_params fp;
  float *p_map, *sx_map, *sy_map, *sz_map;
  double *partials;
};

// Map + integrate; the nine FP64 sums land in dev_out9 (device memory).
int launch_surface_forces(const ForceDev &D, double *dev_out9, cudaStream_t s);
// Per-block FP64 statistics + fixed-order reduction into dev_out7.
int launch_flow_stats(const float *rho, const float *vel, const uint8_t *obs, int32_t nb,
                      int64_t block_offset, int64_t dstride, double *partials, double *dev_out7,
                      cudaStream_t s);
constexpr int kForceThreadsH = 128;
inline size_t force_partial_rows(int n_triangles) {
  return (size_t)((n_triangles + kForceThreadsH - 1) / kForceThreadsH);
}

}  // namespace ol
