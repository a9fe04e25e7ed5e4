// D3Q27 lattice as compile-time functions of the direction index.
//
// Direction order follows lattice.jl:11 (`for z, y, x in -1:1`, x fastest):
// k = (cx+1) + 3(cy+1) + 9(cz+1), 0-based here.  The reference uploads the
// same tables as device arrays and loads them inside its inner loops
// (timestep.jl:161-179); here every index below folds to a constant once the
// 27-direction loops are unrolled.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

namespace ol {

constexpr int Q = 27;
constexpr int BS = 8;          // block edge (blocks.jl:7 BLOCK_SIZE)
constexpr int BCELLS = 512;    // cells per block

__host__ __device__ constexpr int cx_of(int k) { return k % 3 - 1; }
__host__ __device__ constexpr int cy_of(int k) { return (k / 3) % 3 - 1; }
__host__ __device__ constexpr int cz_of(int k) { return k / 9 - 1; }
__host__ __device__ constexpr int opp_of(int k) { return 26 - k; }
// (cx, -cy, cz) and (cx, cy, -cz): timestep.jl:170-175
__host__ __device__ constexpr int mirror_y_of(int k) { return k - 6 * cy_of(k); }
__host__ __device__ constexpr int mirror_z_of(int k) { return k - 18 * cz_of(k); }
__host__ __device__ constexpr int c2_of(int k) {
  return cx_of(k) * cx_of(k) + cy_of(k) * cy_of(k) + cz_of(k) * cz_of(k);
}
// Weights as the Float32 quotients of timestep.jl:167 (8f0/27f0 ...).
__host__ __device__ inline float w_of(int k) {
  const int d2 = c2_of(k);
  return d2 == 0 ? 8.0f / 27.0f
                 : d2 == 1 ? 2.0f / 27.0f : d2 == 2 ? 1.0f / 54.0f : 1.0f / 216.0f;
}

// O(u^2) equilibrium, physics_utils.jl:19-24.
__device__ __forceinline__ float feq2(float rho, float ux, float uy, float uz,
                                      float w, float cx, float cy, float cz) {
  const float cu = cx * ux + cy * uy + cz * uz;
  const float usq = ux * ux + uy * uy + uz * uz;
  return rho * w * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
}

// O(u^4) Hermite equilibrium, physics_utils.jl:39-61.
__device__ __forceinline__ float feq4(float rho, float ux, float uy, float uz,
                                      float w, float cx, float cy, float cz) {
  const float cu = cx * ux + cy * uy + cz * uz;
  const float usq = ux * ux + uy * uy + uz * uz;
  const float cu2 = cu * cu, cu3 = cu2 * cu, cu4 = cu2 * cu2, usq2 = usq * usq;
  float v = 1.0f + 3.0f * cu + 4.5f * cu2 - 1.5f * usq;
  v += 4.5f * cu3 - 4.5f * cu * usq;
  v += 3.375f * cu4 - 6.75f * cu2 * usq + 1.125f * usq2;
  return rho * w * v;
}

__device__ __forceinline__ float feq_auto(float rho, float ux, float uy, float uz,
                                          float w, float cx, float cy, float cz,
                                          int compressible) {
  return compressible ? feq4(rho, ux, uy, uz, w, cx, cy, cz)
                      : feq2(rho, ux, uy, uz, w, cx, cy, cz);
}

// Thermal equilibrium g_eq = w T (1 + 3 c.u), physics_utils.jl:78-83.
__device__ __forceinline__ float geq(float T, float ux, float uy, float uz,
                                     float w, float cx, float cy, float cz) {
  const float cu = cx * ux + cy * uy + cz * uz;
  return w * T * (1.0f + 3.0f * cu);
}

// Inlet turbulence hash (physics_utils.jl:5-17): Int32 products wrap.
__device__ __forceinline__ uint32_t mix_hash(int32_t x) {
  uint32_t h = (uint32_t)x;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  return h ^ (h >> 16);
}
__device__ __forceinline__ float gradient_noise(int32_t gx, int32_t gy,
                                                int32_t gz, int32_t seed) {
  const uint32_t comb = (uint32_t)gx * 374761393u + (uint32_t)gy * 668265263u +
                        (uint32_t)gz * 1274126177u + (uint32_t)seed;
  const uint32_t h = mix_hash((int32_t)comb);
  return (float)(h & 0xFFFFu) / 32768.0f - 1.0f;
}

}  // namespace ol
