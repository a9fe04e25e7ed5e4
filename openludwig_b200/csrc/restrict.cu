// Fine-to-coarse restriction (opt-in; the reference couples the levels one
// way only, coarse to fine, physics_interpolation.jl).  After the two fine
// sub-steps of a coarse step, every coarse cell covered by a fine block takes
// the average of its 2 x 2 x 2 fine children:
//   fbar_k = (sum of the children's f_k) / 8,  rho = sum_k fbar_k,
//   u = sum_k c_k fbar_k / rho,
//   f_k <- feq(rho, u) + (fbar_k - feq(rho, u)) * clamp((tau_c - 1/2) / (tau_f - 1/2), 0.01, 100)
// (the inverse of the coarse-to-fine rescaling of the non-equilibrium part;
// mass-conserving), and rho, u are stored too.  Coarse cells that are solid,
// or have a solid child, keep their own values.  One thread per coarse cell:
// a fine block covers 4 x 4 x 4 coarse cells.
#include "common.cuh"
#include "level_dev.cuh"

namespace ol {
namespace {

struct RestrictDev {
  ol_restrict_view v;
  int64_t fS, cS;  // fine / coarse plane strides (cells)
};

__global__ void k_restrict(const __grid_constant__ RestrictDev R) {
  const ol_restrict_view &v = R.v;
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)v.n_fine * 64) return;
  const int fb = (int)(gid >> 6), q = (int)(gid & 63);
  const int i = q & 3, j = (q >> 2) & 3, l = q >> 4;
  // coarse global cell (1-based) covered by fine cells 2i.., 2j.., 2l.. of block fb
  const int gx = (v.map_x[fb] - 1) * 4 + i + 1;
  const int gy = (v.map_y[fb] - 1) * 4 + j + 1;
  const int gz = (v.map_z[fb] - 1) * 4 + l + 1;
  const int bx = (gx - 1) / 8 + 1, by = (gy - 1) / 8 + 1, bz = (gz - 1) / 8 + 1;
  if (bx > v.dim_x || by > v.dim_y || bz > v.dim_z) return;
  const int pb = v.block_ptr[(bx - 1) + v.dim_x * ((by - 1) + v.dim_y * (bz - 1))];
  if (pb <= 0) return;
  const int64_t cc = (int64_t)(pb - 1) * BCELLS + (gx - 1) % 8 + 8 * ((gy - 1) % 8) +
                     64 * ((gz - 1) % 8);
  if (v.obstacle_coarse[cc]) return;
  int64_t fc[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    fc[s] = (int64_t)fb * BCELLS + (2 * i + (s & 1)) + 8 * (2 * j + ((s >> 1) & 1)) +
            64 * (2 * l + (s >> 2));
    if (v.obstacle_fine[fc[s]]) return;
  }
  float fbar[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    float acc = 0.0f;
#pragma unroll
    for (int s = 0; s < 8; ++s) acc = __fadd_rn(acc, v.f_fine[fc[s] + k * R.fS]);
    fbar[k] = __fmul_rn(acc, 0.125f);
  }
  float rho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    rho = __fadd_rn(rho, fbar[k]);
    if (cx_of(k) == 1) jx = __fadd_rn(jx, fbar[k]); else if (cx_of(k) == -1) jx = __fsub_rn(jx, fbar[k]);
    if (cy_of(k) == 1) jy = __fadd_rn(jy, fbar[k]); else if (cy_of(k) == -1) jy = __fsub_rn(jy, fbar[k]);
    if (cz_of(k) == 1) jz = __fadd_rn(jz, fbar[k]); else if (cz_of(k) == -1) jz = __fsub_rn(jz, fbar[k]);
  }
  const float ux = __fdiv_rn(jx, rho), uy = __fdiv_rn(jy, rho), uz = __fdiv_rn(jz, rho);
  const float tf = v.tau_fine - 0.5f, tc = v.tau_coarse - 0.5f;
  const float sc = tf > 1e-6f ? fminf(fmaxf(__fdiv_rn(tc, tf), 0.01f), 100.0f) : 1.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const float fe = feq_auto(rho, ux, uy, uz, w_of(k), (float)cx_of(k), (float)cy_of(k),
                              (float)cz_of(k), v.compressible);
    v.f_coarse[cc + k * R.cS] = __fadd_rn(fe, __fmul_rn(__fsub_rn(fbar[k], fe), sc));
  }
  v.rho_coarse[cc] = rho;
  v.vel_coarse[cc] = ux;
  v.vel_coarse[cc + R.cS] = uy;
  v.vel_coarse[cc + 2 * R.cS] = uz;
}

}  // namespace
}  // namespace ol

using namespace ol;

extern "C" int ol_restrict(const ol_restrict_view *v, void *stream) {
  OL_CHECK_ARG(v, "ol_restrict: null view");
  OL_CHECK_ARG(v->n_fine >= 0 && v->n_coarse >= 0, "ol_restrict: negative block count");
  if (v->n_fine == 0 || v->n_coarse == 0) return OL_OK;
  OL_CHECK_ARG(v->f_fine && v->obstacle_fine && v->map_x && v->map_y && v->map_z && v->f_coarse &&
                   v->rho_coarse && v->vel_coarse && v->obstacle_coarse && v->block_ptr,
               "ol_restrict: required buffer is null");
  OL_CHECK_ARG(v->f_fine != v->f_coarse, "ol_restrict: fine and coarse populations alias");
  RestrictDev R;
  R.v = *v;
  R.fS = (int64_t)v->n_fine * BCELLS;
  R.cS = (int64_t)v->n_coarse * BCELLS;
  const int64_t n = (int64_t)v->n_fine * 64;
  k_restrict<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(R);
  OL_LAUNCHED("ol_restrict");
  return OL_OK;
}
