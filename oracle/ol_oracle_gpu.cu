/*
 * ol_oracle_gpu.cu -- the oracle's per-cell restatement (ol_oracle_cell.h)
 * run on the GPU, one thread per cell or per boundary cell, in FP64 (and
 * FP32).  This is the accuracy oracle at full benchmark sizes: the plain
 * method of the reference in double precision, fast enough for thousands of
 * steps of the large cases that the CPU instantiation cannot finish in a
 * test.  Built with --fmad=false so every product and sum rounds as written.
 *
 * TEST INFRASTRUCTURE (see ol_oracle_kernels.cpp): loaded only by the tests.
 * Every kernel bounds its thread index by the work size; arguments are raw
 * device pointers owned by the caller, plus the stream to launch on.
 */
#include <cuda_runtime.h>

#include "ol_oracle_cell.h"

using namespace orc;

namespace {

constexpr int kThreads = 128;

template <class R>
__global__ void k_stream_collide(Level<R> L, Parent<R> P, StepParams sp) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)L.nB * NC) return;
  const int b = (int)(i / NC), c = (int)(i % NC);
  cell_step(L, P, sp, b, c % BS + 1, (c / BS) % BS + 1, c / (BS * BS) + 1);
}

template <class R>
__global__ void k_bouzidi(R *f_out, const R *f_post, const uint16_t *q, const int32_t *cb,
                          const int8_t *cx, const int8_t *cy, const int8_t *cz, int n,
                          const int32_t *nbr, int nB, float qmin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bouzidi_cell(f_out, f_post, q, cb, cx, cy, cz, i, nbr, nB, qmin);
}

template <class R>
__global__ void k_thermal(R *g_out, const R *g_in, R *g_post, R *T_out, const R *vel,
                          const uint8_t *obs, const float *sponge, const int32_t *nbr,
                          const int32_t *mx, const int32_t *my, const int32_t *mz, int nB,
                          Parent<R> P, ThermalParams tp) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nB * NC) return;
  const int b = (int)(i / NC), c = (int)(i % NC);
  thermal_cell(g_out, g_in, g_post, T_out, vel, obs, sponge, nbr, mx, my, mz, nB, P, tp, b,
               c % BS + 1, (c / BS) % BS + 1, c / (BS * BS) + 1);
}

unsigned grid_for(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

int status() { return (int)cudaGetLastError(); }

}  // namespace

#define ORCG_LEVEL_ARGS(R)                                                                    \
  R *f_out, const R *f_in, R *f_post, R *rho, R *vel_out, const R *vel_in,                    \
      const uint8_t *obstacle, const float *sponge, const float *wall_dist, const int32_t *nbr, \
      const int32_t *mx, const int32_t *my, const int32_t *mz, int32_t nB, const R *pf,       \
      const R *prho, const R *pvel, const R *pf_old, const R *prho_old, const R *pvel_old,     \
      const int32_t *pptr, int32_t pdx, int32_t pdy, int32_t pdz, int32_t pnB,                \
      const StepParams *sp, cudaStream_t stream

#define ORCG_LEVEL_BODY(R)                                                                    \
  if (nB <= 0) return 0;                                                                      \
  Level<R> L{f_out, f_in, f_post, rho, vel_out, vel_in, obstacle, sponge, wall_dist, nbr, mx, my, \
             mz, nB};                                                                        \
  Parent<R> P{pf, prho, pvel, pf_old, prho_old, pvel_old, pptr, pdx, pdy, pdz, pnB};          \
  k_stream_collide<R><<<grid_for((long long)nB * NC), kThreads, 0, stream>>>(L, P, *sp);      \
  return status();

#define ORCG_BOUZIDI(R)                                                                       \
  if (n <= 0) return 0;                                                                       \
  k_bouzidi<R><<<grid_for(n), kThreads, 0, stream>>>(f_out, f_post, q, cb, cx, cy, cz, n, nbr, \
                                                       nB, qmin);                            \
  return status();

#define ORCG_THERMAL_ARGS(R)                                                                  \
  R *g_out, const R *g_in, R *g_post, R *T_out, const R *vel, const uint8_t *obs,             \
      const float *sponge, const int32_t *nbr, const int32_t *mx, const int32_t *my,          \
      const int32_t *mz, int32_t nB, const R *pg, const R *pT, const R *pvel, const R *pg_old, \
      const R *pT_old, const R *pvel_old, const int32_t *pptr, int32_t pdx, int32_t pdy,      \
      int32_t pdz, int32_t pnB, const ThermalParams *tp, cudaStream_t stream

#define ORCG_THERMAL_BODY(R)                                                                  \
  if (nB <= 0) return 0;                                                                      \
  Parent<R> P{pg, pT, pvel, pg_old, pT_old, pvel_old, pptr, pdx, pdy, pdz, pnB};              \
  k_thermal<R><<<grid_for((long long)nB * NC), kThreads, 0, stream>>>(                        \
      g_out, g_in, g_post, T_out, vel, obs, sponge, nbr, mx, my, mz, nB, P, *tp);             \
  return status();

extern "C" {
int orcg_stream_collide_f32(ORCG_LEVEL_ARGS(float)) { ORCG_LEVEL_BODY(float) }
int orcg_stream_collide_f64(ORCG_LEVEL_ARGS(double)) { ORCG_LEVEL_BODY(double) }

int orcg_bouzidi_f32(float *f_out, const float *f_post, const uint16_t *q, const int32_t *cb,
                     const int8_t *cx, const int8_t *cy, const int8_t *cz, int32_t n,
                     const int32_t *nbr, int32_t nB, float qmin, cudaStream_t stream) {
  ORCG_BOUZIDI(float)
}
int orcg_bouzidi_f64(double *f_out, const double *f_post, const uint16_t *q, const int32_t *cb,
                     const int8_t *cx, const int8_t *cy, const int8_t *cz, int32_t n,
                     const int32_t *nbr, int32_t nB, float qmin, cudaStream_t stream) {
  ORCG_BOUZIDI(double)
}

int orcg_thermal_f32(ORCG_THERMAL_ARGS(float)) { ORCG_THERMAL_BODY(float) }
int orcg_thermal_f64(ORCG_THERMAL_ARGS(double)) { ORCG_THERMAL_BODY(double) }
}  // extern "C"
