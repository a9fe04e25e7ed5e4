// Drop-in stream-collide launch: one CTA per 8^3 block, one thread per cell,
// caller buffers in the reference layout (FP32 populations).
#include "common.cuh"
#include "stream_collide.cuh"

namespace ol {

// The neighbour-table row of the block is staged in shared memory; the
// 27 pull sources of a cell then need no further table reads.  Blocks with
// an absent neighbour first park their boundary pulls in `ghost`.
constexpr int kGhostBytes = 27 * BCELLS * sizeof(float);

// Cumulant fits 64 registers (2 CTAs of 512 threads per SM); the
// regularized-BGK body keeps 27 equilibria in flight and gets 128.
template <int OP, class ST, bool WALE>
__global__ void __launch_bounds__(512, OP == OL_OP_CUMULANT ? 2 : 1)
    k_stream_collide(const __grid_constant__ LevelDev L) {
  __shared__ int nb_blk[27];
  __shared__ int n_missing;
  extern __shared__ float ghost[];
  const int b = blockIdx.x;
  if (threadIdx.x == 0) n_missing = 0;
  __syncthreads();
  if (threadIdx.x < 27) {
    const int nb = L.nbr[b + L.nbr_stride * threadIdx.x];
    nb_blk[threadIdx.x] = nb;
    if (nb <= 0) atomicAdd(&n_missing, 1);
  }
  __syncthreads();
  if (n_missing) fill_ghost<ST>(L, nb_blk, b, threadIdx.x, ghost);
  stream_collide_cell<OP, ST, WALE>(L, nb_blk, ghost, b, threadIdx.x);
}

template <int OP, class ST, bool WALE>
static void set_smem_attr() {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(k_stream_collide<OP, ST, WALE>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kGhostBytes);
    done = true;
  }
}

template <int OP, class ST, bool WALE>
static void launch_one(const LevelDev &L, cudaStream_t s) {
  set_smem_attr<OP, ST, WALE>();
  k_stream_collide<OP, ST, WALE><<<L.n_blocks, BCELLS, kGhostBytes, s>>>(L);
}

template <class ST>
static void launch_sc(const LevelDev &L, cudaStream_t s) {
  const bool wale = L.sp.c_wale != 0.0f;
  if (L.sp.op == OL_OP_CUMULANT) {
    if (wale) launch_one<OL_OP_CUMULANT, ST, true>(L, s);
    else launch_one<OL_OP_CUMULANT, ST, false>(L, s);
  } else {
    if (wale) launch_one<OL_OP_REGULARIZED_BGK, ST, true>(L, s);
    else launch_one<OL_OP_REGULARIZED_BGK, ST, false>(L, s);
  }
}

void launch_stream_collide(const LevelDev &L, bool f16, cudaStream_t s) {
  if (L.n_blocks <= 0) return;
  if (f16) launch_sc<StoreF16S>(L, s);
  else launch_sc<StoreF32>(L, s);
}

// f = f_temp = w_k; optional f_old = w_k, rho_old = 1, vel_old = 0 (main.jl:113-128)
__global__ void k_init_eq(float *f, float *ft, float *fo, float *ro, float *vo,
                          int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const float w = w_of(k);
    f[i + k * n] = w;
    ft[i + k * n] = w;
    if (fo) fo[i + k * n] = w;
  }
  if (fo) {
    ro[i] = 1.0f;
    vo[i] = 0.0f; vo[i + n] = 0.0f; vo[i + 2 * n] = 0.0f;
  }
}

}  // namespace ol

using namespace ol;

extern "C" int ol_stream_collide(const ol_level_view *lv, const ol_parent_view *pv,
                                 const ol_step_params *sp, void *stream) {
  OL_CHECK_ARG(lv && sp, "ol_stream_collide: null level view or params");
  OL_CHECK_ARG(lv->n_blocks >= 0, "ol_stream_collide: n_blocks < 0");
  if (lv->n_blocks == 0) return OL_OK;
  OL_CHECK_ARG(lv->f_in && lv->f_out && lv->rho && lv->vel_out && lv->obstacle &&
                   lv->sponge && lv->neighbor_table && lv->map_x && lv->map_y && lv->map_z,
               "ol_stream_collide: required level buffer is null");
  OL_CHECK_ARG(sp->op == OL_OP_CUMULANT || sp->op == OL_OP_REGULARIZED_BGK,
               "ol_stream_collide: unknown operator %d", sp->op);
  OL_CHECK_ARG(sp->c_wale == 0.0f || lv->vel_in, "ol_stream_collide: WALE needs vel_in");
  OL_CHECK_ARG(!(sp->wall_model_active == 1) || lv->wall_dist,
               "ol_stream_collide: wall model needs wall_dist");
  OL_CHECK_ARG(!(sp->store_post_collision == 1) || lv->f_post,
               "ol_stream_collide: store_post_collision needs f_post");
  OL_CHECK_ARG(lv->f_in != lv->f_out, "ol_stream_collide: f_in aliases f_out");
  LevelDev L = {};
  L.f_in = lv->f_in; L.f_out = lv->f_out; L.f_post = lv->f_post;
  L.rho_out = lv->rho; L.vel_out = lv->vel_out; L.vel_in = lv->vel_in;
  L.obstacle = lv->obstacle; L.sponge = lv->sponge; L.wall_dist = lv->wall_dist;
  L.nbr = lv->neighbor_table; L.map_x = lv->map_x; L.map_y = lv->map_y; L.map_z = lv->map_z;
  L.n_blocks = lv->n_blocks;
  L.block_offset = 0;
  L.dstride = (int64_t)BCELLS * lv->n_blocks;
  L.nbr_stride = lv->n_blocks;
  L.scale = 1.0f; L.inv_scale = 1.0f; L.p_inv_scale = 1.0f;
  L.sp = *sp;
  if (!sp->is_level_1) {
    OL_CHECK_ARG(pv && pv->f && pv->rho && pv->vel && pv->block_ptr && pv->n_blocks > 0,
                 "ol_stream_collide: fine level needs a parent view");
    OL_CHECK_ARG(!(sp->use_temporal_interp == 1 && sp->temporal_weight < 0.99f) ||
                     (pv->f_old && pv->rho_old && pv->vel_old),
                 "ol_stream_collide: temporal interpolation needs parent old state");
    L.pf = pv->f; L.prho = pv->rho; L.pvel = pv->vel;
    L.pf_old = pv->f_old; L.prho_old = pv->rho_old; L.pvel_old = pv->vel_old;
    L.pptr = pv->block_ptr;
    L.pdim_x = pv->dim_x; L.pdim_y = pv->dim_y; L.pdim_z = pv->dim_z;
    L.p_block_offset = 0;
    L.p_dstride = (int64_t)BCELLS * pv->n_blocks;
  }
  launch_stream_collide(L, false, (cudaStream_t)stream);
  OL_LAUNCHED("ol_stream_collide");
  return OL_OK;
}

extern "C" int ol_init_equilibrium(float *f, float *f_temp, float *f_old, float *rho_old,
                                   float *vel_old, int32_t n_blocks, void *stream) {
  OL_CHECK_ARG(n_blocks >= 0, "ol_init_equilibrium: n_blocks < 0");
  if (n_blocks == 0) return OL_OK;
  OL_CHECK_ARG(f && f_temp, "ol_init_equilibrium: null f/f_temp");
  OL_CHECK_ARG(!f_old || (rho_old && vel_old), "ol_init_equilibrium: f_old needs rho_old/vel_old");
  const int64_t n = (int64_t)BCELLS * n_blocks;
  k_init_eq<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(f, f_temp, f_old,
                                                                          rho_old, vel_old, n);
  OL_LAUNCHED("ol_init_equilibrium");
  return OL_OK;
}
