// Thermal DDF launch and its C ABI (stream_collide_thermal!, timestep.jl:101-145).
#include "common.cuh"
#include "thermal.cuh"

namespace ol {

template <class ST>
__global__ void __launch_bounds__(512, 2) k_thermal(const __grid_constant__ ThermalDev D) {
  __shared__ int nbbase[27];
  extern __shared__ float E[];
  const int b = blockIdx.x;
  const bool miss = load_nbbase_sync(D.nbr, D.nbr_stride, D.block_offset, b, threadIdx.x, nbbase);
  stage_thermal<ST>(D, nbbase, b, threadIdx.x, E, D.halo_tab, miss);
  __syncthreads();
  thermal_cell<ST>(D, nbbase, E, b, threadIdx.x);
}

// Boundary values of the absent-neighbour thermal pulls of every block, into
// D.ghost (the flow's ghost pass for the thermal populations).
template <class ST>
__global__ void __launch_bounds__(kGhostThreads, kGhostMinBlocks)
    k_ghost_fill_thermal(const __grid_constant__ ThermalDev D) {
  const int b = D.gblocks ? D.gblocks[blockIdx.x] : (int)blockIdx.x;
  ghost_fill_block<ST>(D, b, ghost_row_of(D, b), ghost_next_row_of(D, b));
}

template <class ST>
static void launch_t(const ThermalDev &D, cudaStream_t s) {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(k_thermal<ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
    done = true;
  }
  const int gn = D.gblocks ? D.n_gblocks : D.n_blocks;
  if (D.ghost && gn > 0) k_ghost_fill_thermal<ST><<<gn, kGhostThreads, 0, s>>>(D);
  k_thermal<ST><<<D.n_blocks, BCELLS, kStageBytes, s>>>(D);
}

void launch_thermal(const ThermalDev &D, bool f16, cudaStream_t s) {
  if (D.n_blocks <= 0) return;
  if (f16) launch_t<StoreF16S>(D, s);
  else launch_t<StoreF32>(D, s);
}

}  // namespace ol

using namespace ol;

extern "C" int ol_thermal(const ol_thermal_view *tv, const ol_thermal_params *tp, void *stream) {
  OL_CHECK_ARG(tv && tp, "ol_thermal: null view or params");
  OL_CHECK_ARG(tv->n_blocks >= 0, "ol_thermal: n_blocks < 0");
  if (tv->n_blocks == 0) return OL_OK;
  OL_CHECK_ARG(tv->g_in && tv->g_out && tv->temperature && tv->vel && tv->obstacle &&
                   tv->sponge && tv->neighbor_table && tv->map_x && tv->map_y && tv->map_z,
               "ol_thermal: required buffer is null");
  OL_CHECK_ARG(tv->g_in != tv->g_out, "ol_thermal: g_in aliases g_out");
  OL_CHECK_ARG(!(tp->store_post_collision == 1) || tv->g_post,
               "ol_thermal: store_post_collision needs g_post");
  ThermalDev D = {};
  D.g_in = tv->g_in; D.g_out = tv->g_out; D.g_post = tv->g_post;
  D.T_out = tv->temperature; D.vel = tv->vel; D.obstacle = tv->obstacle; D.sponge = tv->sponge;
  D.nbr = tv->neighbor_table; D.map_x = tv->map_x; D.map_y = tv->map_y; D.map_z = tv->map_z;
  D.n_blocks = tv->n_blocks;
  D.block_offset = 0;
  D.dstride = (int64_t)BCELLS * tv->n_blocks;
  D.nbr_stride = tv->n_blocks;
  D.scale = 1.0f; D.inv_scale = 1.0f; D.p_inv_scale = 1.0f;
  D.ghost = tv->ghost;
  D.ghost_next = tv->ghost_next;
  D.ghost_mode = tv->ghost_mode;
  D.gblocks = tv->ghost_blocks;
  D.n_gblocks = tv->n_ghost_blocks;
  OL_CHECK_ARG(tv->n_ghost_blocks >= 0 && tv->n_ghost_blocks <= tv->n_blocks &&
                   (tv->n_ghost_blocks == 0 || tv->ghost_blocks),
               "ol_thermal: bad ghost block list");
  OL_CHECK_ARG(tv->ghost_mode >= OL_GHOST_UNPAIRED && tv->ghost_mode <= OL_GHOST_PAIR_SECOND,
               "ol_thermal: unknown ghost_mode %d", tv->ghost_mode);
  OL_CHECK_ARG(tv->ghost_mode == OL_GHOST_UNPAIRED || (tv->ghost && !tp->is_level_1),
               "ol_thermal: ghost pairing needs a fine level and the ghost scratch");
  OL_CHECK_ARG(tv->ghost_mode != OL_GHOST_PAIR_FIRST ||
                   (tv->ghost_next && tv->ghost_next != tv->ghost && tp->temporal_weight == 0.0f),
               "ol_thermal: OL_GHOST_PAIR_FIRST needs a distinct ghost_next and temporal "
               "weight 0");
  OL_CHECK_ARG(tv->ghost_mode != OL_GHOST_PAIR_SECOND || tp->temporal_weight == 0.5f,
               "ol_thermal: OL_GHOST_PAIR_SECOND needs temporal weight 1/2");
  D.tp = *tp;
  D.halo_tab = halo_table_device();
  if (!D.halo_tab) return set_error(OL_ERR_CUDA, "ol_thermal: staging table allocation failed");
  if (!tp->is_level_1) {
    OL_CHECK_ARG(tv->pg && tv->pT && tv->pvel && tv->p_block_ptr && tv->p_n_blocks > 0,
                 "ol_thermal: fine level needs parent thermal state");
    OL_CHECK_ARG(!(tp->use_temporal_interp == 1 && tp->temporal_weight < 0.99f) ||
                     (tv->pg_old && tv->pT_old && tv->pvel_old),
                 "ol_thermal: temporal interpolation needs parent old state");
    D.pg = tv->pg; D.pT = tv->pT; D.pvel = tv->pvel;
    D.pg_old = tv->pg_old; D.pT_old = tv->pT_old; D.pvel_old = tv->pvel_old;
    D.pptr = tv->p_block_ptr;
    D.pdim_x = tv->p_dim_x; D.pdim_y = tv->p_dim_y; D.pdim_z = tv->p_dim_z;
    D.p_block_offset = 0;
    D.p_dstride = (int64_t)BCELLS * tv->p_n_blocks;
  }
  launch_thermal(D, false, (cudaStream_t)stream);
  OL_LAUNCHED("ol_thermal");
  return OL_OK;
}
