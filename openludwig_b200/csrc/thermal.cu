// Thermal DDF launch and its C ABI (stream_collide_thermal!, timestep.jl:101-145).
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "thermal.cuh"
#include "thermal_ws.cuh"

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

static int sm_count() {
  static int n_sm[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!n_sm[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    n_sm[dev] = v;
  }
  return n_sm[dev];
}

// Whether the warp-specialised thermal kernel serves this FP32 level: chosen
// (forced, or by default on levels of at least two blocks per SM); every
// absent-neighbour value precomputed in ghost rows or a level-1
// domain-boundary value; the arrays it bulk-copies 16-byte aligned.
static bool thermal_ws_applies(const ThermalDev &D, int n_sm) {
  auto a16 = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
  const int choice = stream_collide_kernel_choice();
  if (!(choice == OL_SC_KERNEL_WS || (choice == OL_SC_KERNEL_AUTO && D.n_blocks >= 2 * n_sm)))
    return false;
  if (!D.tp.is_level_1 && !D.ghost) return false;
  if (!a16(D.g_in) || !a16(D.vel) || !a16(D.sponge) || !a16(D.obstacle)) return false;
  return fault_word_device() != nullptr && ws_table_device() != nullptr;
}

template <class ST>
static void launch_t(const ThermalDev &D, cudaStream_t s) {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(k_thermal<ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
    if (std::is_same<ST, StoreF32>::value)
      cudaFuncSetAttribute(k_thermal_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, kTwBytes);
    done = true;
  }
  const int gn = D.gblocks ? D.n_gblocks : D.n_blocks;
  if (D.ghost && gn > 0) k_ghost_fill_thermal<ST><<<gn, kGhostThreads, 0, s>>>(D);
  const int n_sm = sm_count();
  if (std::is_same<ST, StoreF32>::value && thermal_ws_applies(D, n_sm)) {
    k_thermal_ws<<<ws_grid(D.n_blocks, n_sm), kWsThreads, kTwBytes, s>>>(D, ws_table_device(),
                                                                         fault_word_device());
    return;
  }
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
