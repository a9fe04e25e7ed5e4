// Drop-in stream-collide launch: one CTA per 8^3 block, one thread per cell,
// caller buffers in the reference layout (FP32 populations).
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "pipe.cuh"
#include "ws.cuh"

namespace ol {

// Packed staging entries: k | dir << 5 | source cell << 10 | E slot << 19,
// sorted by direction so consecutive threads read consecutive sources.
static std::vector<uint32_t> build_halo_table() {
  std::vector<uint32_t> tab;
  for (int k = 0; k < 27; ++k)
    for (int z = 0; z < 8; ++z)
      for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
          const int sx = x - cx_of(k), sy = y - cy_of(k), sz = z - cz_of(k);
          if (sx >= 0 && sx < 8 && sy >= 0 && sy < 8 && sz >= 0 && sz < 8) continue;
          const int ox = sx < 0 ? -1 : (sx > 7 ? 1 : 0);
          const int oy = sy < 0 ? -1 : (sy > 7 ? 1 : 0);
          const int oz = sz < 0 ? -1 : (sz > 7 ? 1 : 0);
          const uint32_t dir = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1);
          const uint32_t src = (sx & 7) + 8 * (sy & 7) + 64 * (sz & 7);
          const uint32_t dst = e_index(sx, sy, sz);
          tab.push_back((uint32_t)k | dir << 5 | src << 10 | dst << 19);
        }
  // then the ring positions of the 10^3 staging plane, in slot order
  for (int p = 0; p < 1000; ++p) {
    const int x = p % 10 - 1, y = (p / 10) % 10 - 1, z = p / 100 - 1;
    if (x >= 0 && x < 8 && y >= 0 && y < 8 && z >= 0 && z < 8) continue;
    tab.push_back((uint32_t)p);
  }
  // then, per halo entry, the ring index of its staging slot
  std::vector<int> ring_of(1000, -1);
  for (int q = 0; q < kRingEntries; ++q) ring_of[tab[kHaloEntries + q]] = q;
  for (int i = 0; i < kHaloEntries; ++i) tab.push_back((uint32_t)ring_of[tab[i] >> 19]);
  return tab;
}

const uint32_t *halo_table_device() {
  static std::mutex mu;
  static uint32_t *per_dev[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!per_dev[dev]) {
    const std::vector<uint32_t> tab = build_halo_table();
    if ((int)tab.size() != kHaloTableSize) return nullptr;
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, tab.size() * sizeof(uint32_t)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
        cudaSuccess) {
      cudaFree(d);
      return nullptr;
    }
    per_dev[dev] = d;
  }
  return per_dev[dev];
}

// Loader table of the warp-specialised kernel (ws.cuh): the staging table's
// out-of-block pulls in the same order, with the destination cell (the
// pulling cell) in place of the 10^3 slot, then the face-halo velocity slots.
static std::vector<uint32_t> build_ws_table() {
  const std::vector<uint32_t> halo = build_halo_table();
  std::vector<uint32_t> tab;
  for (int i = 0; i < kHaloEntries; ++i) {
    const uint32_t e = halo[i];
    const int k = e & 31, slot = e >> 19;
    const int dx = slot % 10 - 1 + cx_of(k), dy = (slot / 10) % 10 - 1 + cy_of(k),
              dz = slot / 100 - 1 + cz_of(k);
    const uint32_t d = (uint32_t)(dx + 8 * dy + 64 * dz);
    tab.push_back((e & ((1u << 19) - 1)) | d << 19);
  }
  const int faces[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  for (const auto &f : faces) {
    const uint32_t dir = (f[0] + 1) + 3 * (f[1] + 1) + 9 * (f[2] + 1);
    for (int z = 0; z < 8; ++z)
      for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
          const bool on = (f[0] < 0 && x == 0) || (f[0] > 0 && x == 7) || (f[1] < 0 && y == 0) ||
                          (f[1] > 0 && y == 7) || (f[2] < 0 && z == 0) || (f[2] > 0 && z == 7);
          if (on) tab.push_back(dir | (uint32_t)(x + 8 * y + 64 * z) << 5);
        }
  }
  // the FP32 compute-stage slot of each out-of-block pull
  for (int i = 0; i < kHaloEntries; ++i) {
    const uint32_t e = tab[i];
    const int k = e & 31, d = (int)(e >> 19);
    tab.push_back((uint32_t)(k * kSPlane + kSPad + d - cx_of(k)));
  }
  return tab;
}

const uint32_t *ws_table_device() {
  static std::mutex mu;
  static uint32_t *per_dev[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!per_dev[dev]) {
    const std::vector<uint32_t> tab = build_ws_table();
    if ((int)tab.size() != kWsTableTotal) return nullptr;
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, tab.size() * sizeof(uint32_t)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
        cudaSuccess) {
      cudaFree(d);
      return nullptr;
    }
    per_dev[dev] = d;
  }
  return per_dev[dev];
}

// Per-device fault word of the warp-specialised kernels (bits kWsFault*):
// set when one of their bounded waits runs out; read and cleared by
// ol_pipeline_fault.
int *fault_word_device() {
  static std::mutex mu;
  static int *per_dev[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!per_dev[dev]) {
    int *d = nullptr;
    if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return nullptr;
    if (cudaMemset(d, 0, sizeof(int)) != cudaSuccess) {
      cudaFree(d);
      return nullptr;
    }
    per_dev[dev] = d;
  }
  return per_dev[dev];
}

// Stream-collide kernel selection (ol_set_stream_collide_kernel): 0 = by
// level (warp-specialised persistent kernel where it applies and the level
// spans at least two waves of it), 1 = one CTA per block, 2 = the
// warp-specialised kernel wherever it applies.
static int g_sc_kernel = OL_SC_KERNEL_AUTO;
static int g_ws_max_ctas = 0;  // > 0: cap on the warp-specialised grid

int stream_collide_kernel_choice() { return g_sc_kernel; }
int ws_grid(int64_t n_items, int n_sm) {
  int64_t g = n_items < n_sm ? n_items : n_sm;
  if (g_ws_max_ctas > 0 && g > g_ws_max_ctas) g = g_ws_max_ctas;
  return (int)(g < 1 ? 1 : g);
}

// One CTA per block: neighbour offsets, then the staged pull windows, then
// the cell update.  Cumulant fits 64 registers (2 CTAs of 512 threads per
// SM, 2 x 105 KB of staging); regularized BGK keeps 27 equilibria in flight
// and gets 128.
template <int OP, class ST, bool WALE>
__global__ void __launch_bounds__(512, OP == OL_OP_CUMULANT ? 2 : 1)
    k_stream_collide(const __grid_constant__ LevelDev L) {
  __shared__ int nbbase[27];
  extern __shared__ float E[];
  const int b = blockIdx.x;
  // the own block's planes and masks do not depend on the neighbour table:
  // their loads are in flight while it is read
  const int64_t own0 = (L.block_offset + b) * BCELLS;
  if (L.prefetch_ahead > 0) prefetch_block_l2<ST>(L, b + L.prefetch_ahead, threadIdx.x);
  pdl_wait();  // f_in, ghost rows: written by the launches before this one
  OwnRegs<ST> r;
  own_load(L.f_in, L.dstride, own0, threadIdx.x, r);
  const bool obs = L.obstacle[own0 + threadIdx.x] != 0;
  const float spg = L.sponge[own0 + threadIdx.x];
  const bool miss = load_nbbase_sync(L.nbr, L.nbr_stride, L.block_offset, b, threadIdx.x, nbbase);
  stage_flow<ST>(L, nbbase, b, threadIdx.x, E, miss, r);
  __syncthreads();
  stream_collide_cell<OP, ST, WALE>(L, nbbase, E, b, threadIdx.x, obs, spg);
}

template <int OP, class ST, bool WALE>
static void launch_one(const LevelDev &L0, cudaStream_t s) {
  static bool done = false;
  static int resident = 0;  // CTAs of this kernel resident on the whole device
  if (!done) {
    cudaFuncSetAttribute(k_stream_collide<OP, ST, WALE>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
    int dev = 0, n_sm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stream_collide<OP, ST, WALE>,
                                                      BCELLS, kStageBytes) == cudaSuccess)
      resident = n_sm * per_sm;
    done = true;
  }
  // CTA b prefetches a block that starts about 3/4 of a wave later (measured
  // on the cube's finest level: 1/2 wave 261, 3/4 259, 1 263, 5/4 269 us per
  // call; farther ahead the lines are gone again before they are staged); a
  // level of fewer than four waves has little to hide and skips it
  LevelDev L = L0;
  L.prefetch_ahead = L.n_blocks >= 4 * resident ? resident * 3 / 4 : 0;
  launch_pdl(k_stream_collide<OP, ST, WALE>, L.n_blocks, BCELLS, kStageBytes, s, L);
}

// Warp-specialised persistent kernel over the level's blocks: one CTA per
// SM (or per block when the level is smaller).
template <int OP, class ST, bool WALE>
static void launch_ws(const LevelDev &L, int n_sm, cudaStream_t s) {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(k_sc_ws<OP, ST, WALE, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         ws_smem_bytes<ST>());
    done = true;
  }
  const int grid = ws_grid(L.n_blocks, n_sm);
  launch_pdl(k_sc_ws<OP, ST, WALE, false>, grid, kWsThreads, ws_smem_bytes<ST>(), s, L,
             (const LevelDev *)nullptr, (const WorkItem *)nullptr, 0, ws_table_device(),
             fault_word_device());
}

static int device_sm_count() {
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

// Whether the warp-specialised kernel serves this level: cumulant operator;
// every absent-neighbour value either precomputed in ghost rows or a
// level-1 domain-boundary value its loader evaluates; the arrays it moves
// with bulk copies 16-byte aligned.
static bool ws_applies(const LevelDev &L) {
  auto a16 = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
  if (L.sp.op != OL_OP_CUMULANT) return false;
  if (!L.sp.is_level_1 && !L.ghost) return false;
  if (!a16(L.f_in) || !a16(L.obstacle) || !a16(L.sponge)) return false;
  if (L.sp.c_wale != 0.0f && !a16(L.vel_in)) return false;
  if (L.sp.wall_model_active == 1 && L.wall_dist && !a16(L.wall_dist)) return false;
  return fault_word_device() != nullptr && ws_table_device() != nullptr;
}

template <int OP, bool WALE>
static void launch_pipe(const LevelDev &L, cudaStream_t s) {
  static bool done = false;
  static int n_sm = 148;
  if (!done) {
    cudaFuncSetAttribute(k_sc_pipe<OP, WALE, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kPipeBytes);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    done = true;
  }
  const int resident = n_sm * (OP == OL_OP_CUMULANT ? 2 : 1);
  const int grid = L.n_blocks < resident ? L.n_blocks : resident;
  k_sc_pipe<OP, WALE, false><<<grid, BCELLS, kPipeBytes, s>>>(L, nullptr, nullptr, 0);
}

template <class ST>
static void launch_sc(const LevelDev &L, cudaStream_t s) {
  const bool wale = L.sp.c_wale != 0.0f;
  const int n_sm = device_sm_count();
  const bool ws = g_sc_kernel == OL_SC_KERNEL_WS ||
                  (g_sc_kernel == OL_SC_KERNEL_AUTO && L.n_blocks >= 2 * n_sm &&
                   std::is_same<ST, StoreF32>::value);
  if (ws && ws_applies(L)) {
    if (wale) launch_ws<OL_OP_CUMULANT, ST, true>(L, n_sm, s);
    else launch_ws<OL_OP_CUMULANT, ST, false>(L, n_sm, s);
    return;
  }
  if (L.sp.op == OL_OP_CUMULANT) {
    if (wale) launch_one<OL_OP_CUMULANT, ST, true>(L, s);
    else launch_one<OL_OP_CUMULANT, ST, false>(L, s);
  } else {
    if (wale) launch_one<OL_OP_REGULARIZED_BGK, ST, true>(L, s);
    else launch_one<OL_OP_REGULARIZED_BGK, ST, false>(L, s);
  }
}

// FP32 launches use one CTA per block (two resident per SM) with synchronous
// staging; OL_PIPELINE=1 in the environment selects the software-pipelined
// persistent kernel instead (one CTA per SM, cp.async double buffering).
static bool use_pipeline() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("OL_PIPELINE");
    v = (e && e[0] == '1') ? 1 : 0;
  }
  return v == 1;
}

void launch_stream_collide(const LevelDev &L, bool f16, cudaStream_t s) {
  if (L.n_blocks <= 0) return;
  const int gn = L.gblocks ? L.n_gblocks : L.n_blocks;
  if (L.ghost && gn > 0) {
    if (f16) launch_pdl(k_ghost_fill<StoreF16S>, gn, kGhostThreads, 0, s, L);
    else launch_pdl(k_ghost_fill<StoreF32>, gn, kGhostThreads, 0, s, L);
  }
  if (f16 || !use_pipeline()) {
    if (!f16) { launch_sc<StoreF32>(L, s); return; }
    launch_sc<StoreF16S>(L, s);
  } else {
    const bool wale = L.sp.c_wale != 0.0f;
    if (L.sp.op == OL_OP_CUMULANT) {
      if (wale) launch_pipe<OL_OP_CUMULANT, true>(L, s);
      else launch_pipe<OL_OP_CUMULANT, false>(L, s);
    } else {
      if (wale) launch_pipe<OL_OP_REGULARIZED_BGK, true>(L, s);
      else launch_pipe<OL_OP_REGULARIZED_BGK, false>(L, s);
    }
  }
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
  L.ghost = lv->ghost;
  L.ghost_next = lv->ghost_next;
  L.ghost_mode = lv->ghost_mode;
  L.gblocks = lv->ghost_blocks;
  L.n_gblocks = lv->n_ghost_blocks;
  OL_CHECK_ARG(lv->n_ghost_blocks >= 0 && lv->n_ghost_blocks <= lv->n_blocks &&
                   (lv->n_ghost_blocks == 0 || lv->ghost_blocks),
               "ol_stream_collide: bad ghost block list");
  OL_CHECK_ARG(lv->ghost_mode >= OL_GHOST_UNPAIRED && lv->ghost_mode <= OL_GHOST_PAIR_SECOND,
               "ol_stream_collide: unknown ghost_mode %d", lv->ghost_mode);
  OL_CHECK_ARG(lv->ghost_mode == OL_GHOST_UNPAIRED || (lv->ghost && !sp->is_level_1),
               "ol_stream_collide: ghost pairing needs a fine level and the ghost scratch");
  OL_CHECK_ARG(lv->ghost_mode != OL_GHOST_PAIR_FIRST ||
                   (lv->ghost_next && lv->ghost_next != lv->ghost && sp->temporal_weight == 0.0f),
               "ol_stream_collide: OL_GHOST_PAIR_FIRST needs a distinct ghost_next and "
               "temporal weight 0");
  OL_CHECK_ARG(lv->ghost_mode != OL_GHOST_PAIR_SECOND || sp->temporal_weight == 0.5f,
               "ol_stream_collide: OL_GHOST_PAIR_SECOND needs temporal weight 1/2");
  L.sp = *sp;
  OL_CHECK_ARG((int64_t)lv->n_blocks * BCELLS < (1LL << 31),
               "ol_stream_collide: n_blocks too large for 32-bit plane offsets");
  L.halo_tab = halo_table_device();
  if (!L.halo_tab) return set_error(OL_ERR_CUDA, "ol_stream_collide: staging table allocation failed");
  if (!sp->is_level_1) {
    OL_CHECK_ARG(pv && pv->f && pv->rho && pv->vel && pv->block_ptr && pv->n_blocks > 0,
                 "ol_stream_collide: fine level needs a parent view");
    OL_CHECK_ARG(!(sp->use_temporal_interp == 1 && sp->temporal_weight < 0.99f) ||
                     (pv->f_old && pv->rho_old && pv->vel_old),
                 "ol_stream_collide: temporal interpolation needs parent old state");
    OL_CHECK_ARG((int64_t)pv->n_blocks * BCELLS < (1LL << 31),
                 "ol_stream_collide: parent n_blocks too large for 32-bit cell indices");
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

extern "C" int ol_set_stream_collide_kernel(int32_t choice, int32_t max_ctas) {
  OL_CHECK_ARG(choice == OL_SC_KERNEL_AUTO || choice == OL_SC_KERNEL_BLOCK ||
                   choice == OL_SC_KERNEL_WS,
               "ol_set_stream_collide_kernel: unknown choice %d", choice);
  OL_CHECK_ARG(max_ctas >= 0, "ol_set_stream_collide_kernel: max_ctas < 0");
  g_sc_kernel = choice;
  g_ws_max_ctas = max_ctas;
  return OL_OK;
}

extern "C" int ol_pipeline_fault(int32_t *flags) {
  OL_CHECK_ARG(flags, "ol_pipeline_fault: null output");
  int *d = fault_word_device();
  if (!d) return set_error(OL_ERR_CUDA, "ol_pipeline_fault: fault word allocation failed");
  int v = 0;
  OL_CUDA(cudaMemcpy(&v, d, sizeof(int), cudaMemcpyDeviceToHost));
  OL_CUDA(cudaMemset(d, 0, sizeof(int)));
  *flags = v;
  return OL_OK;
}

extern "C" int ol_staging_tables(uint32_t *halo, int32_t halo_cap, uint32_t *ws, int32_t ws_cap,
                                 int32_t *sizes) {
  OL_CHECK_ARG(sizes, "ol_staging_tables: null sizes");
  const std::vector<uint32_t> h = build_halo_table(), w = build_ws_table();
  sizes[0] = (int32_t)h.size();
  sizes[1] = (int32_t)w.size();
  sizes[2] = kSPlane;
  sizes[3] = kSPad;
  if (halo && halo_cap >= (int32_t)h.size()) std::copy(h.begin(), h.end(), halo);
  if (ws && ws_cap >= (int32_t)w.size()) std::copy(w.begin(), w.end(), ws);
  return OL_OK;
}

extern "C" int64_t ol_ghost_floats(int32_t n_blocks) {
  return n_blocks > 0 ? (int64_t)n_blocks * kHaloEntries : 0;
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
