// Native context: a device block pool shared by many cases, FP32 or
// FP16-shifted population storage, and a coarse time step for every resident
// case replayed from one CUDA graph.
//
// Schedule.  One coarse step of a case with L levels is the pre-order walk
// of the 2:1 recursion (solver_control.jl:6-218): level 1 once, then each
// child twice per parent step, the second child sub-step at temporal weight
// 1/2.  With Lmax the deepest resident case, the walk for Lmax gives the
// slot sequence (level, sub-step j); a case of depth L takes part in the
// slots of levels <= L, which keeps its own order intact.  Each slot is one
// persistent stream-collide launch per kernel variant over the work list of
// all (case, level, block) items of that slot, followed by the batched
// Bouzidi gather/scatter of the slot.
//
// Time-dependent fields (A/B parity, inlet ramp, noise seed, parent state
// pointers) live in the descriptors in device memory and are refreshed by
// k_advance at the head of each replay from each case's device clock, so
// the captured graph is valid for every step; k_tick advances the clocks at
// the tail.  copy_to_old! (blocks.jl:241-252) needs no copy here: the
// parent's pull source of its current step stays untouched until its next
// step, so "old" f/vel are the other half of the A/B pair, and rho (a single
// buffer in the reference) is kept as an A/B pair too.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "batched.cuh"
#include "coeffs.cuh"
#include "pipe.cuh"
#include "ws.cuh"
#include "common.cuh"
#include "forces.cuh"

namespace ol {

// ------------------------------------------------------------------ kernels

__global__ void k_advance(LevelDev *descs, ThermalDev *tdescs, const DescMeta *meta,
                          const CaseDev *cases, PoolBufs P, int n_desc) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n_desc) return;
  const DescMeta m = meta[d];
  const CaseDev c = cases[m.case_slot];
  const int64_t t = c.t + 1;  // the coarse step being executed (reference t starts at 1)
  const int64_t t_sub = t * ((int64_t)1 << (m.level - 1)) + m.j;
  const bool even = (t_sub & 1) == 0;
  LevelDev &L = descs[d];
  L.f_in = even ? P.fA : P.fB;
  L.f_out = even ? P.fB : P.fA;
  L.vel_in = even ? P.velA : P.velB;
  L.vel_out = even ? P.velB : P.velA;
  L.rho_out = even ? P.rhoB : P.rhoA;
  // inlet ramp evaluated per batch of async_depth steps at the batch end (main.jl:214-218)
  const int ad = c.async_depth > 0 ? c.async_depth : 1;
  const int64_t batch_end = ((t - 1) / ad + 1) * ad;
  float prog = 1.0f;
  if (c.ramp_steps > 0 && batch_end <= c.ramp_steps)
    prog = 0.5f * (1.0f - cosf(3.14159265358979f * (float)batch_end / (float)c.ramp_steps));
  L.sp.u_inlet = c.u_target * prog;
  L.sp.time_step_seed = (int32_t)(t_sub % 1000000);
  L.sp.temporal_weight = (t_sub & 1) ? 0.5f : 0.0f;
  if (m.has_parent) {
    const int64_t tp = t * ((int64_t)1 << (m.level - 2)) + (m.j >> 1);
    const bool pe = (tp & 1) == 0;
    L.pf = pe ? P.fB : P.fA;          // parent f_out of its current step
    L.pf_old = pe ? P.fA : P.fB;      // parent f_in (untouched pull source)
    L.prho = pe ? P.rhoB : P.rhoA;
    L.prho_old = pe ? P.rhoA : P.rhoB;
    L.pvel = pe ? P.velB : P.velA;
    L.pvel_old = pe ? P.velA : P.velB;
  }
  if (m.ddf) {
    ThermalDev &D = tdescs[d];
    D.g_in = even ? P.gA : P.gB;
    D.g_out = even ? P.gB : P.gA;
    D.T_out = even ? P.TB : P.TA;
    D.vel = L.vel_out;
    D.tp.u_inlet = L.sp.u_inlet;
    D.tp.temporal_weight = L.sp.temporal_weight;
    if (m.has_parent) {
      const int64_t tp = t * ((int64_t)1 << (m.level - 2)) + (m.j >> 1);
      const bool pe = (tp & 1) == 0;
      D.pg = pe ? P.gB : P.gA;
      D.pg_old = pe ? P.gA : P.gB;
      D.pT = pe ? P.TB : P.TA;
      D.pT_old = pe ? P.TA : P.TB;
      D.pvel = pe ? P.velB : P.velA;
      D.pvel_old = pe ? P.velA : P.velB;
    }
  }
}

__global__ void k_tick(CaseDev *cases, int n_cases, int only_slot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_cases && (only_slot < 0 || i == only_slot)) cases[i].t += 1;
}

// Descriptor of the current work item, copied into shared memory by the CTA.
template <class DEV>
__device__ __forceinline__ void copy_desc(DEV *dst, const DEV *src, int t) {
  constexpr int n4 = sizeof(DEV) / 4;
  static_assert(sizeof(DEV) % 4 == 0, "descriptor size");
  const uint32_t *s = (const uint32_t *)src;
  uint32_t *d = (uint32_t *)dst;
  for (int i = t; i < n4; i += blockDim.x) d[i] = s[i];
}

// Boundary values of absent neighbours for the ghost blocks of many cases:
// one CTA per (descriptor, block) item.
template <class ST>
__global__ void __launch_bounds__(kGhostThreads, kGhostMinBlocks)
    k_ghost_fill_b(const LevelDev *__restrict__ descs, const WorkItem *__restrict__ items) {
  __shared__ __align__(16) LevelDev L;
  const WorkItem w = items[blockIdx.x];
  copy_desc(&L, descs + w.desc, threadIdx.x);
  __syncthreads();
  ghost_fill_block<ST>(L, w.block, ghost_row_of(L, w.block), ghost_next_row_of(L, w.block));
}

// The same for the thermal populations of DDF cases (thermal descriptors).
template <class ST>
__global__ void __launch_bounds__(kGhostThreads, kGhostMinBlocks)
    k_ghost_fill_tb(const ThermalDev *__restrict__ tdescs, const WorkItem *__restrict__ items) {
  __shared__ __align__(16) ThermalDev D;
  const WorkItem w = items[blockIdx.x];
  copy_desc(&D, tdescs + w.desc, threadIdx.x);
  __syncthreads();
  ghost_fill_block<ST>(D, w.block, ghost_row_of(D, w.block), ghost_next_row_of(D, w.block));
}

template <int OP, class ST, bool WALE, bool DDF>
__global__ void __launch_bounds__(512, OP == OL_OP_CUMULANT ? 2 : 1)
    k_sc_batched(const LevelDev *__restrict__ descs, const ThermalDev *__restrict__ tdescs,
                 const WorkItem *__restrict__ items, int n_items) {
  __shared__ __align__(16) LevelDev L;
  __shared__ __align__(16) ThermalDev D;
  __shared__ int nbbase[27];
  extern __shared__ float E[];
  const int t = threadIdx.x;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const WorkItem w = items[it];
    copy_desc(&L, descs + w.desc, t);
    if (DDF) copy_desc(&D, tdescs + w.desc, t);
    // this CTA's next item into L2 (measured: better than 3/4 of a grid ahead
    // here, where the CTAs stay resident and walk the list in step)
    if (it + (int)gridDim.x < n_items && t < 33) {
      const WorkItem w2 = items[it + gridDim.x];
      prefetch_block_l2<ST>(descs[w2.desc], w2.block, t);
    }
    __syncthreads();
    const int64_t own0 = (L.block_offset + w.block) * BCELLS;
    OwnRegs<ST> r;
    own_load(L.f_in, L.dstride, own0, t, r);
    const bool obs = L.obstacle[own0 + t] != 0;
    const float spg = L.sponge[own0 + t];
    const bool miss = load_nbbase_sync(L.nbr, L.nbr_stride, L.block_offset, w.block, t, nbbase);
    stage_flow<ST>(L, nbbase, w.block, t, E, miss, r);
    __syncthreads();
    stream_collide_cell<OP, ST, WALE>(L, nbbase, E, w.block, t, obs, spg);
    if (DDF) {
      __syncthreads();
      stage_thermal<ST>(D, nbbase, w.block, t, E, L.halo_tab, miss);
      __syncthreads();
      thermal_cell<ST>(D, nbbase, E, w.block, t);
    }
    __syncthreads();
  }
}

// Bouzidi for the Bouzidi lists of many cases over their static lists of cut
// links (built at case admission): one thread per link, the corrected
// values gathered into scratch, then scattered (the arithmetic of
// bouzidi_value, as the drop-in link kernels).
template <class ST>
__global__ void k_bouz_links_gather_b(const LevelDev *descs, const ThermalDev *tdescs,
                                      const BouzDev *bd, const BouzLinkItem *items, int64_t n,
                                      float *scratch) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const BouzLinkItem it = items[j];
  const BouzDev &B = bd[it.bdesc];
  using T = typename ST::T;
  const T *f = (const T *)(B.thermal ? tdescs[B.desc].g_out : descs[B.desc].f_out);
  const ol_bouzidi_link L = B.links[it.link];
  const int k = L.k;
  const size_t cell0 = (size_t)B.block_offset * BCELLS;
  const size_t own = cell0 + (size_t)L.cell;
  const float fk = ST::load(f, own + (size_t)k * B.dstride, k, B.inv_scale);
  float fother;
  if (L.q < 0.5f)
    fother = L.far_cell >= 0
                 ? ST::load(f, cell0 + (size_t)L.far_cell + (size_t)k * B.dstride, k, B.inv_scale)
                 : fk;
  else
    fother = ST::load(f, own + (size_t)opp_of(k) * B.dstride, opp_of(k), B.inv_scale);
  scratch[B.scratch_off + it.link] = bouzidi_value(L.q, fk, fother);
}

template <class ST>
__global__ void k_bouz_links_scatter_b(const LevelDev *descs, const ThermalDev *tdescs,
                                       const BouzDev *bd, const BouzLinkItem *items, int64_t n,
                                       const float *scratch) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const BouzLinkItem it = items[j];
  const BouzDev &B = bd[it.bdesc];
  void *f = B.thermal ? tdescs[B.desc].g_out : descs[B.desc].f_out;
  const ol_bouzidi_link L = B.links[it.link];
  const int ko = opp_of(L.k);
  ST::store((typename ST::T *)f, (size_t)B.block_offset * BCELLS + (size_t)L.cell +
                                     (size_t)ko * B.dstride,
            ko, B.scale, scratch[B.scratch_off + it.link]);
}

// Initial state of a pool region (main.jl:113-150): f = w (shifted FP16: 0),
// rho = 1, u = 0, g = w T0, T = T0, on both halves of every A/B pair.
template <class ST>
__global__ void k_init_region(PoolBufs P, int64_t first_cell, int64_t n_cells, int64_t dstride,
                              float scale, int ddf, float T0) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_cells) return;
  const int64_t c = first_cell + i;
  typename ST::T *fa = (typename ST::T *)P.fA, *fb = (typename ST::T *)P.fB;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    ST::store(fa, c + k * dstride, k, scale, w_of(k));
    ST::store(fb, c + k * dstride, k, scale, w_of(k));
  }
  P.rhoA[c] = 1.0f; P.rhoB[c] = 1.0f;
  for (int a = 0; a < 3; ++a) { P.velA[c + a * dstride] = 0.0f; P.velB[c + a * dstride] = 0.0f; }
  if (ddf) {
    typename ST::T *ga = (typename ST::T *)P.gA, *gb = (typename ST::T *)P.gB;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      ST::store(ga, c + k * dstride, k, scale, w_of(k) * T0);
      ST::store(gb, c + k * dstride, k, scale, w_of(k) * T0);
    }
    P.TA[c] = T0; P.TB[c] = T0;
  }
}

template <class ST>
__global__ void k_decode_region(const void *f, int64_t first_cell, int64_t n_cells, int64_t dstride,
                                float inv_scale, float *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_cells) return;
#pragma unroll
  for (int k = 0; k < 27; ++k)
    out[i + k * n_cells] =
        ST::load((const typename ST::T *)f, first_cell + i + k * dstride, k, inv_scale);
}

// ------------------------------------------------------------------ host

struct DevLevel {
  int32_t n_blocks = 0;
  int64_t block_offset = 0;
  int32_t *nbr = nullptr, *mx = nullptr, *my = nullptr, *mz = nullptr, *bptr = nullptr;
  int32_t dims[3] = {0, 0, 0};
  int32_t n_boundary = 0;
  uint16_t *q = nullptr;
  ol_bouzidi_link *links = nullptr;  // cut links, level-local cells
  int32_t n_links = 0;
  int32_t *cb = nullptr;
  int8_t *cx = nullptr, *cy = nullptr, *cz = nullptr;
  float tau = 0.5f, tau_g = 0.5f, scale = 1.0f;
  // refined levels: precomputed absent-neighbour values of the blocks that
  // have an absent neighbour (compact rows), block -> row index
  float *ghost = nullptr;
  float *ghost_g = nullptr;  // the same rows for the thermal populations (DDF cases)
  // rows of the second child sub-step of each parent step, written by the
  // first one's ghost pass (ghost pairing, LevelDev::ghost_mode)
  float *ghost2 = nullptr;
  float *ghost_g2 = nullptr;
  int32_t *gidx = nullptr;
  std::vector<int32_t> ghost_blocks;  // host copy of the blocks with a row
  std::vector<int32_t> edge_blocks;   // those of them with domain-boundary values
  std::vector<int32_t> ghost_work;    // absent-neighbour pulls of each, in list order
  std::vector<int32_t> edge_work;     // domain-boundary pulls of each edge block
};

// Out-of-block pulls a block makes from its neighbour in direction d: 484
// from a face neighbour, 22 from an edge, 1 from a corner (3176 in all).
static int pulls_from_neighbour(int d) {
  const int m = std::abs(d % 3 - 1) + std::abs((d / 3) % 3 - 1) + std::abs(d / 9 - 1);
  return m == 1 ? 484 : m == 2 ? 22 : m == 3 ? 1 : 0;
}

// The blocks with a nonzero work[b], largest first (ties by block id), and
// their work in that order: the ghost pass's visit order, so that its last
// CTAs are its shortest ones.
static void order_by_work(const std::vector<int32_t> &work, std::vector<int32_t> &blocks,
                          std::vector<int32_t> &sorted_work) {
  blocks.clear();
  for (int b = 0; b < (int)work.size(); ++b)
    if (work[b] > 0) blocks.push_back(b);
  std::stable_sort(blocks.begin(), blocks.end(),
                   [&](int32_t a, int32_t b) { return work[a] > work[b]; });
  sorted_work.clear();
  for (int32_t b : blocks) sorted_work.push_back(work[b]);
}

// Blocks of a level with at least one absent neighbour (neighbour table
// nB x 27 column-major, 0 = absent), by absent-neighbour pulls.
static void blocks_with_absent_neighbour(const ol_level_desc &S, std::vector<int32_t> &blocks,
                                         std::vector<int32_t> &work_out) {
  std::vector<int32_t> work((size_t)S.n_blocks, 0);
  for (int b = 0; b < S.n_blocks; ++b)
    for (int d = 0; d < 27; ++d)
      if (d != 13 && S.neighbor_table[b + (size_t)S.n_blocks * d] <= 0)
        work[b] += pulls_from_neighbour(d);
  order_by_work(work, blocks, work_out);
}
static size_t count_blocks_with_absent_neighbour(const ol_level_desc &S) {
  std::vector<int32_t> blocks, work;
  blocks_with_absent_neighbour(S, blocks, work);
  return blocks.size();
}

// The blocks with an absent neighbour not wholly inside the level's domain
// (n*_global cells per axis), by their pulls from such neighbours: the only
// blocks whose values the second sub-step of a pair evaluates (domain
// boundary conditions); every other absent-neighbour value is coarse-to-fine
// and set by the first.
static void blocks_with_domain_edge(const ol_level_desc &S, int nxg, int nyg, int nzg,
                                    std::vector<int32_t> &blocks,
                                    std::vector<int32_t> &work_out) {
  auto inside = [](int nb, int ng) { return nb >= 1 && (int64_t)nb * BS <= ng; };
  std::vector<int32_t> work((size_t)S.n_blocks, 0);
  for (int b = 0; b < S.n_blocks; ++b)
    for (int d = 0; d < 27; ++d) {
      if (d == 13 || S.neighbor_table[b + (size_t)S.n_blocks * d] > 0) continue;
      const int nbx = S.map_x[b] + d % 3 - 1, nby = S.map_y[b] + (d / 3) % 3 - 1,
                nbz = S.map_z[b] + d / 9 - 1;
      if (!inside(nbx, nxg) || !inside(nby, nyg) || !inside(nbz, nzg))
        work[b] += pulls_from_neighbour(d);
    }
  order_by_work(work, blocks, work_out);
}

struct NCase {
  int32_t id = -1;
  int32_t slot = -1;
  std::vector<DevLevel> levels;
  ol_step_params sp{};
  ol_thermal_params tp{};
  int ddf = 0;
  int nx = 0, ny = 0, nz = 0;
  float u_target = 0.f;
  float q_min = 0.001f;
  int ramp_steps = 0, async_depth = 8;
  int n_tri = 0;
  float *mesh = nullptr;  // 7 * n_tri floats: cx cy cz nx ny nz area
  ol_force_params force{};
  double *partials = nullptr;
  size_t bytes = 0;
  int64_t steps = 0;
};

struct Launch {
  int kind;     // 0 = stream-collide, 1/2 = bouzidi gather/scatter, 3/4 = flow/thermal ghosts
  int op = 0, wale = 0, ddf = 0;
  int64_t off = 0, n = 0;   // items (kind 0) or links (kind 1/2)
};

}  // namespace ol

struct ol_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t budget = 0, used = 0;
  bool f16 = false, ddf_pool = false;
  int n_sm = 148;
  int64_t capacity = 0;  // blocks
  ol::PoolBufs P{};
  uint8_t *obst = nullptr;
  float *sponge = nullptr, *wd = nullptr;
  std::map<int64_t, int64_t> free_ranges;  // start -> length (blocks)
  std::map<int32_t, std::unique_ptr<ol::NCase>> cases;
  int32_t next_id = 1;
  int32_t max_slots = 0;
  std::vector<int32_t> free_slots;
  ol::CaseDev *d_cases = nullptr;
  // plan
  ol::LevelDev *d_descs = nullptr;
  ol::ThermalDev *d_tdescs = nullptr;
  ol::DescMeta *d_meta = nullptr;
  ol::WorkItem *d_items = nullptr;
  ol::BouzDev *d_bdescs = nullptr;
  ol::BouzLinkItem *d_blitems = nullptr;
  float *d_bscratch = nullptr;
  int n_desc = 0;
  std::vector<ol::Launch> plan;
  int64_t launches_per_step = 0;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;
  // persistent grid = grid_mult * resident CTAs; 0 = one CTA per item;
  // -1 = software-pipelined kernel (FP32 without DDF); -2 = warp-specialised
  // persistent kernel (cumulant without DDF; the other variants then take
  // one CTA per item)
  int grid_mult = -2;
  // per collision variant [op][wale][ddf]: its own shape, or kShapeDefault
  // to follow grid_mult (set by ol_ctx_autotune when the mix holds more than
  // one variant)
  int variant_shape[2][2][2] = {{{-99, -99}, {-99, -99}}, {{-99, -99}, {-99, -99}}};
  // >= 0: the plan holds this case only (ol_ctx_case_step), -1: every case
  int32_t only_case = -1;
  int64_t launches = 0;
  double *d_out = nullptr;
  std::mutex mu;
};

namespace ol {

static size_t per_block_bytes(bool f16, bool ddf) {
  const size_t fb = f16 ? 2 : 4;
  size_t b = (size_t)BCELLS * (2 * 27 * fb + 2 * 4 + 2 * 12 + 1 + 4 + 4);
  if (ddf) b += (size_t)BCELLS * (2 * 27 * fb + 2 * 4);
  return b;
}

// IEEE binary16 bits -> float on the host (exact; the q-map holds binary16).
static float half_bits_to_float_host(uint16_t h) {
  const int e = (h >> 10) & 31, m = h & 1023;
  float v;
  if (e == 0) v = std::ldexp((float)m, -24);
  else if (e == 31) v = m ? NAN : INFINITY;
  else v = std::ldexp((float)(m | 1024), e - 25);
  return (h & 0x8000) ? -v : v;
}

// The level's cut links (q in (q_min, 1]) in direction-major order, as
// k_bouzidi_build_links builds them on the device for the drop-in path.
static std::vector<ol_bouzidi_link> cut_links(const ol_level_desc &S, float q_min) {
  std::vector<ol_bouzidi_link> out;
  const size_t Sd = (size_t)S.n_blocks * BCELLS;
  for (int k = 0; k < 27; ++k)
    for (int i = 0; i < S.n_boundary; ++i) {
      const int b = S.cell_block[i] - 1;
      const int x = S.cell_x[i] - 1, y = S.cell_y[i] - 1, z = S.cell_z[i] - 1;
      const int own = b * BCELLS + x + BS * y + BS * BS * z;
      const uint16_t h = S.q_map[own + k * Sd];
      // positive binary16 values order like their bits: skip 0, negatives,
      // NaN and values above 1 (0x3C00) before converting
      if (h == 0 || (h & 0x8000) || h > 0x3C00) continue;
      const float q = half_bits_to_float_host(h);
      if (!(q > q_min && q <= 1.0f)) continue;
      ol_bouzidi_link L{own, -1, q, k};
      if (q < 0.5f) {
        const int nx = x - cx_of(k), ny = y - cy_of(k), nz = z - cz_of(k);
        if (nx >= 0 && nx < BS && ny >= 0 && ny < BS && nz >= 0 && nz < BS) {
          L.far_cell = b * BCELLS + nx + BS * ny + BS * BS * nz;
        } else {
          const int ox = nx < 0 ? -1 : (nx >= BS ? 1 : 0);
          const int oy = ny < 0 ? -1 : (ny >= BS ? 1 : 0);
          const int oz = nz < 0 ? -1 : (nz >= BS ? 1 : 0);
          const int nb = S.neighbor_table[b + (size_t)S.n_blocks *
                                                  ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1))];
          if (nb > 0) L.far_cell = (nb - 1) * BCELLS + (nx & 7) + BS * (ny & 7) + BS * BS * (nz & 7);
        }
      }
      out.push_back(L);
    }
  return out;
}

static size_t case_meta_bytes(const ol_case_desc *cd) {
  size_t b = 0;
  for (int l = 0; l < cd->n_levels; ++l) {
    const ol_level_desc &L = cd->levels[l];
    b += (size_t)L.n_blocks * (27 + 3) * 4 + (size_t)L.dim_x * L.dim_y * L.dim_z * 4;
    b += (size_t)L.n_boundary * (27 * 2 + 4 + 3);
    if (L.n_boundary > 0)
      b += cut_links(L, cd->q_min_threshold > 0.0f ? cd->q_min_threshold : 0.001f).size() *
           sizeof(ol_bouzidi_link);
    if (l > 0)  // ghost rows of both sub-steps of a pair, flow (+ thermal)
      b += count_blocks_with_absent_neighbour(L) * kHaloEntries * sizeof(float) * 2 *
               (cd->ddf ? 2 : 1) +
           (size_t)L.n_blocks * sizeof(int32_t);
  }
  b += (size_t)cd->n_triangles * 7 * 4 + force_partial_rows(cd->n_triangles) * 9 * 8 + 256;
  return b;
}

static int64_t range_alloc(ol_ctx *c, int64_t n) {
  for (auto it = c->free_ranges.begin(); it != c->free_ranges.end(); ++it) {
    if (it->second >= n) {
      const int64_t start = it->first, len = it->second;
      c->free_ranges.erase(it);
      if (len > n) c->free_ranges[start + n] = len - n;
      return start;
    }
  }
  return -1;
}

static void range_free(ol_ctx *c, int64_t start, int64_t n) {
  auto it = c->free_ranges.emplace(start, n).first;
  auto nx = std::next(it);
  if (nx != c->free_ranges.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    c->free_ranges.erase(nx);
  }
  if (it != c->free_ranges.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      c->free_ranges.erase(it);
    }
  }
}

template <class T>
static int upload(T **dst, const T *src, size_t n) {
  *dst = nullptr;
  if (n == 0) return OL_OK;
  OL_CUDA(cudaMalloc(dst, n * sizeof(T)));
  OL_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return OL_OK;
}

static void free_case_meta(NCase &c) {
  for (auto &L : c.levels) {
    cudaFree(L.nbr); cudaFree(L.mx); cudaFree(L.my); cudaFree(L.mz); cudaFree(L.bptr);
    cudaFree(L.q); cudaFree(L.cb); cudaFree(L.cx); cudaFree(L.cy); cudaFree(L.cz);
    cudaFree(L.links);
    cudaFree(L.ghost); cudaFree(L.ghost_g); cudaFree(L.ghost2); cudaFree(L.ghost_g2);
    cudaFree(L.gidx);
  }
  cudaFree(c.mesh);
  cudaFree(c.partials);
}

static void free_plan(ol_ctx *c) {
  if (c->exec) cudaGraphExecDestroy(c->exec);
  c->exec = nullptr;
  cudaFree(c->d_descs); cudaFree(c->d_tdescs); cudaFree(c->d_meta); cudaFree(c->d_items);
  cudaFree(c->d_bdescs); cudaFree(c->d_blitems); cudaFree(c->d_bscratch);
  c->d_descs = nullptr; c->d_tdescs = nullptr; c->d_meta = nullptr; c->d_items = nullptr;
  c->d_bdescs = nullptr; c->d_blitems = nullptr; c->d_bscratch = nullptr;
  c->plan.clear();
  c->n_desc = 0;
}

static int kernel_occupancy(int op) { return op == OL_OP_CUMULANT ? 2 : 1; }

constexpr int kGridWs = -2;
constexpr int kShapeDefault = -99;

// Launch shape of a stream-collide launch group: its variant's own shape
// when the autotuner set one, else the context's.
static int shape_for(const ol_ctx *c, const Launch &l) {
  const int s = c->variant_shape[l.op & 1][l.wale ? 1 : 0][l.ddf ? 1 : 0];
  return s == kShapeDefault ? c->grid_mult : s;
}

template <int OP, class ST, bool WALE, bool DDF>
static void launch_variant(ol_ctx *c, const Launch &l) {
  if constexpr (OP == OL_OP_CUMULANT && !DDF) {
    // by default FP32 only: with FP16-shifted storage the warp-specialised
    // kernel measured slower than one CTA per item (its consumers decode
    // every landed value)
    const int choice = stream_collide_kernel_choice();
    const bool f32 = std::is_same<ST, StoreF32>::value;
    if (choice == OL_SC_KERNEL_WS ||
        (f32 && shape_for(c, l) == kGridWs && choice == OL_SC_KERNEL_AUTO)) {
      const int grid = ws_grid(l.n, c->n_sm);
      k_sc_ws<OP, ST, WALE, true><<<(unsigned)grid, kWsThreads, ws_smem_bytes<ST>(), c->stream>>>(
          LevelDev{}, c->d_descs, c->d_items + l.off, (int)l.n, ws_table_device(),
          fault_word_device());
      return;
    }
  }
  const int gm = shape_for(c, l);
  if (std::is_same<ST, StoreF32>::value && !DDF && gm == -1) {
    // software-pipelined persistent kernel: all resident CTAs
    const int64_t grid = std::min<int64_t>(l.n, (int64_t)c->n_sm * kernel_occupancy(OP));
    k_sc_pipe<OP, WALE, true><<<(unsigned)grid, BCELLS, kPipeBytes, c->stream>>>(
        LevelDev{}, c->d_descs, c->d_items + l.off, (int)l.n);
    return;
  }
  const int64_t resident = (int64_t)c->n_sm * kernel_occupancy(OP);
  int64_t grid = gm <= 0 ? l.n : std::min<int64_t>(l.n, resident * gm);
  if (grid < 1) grid = 1;
  k_sc_batched<OP, ST, WALE, DDF><<<(unsigned)grid, BCELLS, kStageBytes, c->stream>>>(
      c->d_descs, c->d_tdescs, c->d_items + l.off, (int)l.n);
}

template <class ST>
static void launch_sc_dispatch(ol_ctx *c, const Launch &l) {
#define OL_VAR(OPV, W, D)                                                  \
  if (l.op == OPV && l.wale == W && l.ddf == D) {                          \
    launch_variant<OPV, ST, W != 0, D != 0>(c, l);                         \
    return;                                                                \
  }
  OL_VAR(0, 0, 0) OL_VAR(0, 1, 0) OL_VAR(0, 0, 1) OL_VAR(0, 1, 1)
  OL_VAR(1, 0, 0) OL_VAR(1, 1, 0) OL_VAR(1, 0, 1) OL_VAR(1, 1, 1)
#undef OL_VAR
}

static void record_step(ol_ctx *c) {
  const int nd = c->n_desc;
  k_advance<<<(nd + 127) / 128, 128, 0, c->stream>>>(c->d_descs, c->d_tdescs, c->d_meta,
                                                     c->d_cases, c->P, nd);
  for (const Launch &l : c->plan) {
    if (l.kind == 0) {
      if (c->f16) launch_sc_dispatch<StoreF16S>(c, l);
      else launch_sc_dispatch<StoreF32>(c, l);
    } else if (l.kind == 4) {
      if (c->f16)
        k_ghost_fill_tb<StoreF16S><<<(unsigned)l.n, kGhostThreads, 0, c->stream>>>(
            c->d_tdescs, c->d_items + l.off);
      else
        k_ghost_fill_tb<StoreF32><<<(unsigned)l.n, kGhostThreads, 0, c->stream>>>(
            c->d_tdescs, c->d_items + l.off);
    } else if (l.kind == 3) {
      if (c->f16)
        k_ghost_fill_b<StoreF16S><<<(unsigned)l.n, kGhostThreads, 0, c->stream>>>(
            c->d_descs, c->d_items + l.off);
      else
        k_ghost_fill_b<StoreF32><<<(unsigned)l.n, kGhostThreads, 0, c->stream>>>(
            c->d_descs, c->d_items + l.off);
    } else {
      const unsigned g = (unsigned)((l.n + 255) / 256);
      const BouzLinkItem *items = c->d_blitems + l.off;
      if (l.kind == 1) {
        if (c->f16)
          k_bouz_links_gather_b<StoreF16S><<<g, 256, 0, c->stream>>>(
              c->d_descs, c->d_tdescs, c->d_bdescs, items, l.n, c->d_bscratch);
        else
          k_bouz_links_gather_b<StoreF32><<<g, 256, 0, c->stream>>>(
              c->d_descs, c->d_tdescs, c->d_bdescs, items, l.n, c->d_bscratch);
      } else {
        if (c->f16)
          k_bouz_links_scatter_b<StoreF16S><<<g, 256, 0, c->stream>>>(
              c->d_descs, c->d_tdescs, c->d_bdescs, items, l.n, c->d_bscratch);
        else
          k_bouz_links_scatter_b<StoreF32><<<g, 256, 0, c->stream>>>(
              c->d_descs, c->d_tdescs, c->d_bdescs, items, l.n, c->d_bscratch);
      }
    }
  }
  const int only_slot = c->only_case >= 0 ? c->cases.at(c->only_case)->slot : -1;
  k_tick<<<(c->max_slots + 127) / 128, 128, 0, c->stream>>>(c->d_cases, c->max_slots, only_slot);
}

// Build descriptors, work lists and the per-coarse-step graph.
static int rebuild(ol_ctx *c) {
  free_plan(c);
  c->dirty = false;
  if (c->cases.empty()) return OL_OK;
  int lmax = 0;
  for (auto &kv : c->cases)
    if (c->only_case < 0 || kv.first == c->only_case)
      lmax = std::max<int>(lmax, (int)kv.second->levels.size());
  std::vector<std::pair<int, int>> slots;  // (level, j)
  struct Walk {
    static void go(int l, int j, int lmax, std::vector<std::pair<int, int>> &out) {
      out.emplace_back(l, j);
      if (l < lmax) { go(l + 1, 2 * j, lmax, out); go(l + 1, 2 * j + 1, lmax, out); }
    }
  };
  Walk::go(1, 0, lmax, slots);

  std::vector<LevelDev> descs;
  std::vector<ThermalDev> tdescs;
  std::vector<DescMeta> meta;
  std::vector<WorkItem> items;
  std::vector<BouzDev> bdescs;
  std::vector<BouzLinkItem> blitems;  // one per cut link of the slot's lists
  std::vector<int32_t> bcount;         // links of each Bouzidi list
  int64_t scratch_max = 0;
  const int64_t dstride = c->capacity * BCELLS;
  const uint32_t *tab = halo_table_device();
  if (!tab) return set_error(OL_ERR_CUDA, "staging table allocation failed");
  int64_t per_step = 2;  // advance + tick

  for (const auto &sl : slots) {
    const int l = sl.first, j = sl.second;
    // descriptors of this slot, grouped by kernel variant
    std::map<int, std::vector<int>> groups;  // variant -> descriptor ids
    int64_t scratch_off = 0;
    std::vector<int> bz_flow, bz_therm;
    // (work, item): each ghost launch visits the blocks of all cases largest first
    std::vector<std::pair<int32_t, WorkItem>> ghost_items, tghost_items;
    for (auto &kv : c->cases) {
      NCase &cs = *kv.second;
      if (c->only_case >= 0 && kv.first != c->only_case) continue;
      if ((int)cs.levels.size() < l) continue;
      const DevLevel &V = cs.levels[l - 1];
      const int d = (int)descs.size();
      LevelDev L{};
      L.f_post = nullptr;
      L.obstacle = c->obst; L.sponge = c->sponge; L.wall_dist = c->wd;
      L.nbr = V.nbr; L.map_x = V.mx; L.map_y = V.my; L.map_z = V.mz;
      L.n_blocks = V.n_blocks;
      L.block_offset = V.block_offset;
      L.dstride = dstride;
      L.nbr_stride = V.n_blocks;
      L.scale = V.scale; L.inv_scale = 1.0f / V.scale;
      L.sp = cs.sp;
      L.sp.tau_molecular = V.tau;
      L.sp.is_level_1 = l == 1;
      const int sc = 1 << (l - 1);
      L.sp.nx_global = cs.nx * sc; L.sp.ny_global = cs.ny * sc; L.sp.nz_global = cs.nz * sc;
      L.sp.store_post_collision = 0;
      L.status = &c->d_cases[cs.slot].status;
      L.halo_tab = tab;
      if (l > 1) {
        const DevLevel &PV = cs.levels[l - 2];
        L.sp.tau_parent = PV.tau;
        L.pptr = PV.bptr; L.pdim_x = PV.dims[0]; L.pdim_y = PV.dims[1]; L.pdim_z = PV.dims[2];
        L.p_block_offset = PV.block_offset;
        L.p_dstride = dstride;
        L.p_inv_scale = 1.0f / PV.scale;
        // j even: first child sub-step of a parent step (weight 0), j odd:
        // the second (weight 1/2); for level >= 2 the parity of t_sub is j's
        const bool first = (j & 1) == 0;
        L.ghost = first ? V.ghost : V.ghost2;
        L.ghost_next = V.ghost2;
        L.ghost_mode = first ? kGhostPairFirst : kGhostPairSecond;
        L.gidx = V.gidx;
        const auto &gb = first ? V.ghost_blocks : V.edge_blocks;
        const auto &gw = first ? V.ghost_work : V.edge_work;
        for (size_t q = 0; q < gb.size(); ++q) ghost_items.push_back({gw[q], WorkItem{d, gb[q]}});
      } else {
        L.sp.tau_parent = 0.5f;
        L.p_inv_scale = 1.0f;
      }
      ThermalDev D{};
      if (cs.ddf) {
        D.g_post = nullptr; D.obstacle = c->obst; D.sponge = c->sponge;
        D.nbr = V.nbr; D.map_x = V.mx; D.map_y = V.my; D.map_z = V.mz;
        D.n_blocks = V.n_blocks; D.block_offset = V.block_offset; D.dstride = dstride;
        D.nbr_stride = V.n_blocks; D.scale = V.scale; D.inv_scale = 1.0f / V.scale;
        D.tp = cs.tp;
        D.tp.tau_g = V.tau_g;
        D.tp.is_level_1 = l == 1;
        D.tp.nx_global = cs.nx * sc; D.tp.ny_global = cs.ny * sc; D.tp.nz_global = cs.nz * sc;
        D.tp.store_post_collision = 0;
        D.halo_tab = tab;
        if (l > 1) {
          const DevLevel &PV = cs.levels[l - 2];
          D.tp.tau_g_parent = PV.tau_g;
          D.pptr = PV.bptr; D.pdim_x = PV.dims[0]; D.pdim_y = PV.dims[1]; D.pdim_z = PV.dims[2];
          D.p_block_offset = PV.block_offset; D.p_dstride = dstride;
          D.p_inv_scale = 1.0f / PV.scale;
          const bool first = (j & 1) == 0;
          D.ghost = first ? V.ghost_g : V.ghost_g2;
          D.ghost_next = V.ghost_g2;
          D.ghost_mode = first ? kGhostPairFirst : kGhostPairSecond;
          D.gidx = V.gidx;
          const auto &gb = first ? V.ghost_blocks : V.edge_blocks;
          const auto &gw = first ? V.ghost_work : V.edge_work;
          for (size_t q = 0; q < gb.size(); ++q)
            tghost_items.push_back({gw[q], WorkItem{d, gb[q]}});
        } else {
          D.tp.tau_g_parent = 0.5f;
          D.p_inv_scale = 1.0f;
        }
      }
      descs.push_back(L);
      tdescs.push_back(D);
      DescMeta m{};
      m.case_slot = cs.slot; m.level = l; m.j = j; m.has_parent = l > 1; m.ddf = cs.ddf;
      meta.push_back(m);
      const int variant = cs.sp.op * 4 + (cs.sp.c_wale != 0.0f ? 2 : 0) + (cs.ddf ? 1 : 0);
      groups[variant].push_back(d);
      if (V.n_links > 0) {
        BouzDev B{};
        B.q = V.q; B.dense_q = 0; B.cell_block = V.cb; B.cell_x = V.cx; B.cell_y = V.cy;
        B.cell_z = V.cz; B.n_boundary = V.n_boundary; B.nbr = V.nbr; B.nbr_stride = V.n_blocks;
        B.block_offset = V.block_offset; B.dstride = dstride; B.q_min = cs.q_min;
        B.scale = V.scale; B.inv_scale = 1.0f / V.scale; B.desc = d; B.thermal = 0;
        B.links = V.links;
        B.scratch_off = scratch_off;
        scratch_off += V.n_links;
        bz_flow.push_back((int)bdescs.size());
        bdescs.push_back(B);
        bcount.push_back(V.n_links);
        if (cs.ddf) {
          B.thermal = 1;
          B.scratch_off = scratch_off;
          scratch_off += V.n_links;
          bz_therm.push_back((int)bdescs.size());
          bdescs.push_back(B);
          bcount.push_back(V.n_links);
        }
      }
    }
    auto ghost_launch = [&](std::vector<std::pair<int32_t, WorkItem>> &gi, int kind) {
      if (gi.empty()) return;
      std::stable_sort(gi.begin(), gi.end(),
                       [](const std::pair<int32_t, WorkItem> &a,
                          const std::pair<int32_t, WorkItem> &b) { return a.first > b.first; });
      Launch gl{};
      gl.kind = kind;
      gl.off = (int64_t)items.size();
      for (const auto &w : gi) items.push_back(w.second);
      gl.n = (int64_t)gi.size();
      c->plan.push_back(gl);
      ++per_step;
    };
    ghost_launch(ghost_items, 3);   // boundary values of the refined levels first
    ghost_launch(tghost_items, 4);  // and of the thermal populations of DDF cases
    for (auto &g : groups) {
      Launch ln{};
      ln.kind = 0;
      ln.op = g.first / 4; ln.wale = (g.first >> 1) & 1; ln.ddf = g.first & 1;
      ln.off = (int64_t)items.size();
      for (int d : g.second)
        for (int b = 0; b < descs[d].n_blocks; ++b) items.push_back(WorkItem{d, b});
      ln.n = (int64_t)items.size() - ln.off;
      if (ln.n > 0) { c->plan.push_back(ln); ++per_step; }
    }
    for (int pass = 0; pass < 2; ++pass) {
      const std::vector<int> &lst = pass == 0 ? bz_flow : bz_therm;
      if (lst.empty()) continue;
      const int64_t first = (int64_t)blitems.size();
      for (int bi : lst)
        for (int l = 0; l < bcount[bi]; ++l) blitems.push_back(BouzLinkItem{bi, l});
      Launch g{}; g.kind = 1; g.off = first; g.n = (int64_t)blitems.size() - first;
      Launch s2 = g; s2.kind = 2;
      c->plan.push_back(g);
      c->plan.push_back(s2);
      per_step += 2;
    }
    scratch_max = std::max(scratch_max, scratch_off);
  }
  c->n_desc = (int)descs.size();
  int rc;
  if ((rc = upload(&c->d_descs, descs.data(), descs.size()))) return rc;
  if ((rc = upload(&c->d_tdescs, tdescs.data(), tdescs.size()))) return rc;
  if ((rc = upload(&c->d_meta, meta.data(), meta.size()))) return rc;
  if ((rc = upload(&c->d_items, items.data(), items.size()))) return rc;
  if ((rc = upload(&c->d_bdescs, bdescs.data(), bdescs.size()))) return rc;
  if ((rc = upload(&c->d_blitems, blitems.data(), blitems.size()))) return rc;
  if (scratch_max > 0) OL_CUDA(cudaMalloc(&c->d_bscratch, scratch_max * sizeof(float)));
  c->launches_per_step = per_step;

  // warm the kernel attributes outside capture, then capture one coarse step
  cudaGraph_t g = nullptr;
  OL_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  record_step(c);
  const cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  if (ce != cudaSuccess) return cuda_status(ce, "cudaStreamEndCapture");
  const cudaError_t ie = cudaGraphInstantiate(&c->exec, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return cuda_status(ie, "cudaGraphInstantiate");
  return OL_OK;
}

// Dynamic shared memory above 48 KB must be enabled before any capture.
template <class ST>
static void prepare_attributes_st() {
  const int a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaFuncSetAttribute(k_sc_batched<0, ST, false, false>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<0, ST, true, false>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<0, ST, false, true>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<0, ST, true, true>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<1, ST, false, false>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<1, ST, true, false>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<1, ST, false, true>, (cudaFuncAttribute)a, kStageBytes);
  cudaFuncSetAttribute(k_sc_batched<1, ST, true, true>, (cudaFuncAttribute)a, kStageBytes);
}
static int prepare_attributes() {
  const int a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaFuncSetAttribute(k_sc_pipe<0, false, true>, (cudaFuncAttribute)a, kPipeBytes);
  cudaFuncSetAttribute(k_sc_pipe<0, true, true>, (cudaFuncAttribute)a, kPipeBytes);
  cudaFuncSetAttribute(k_sc_pipe<1, false, true>, (cudaFuncAttribute)a, kPipeBytes);
  cudaFuncSetAttribute(k_sc_pipe<1, true, true>, (cudaFuncAttribute)a, kPipeBytes);
  prepare_attributes_st<StoreF32>();
  prepare_attributes_st<StoreF16S>();
  cudaFuncSetAttribute(k_sc_ws<0, StoreF32, false, true>, (cudaFuncAttribute)a,
                       ws_smem_bytes<StoreF32>());
  cudaFuncSetAttribute(k_sc_ws<0, StoreF32, true, true>, (cudaFuncAttribute)a,
                       ws_smem_bytes<StoreF32>());
  cudaFuncSetAttribute(k_sc_ws<0, StoreF16S, false, true>, (cudaFuncAttribute)a,
                       ws_smem_bytes<StoreF16S>());
  cudaFuncSetAttribute(k_sc_ws<0, StoreF16S, true, true>, (cudaFuncAttribute)a,
                       ws_smem_bytes<StoreF16S>());
  if (!fault_word_device() || !ws_table_device())
    return set_error(OL_ERR_CUDA, "warp-specialised kernel tables: allocation failed");
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? OL_OK : cuda_status(e, "cudaFuncSetAttribute");
}

}  // namespace ol

using namespace ol;

extern "C" int ol_ctx_create(ol_ctx **out, int device, size_t budget, int store_kind) {
  OL_CHECK_ARG(out, "ol_ctx_create: null out");
  *out = nullptr;
  const bool f16 = (store_kind & 1) == OL_STORE_F16;
  const bool ddf = (store_kind & 2) != 0;
  OL_CHECK_ARG((store_kind & ~3) == 0, "ol_ctx_create: unknown store kind %d", store_kind);
  OL_CUDA(cudaSetDevice(device));
  std::unique_ptr<ol_ctx> c(new ol_ctx());
  c->device = device;
  c->f16 = f16;
  c->ddf_pool = ddf;
  c->budget = budget;
  OL_CUDA(cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, device));
  OL_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  const size_t pb = per_block_bytes(f16, ddf);
  const size_t pool_bytes = budget - budget / 16;  // 1/16 kept for per-case metadata
  c->capacity = (int64_t)(pool_bytes / pb);
  OL_CHECK_ARG(c->capacity >= 1, "ol_ctx_create: budget below one block");
  OL_CHECK_ARG(c->capacity * BCELLS < (1LL << 31), "ol_ctx_create: pool beyond 32-bit plane offsets");
  const size_t cells = (size_t)c->capacity * BCELLS;
  const size_t fb = f16 ? 2 : 4;
  OL_CUDA(cudaMalloc(&c->P.fA, cells * 27 * fb));
  OL_CUDA(cudaMalloc(&c->P.fB, cells * 27 * fb));
  OL_CUDA(cudaMalloc(&c->P.rhoA, cells * 4));
  OL_CUDA(cudaMalloc(&c->P.rhoB, cells * 4));
  OL_CUDA(cudaMalloc(&c->P.velA, cells * 12));
  OL_CUDA(cudaMalloc(&c->P.velB, cells * 12));
  if (ddf) {
    OL_CUDA(cudaMalloc(&c->P.gA, cells * 27 * fb));
    OL_CUDA(cudaMalloc(&c->P.gB, cells * 27 * fb));
    OL_CUDA(cudaMalloc(&c->P.TA, cells * 4));
    OL_CUDA(cudaMalloc(&c->P.TB, cells * 4));
  }
  OL_CUDA(cudaMalloc(&c->obst, cells));
  OL_CUDA(cudaMalloc(&c->sponge, cells * 4));
  OL_CUDA(cudaMalloc(&c->wd, cells * 4));
  c->used = (size_t)c->capacity * pb;
  c->free_ranges[0] = c->capacity;
  c->max_slots = 256;
  OL_CUDA(cudaMalloc(&c->d_cases, sizeof(CaseDev) * c->max_slots));
  OL_CUDA(cudaMemset(c->d_cases, 0, sizeof(CaseDev) * c->max_slots));
  for (int i = c->max_slots - 1; i >= 0; --i) c->free_slots.push_back(i);
  OL_CUDA(cudaMalloc(&c->d_out, 16 * sizeof(double)));
  if (!halo_table_device()) return set_error(OL_ERR_CUDA, "staging table allocation failed");
  {
    const int rc = prepare_attributes();
    if (rc) return rc;
  }
  c->used = 0;
  *out = c.release();
  return OL_OK;
}

extern "C" int ol_ctx_destroy(ol_ctx *c) {
  if (!c) return OL_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  free_plan(c);
  for (auto &kv : c->cases) free_case_meta(*kv.second);
  cudaFree(c->P.fA); cudaFree(c->P.fB); cudaFree(c->P.rhoA); cudaFree(c->P.rhoB);
  cudaFree(c->P.velA); cudaFree(c->P.velB); cudaFree(c->P.gA); cudaFree(c->P.gB);
  cudaFree(c->P.TA); cudaFree(c->P.TB); cudaFree(c->obst); cudaFree(c->sponge); cudaFree(c->wd);
  cudaFree(c->d_cases); cudaFree(c->d_out);
  cudaStreamDestroy(c->stream);
  delete c;
  return OL_OK;
}

static int validate_case(ol_ctx *c, const ol_case_desc *cd) {
  OL_CHECK_ARG(cd && cd->n_levels >= 1 && cd->levels, "case: needs at least one level");
  OL_CHECK_ARG(cd->n_levels <= 8, "case: at most 8 levels");
  OL_CHECK_ARG(!cd->ddf || c->ddf_pool, "case: thermal DDF needs a context created with the DDF flag");
  OL_CHECK_ARG(cd->params.op == OL_OP_CUMULANT || cd->params.op == OL_OP_REGULARIZED_BGK,
               "case: unknown operator");
  for (int l = 0; l < cd->n_levels; ++l) {
    const ol_level_desc &L = cd->levels[l];
    OL_CHECK_ARG(L.n_blocks > 0 && L.map_x && L.map_y && L.map_z && L.neighbor_table &&
                     L.block_ptr && L.obstacle && L.sponge,
                 "case: level %d is missing arrays", l + 1);
    OL_CHECK_ARG(L.n_boundary == 0 || (L.q_map && L.cell_block && L.cell_x && L.cell_y && L.cell_z),
                 "case: level %d Bouzidi lists missing", l + 1);
    OL_CHECK_ARG(L.store_scale > 0.0f || !c->f16, "case: level %d needs a positive FP16 scale", l + 1);
  }
  return OL_OK;
}

extern "C" int ol_ctx_case_footprint(ol_ctx *c, const ol_case_desc *cd, size_t *bytes) {
  OL_CHECK_ARG(c && cd && bytes, "ol_ctx_case_footprint: null argument");
  int rc = validate_case(c, cd);
  if (rc) return rc;
  size_t blocks = 0;
  for (int l = 0; l < cd->n_levels; ++l) blocks += cd->levels[l].n_blocks;
  *bytes = blocks * per_block_bytes(c->f16, c->ddf_pool) + case_meta_bytes(cd);
  return OL_OK;
}

extern "C" int ol_ctx_case_add(ol_ctx *c, const ol_case_desc *cd, int32_t *case_id) {
  OL_CHECK_ARG(c && cd && case_id, "ol_ctx_case_add: null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  OL_CUDA(cudaSetDevice(c->device));
  int rc = validate_case(c, cd);
  if (rc) return rc;
  size_t fp = 0;
  ol_ctx_case_footprint(c, cd, &fp);
  if (c->used + fp > c->budget)
    return set_error(OL_ERR_NOMEM, "ol_ctx_case_add: footprint %zu B exceeds the remaining budget %zu B",
                     fp, c->budget - c->used);
  if (c->free_slots.empty()) return set_error(OL_ERR_NOMEM, "ol_ctx_case_add: too many resident cases");
  OL_CUDA(cudaStreamSynchronize(c->stream));
  std::unique_ptr<NCase> cs(new NCase());
  cs->levels.resize(cd->n_levels);
  std::vector<std::pair<int64_t, int64_t>> got;
  for (int l = 0; l < cd->n_levels; ++l) {
    const int64_t off = range_alloc(c, cd->levels[l].n_blocks);
    if (off < 0) {
      for (auto &g : got) range_free(c, g.first, g.second);
      return set_error(OL_ERR_NOMEM, "ol_ctx_case_add: block pool fragmented/full");
    }
    got.emplace_back(off, cd->levels[l].n_blocks);
    cs->levels[l].block_offset = off;
  }
  const int64_t dstride = c->capacity * BCELLS;
  for (int l = 0; l < cd->n_levels; ++l) {
    const ol_level_desc &S = cd->levels[l];
    DevLevel &V = cs->levels[l];
    V.n_blocks = S.n_blocks;
    V.dims[0] = S.dim_x; V.dims[1] = S.dim_y; V.dims[2] = S.dim_z;
    V.tau = S.tau; V.tau_g = S.tau_g; V.scale = c->f16 ? S.store_scale : 1.0f;
    if ((rc = upload(&V.nbr, S.neighbor_table, (size_t)S.n_blocks * 27))) return rc;
    if ((rc = upload(&V.mx, S.map_x, (size_t)S.n_blocks))) return rc;
    if ((rc = upload(&V.my, S.map_y, (size_t)S.n_blocks))) return rc;
    if ((rc = upload(&V.mz, S.map_z, (size_t)S.n_blocks))) return rc;
    if ((rc = upload(&V.bptr, S.block_ptr, (size_t)S.dim_x * S.dim_y * S.dim_z))) return rc;
    const size_t c0 = (size_t)V.block_offset * BCELLS, nc = (size_t)S.n_blocks * BCELLS;
    OL_CUDA(cudaMemcpy(c->obst + c0, S.obstacle, nc, cudaMemcpyHostToDevice));
    OL_CUDA(cudaMemcpy(c->sponge + c0, S.sponge, nc * 4, cudaMemcpyHostToDevice));
    if (S.wall_dist) {
      OL_CUDA(cudaMemcpy(c->wd + c0, S.wall_dist, nc * 4, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> far(nc, 100.0f);
      OL_CUDA(cudaMemcpy(c->wd + c0, far.data(), nc * 4, cudaMemcpyHostToDevice));
    }
    if (l > 0) {
      blocks_with_absent_neighbour(S, V.ghost_blocks, V.ghost_work);
      std::vector<int32_t> gi((size_t)S.n_blocks, -1);
      for (size_t r = 0; r < V.ghost_blocks.size(); ++r) gi[V.ghost_blocks[r]] = (int32_t)r;
      if ((rc = upload(&V.gidx, gi.data(), gi.size()))) return rc;
      const int sc = 1 << l;
      blocks_with_domain_edge(S, cd->nx * sc, cd->ny * sc, cd->nz * sc, V.edge_blocks,
                              V.edge_work);
      if (!V.ghost_blocks.empty()) {
        const size_t gb = V.ghost_blocks.size() * kHaloEntries * sizeof(float);
        OL_CUDA(cudaMalloc(&V.ghost, gb));
        OL_CUDA(cudaMalloc(&V.ghost2, gb));
        if (cd->ddf) {
          OL_CUDA(cudaMalloc(&V.ghost_g, gb));
          OL_CUDA(cudaMalloc(&V.ghost_g2, gb));
        }
      }
    }
    V.n_boundary = S.n_boundary;
    if (S.n_boundary > 0) {
      // dense q-map -> sparse rows of 27 for the boundary cells
      std::vector<uint16_t> qs((size_t)S.n_boundary * 27);
      const size_t Sd = (size_t)S.n_blocks * BCELLS;
      for (int i = 0; i < S.n_boundary; ++i) {
        const size_t own = (size_t)(S.cell_block[i] - 1) * BCELLS + (S.cell_x[i] - 1) +
                           8 * (S.cell_y[i] - 1) + 64 * (S.cell_z[i] - 1);
        for (int k = 0; k < 27; ++k) qs[(size_t)i * 27 + k] = S.q_map[own + k * Sd];
      }
      if ((rc = upload(&V.q, qs.data(), qs.size()))) return rc;
      const std::vector<ol_bouzidi_link> links =
          cut_links(S, cd->q_min_threshold > 0.0f ? cd->q_min_threshold : 0.001f);
      V.n_links = (int32_t)links.size();
      if (!links.empty() && (rc = upload(&V.links, links.data(), links.size()))) return rc;
      if ((rc = upload(&V.cb, S.cell_block, (size_t)S.n_boundary))) return rc;
      if ((rc = upload(&V.cx, S.cell_x, (size_t)S.n_boundary))) return rc;
      if ((rc = upload(&V.cy, S.cell_y, (size_t)S.n_boundary))) return rc;
      if ((rc = upload(&V.cz, S.cell_z, (size_t)S.n_boundary))) return rc;
    }
    const int64_t n = (int64_t)S.n_blocks * BCELLS;
    const float T0 = cd->ddf ? cd->T_initial : 1.0f;
    if (c->f16)
      k_init_region<StoreF16S><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
          c->P, (int64_t)V.block_offset * BCELLS, n, dstride, V.scale, cd->ddf, T0);
    else
      k_init_region<StoreF32><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
          c->P, (int64_t)V.block_offset * BCELLS, n, dstride, 1.0f, cd->ddf, T0);
    OL_LAUNCHED("k_init_region");
  }
  cs->sp = cd->params;
  cs->tp = cd->tparams;
  cs->ddf = cd->ddf;
  cs->nx = cd->nx; cs->ny = cd->ny; cs->nz = cd->nz;
  cs->u_target = cd->u_target;
  cs->q_min = cd->q_min_threshold > 0.0f ? cd->q_min_threshold : 0.001f;
  cs->ramp_steps = cd->ramp_steps;
  cs->async_depth = cd->async_depth > 0 ? cd->async_depth : 8;
  cs->n_tri = cd->n_triangles;
  cs->force = cd->force;
  if (cd->n_triangles > 0) {
    std::vector<float> m((size_t)cd->n_triangles * 7);
    const float *src[7] = {cd->tri_cx, cd->tri_cy, cd->tri_cz, cd->tri_nx, cd->tri_ny, cd->tri_nz,
                           cd->tri_area};
    for (int a = 0; a < 7; ++a) {
      OL_CHECK_ARG(src[a], "case: triangle array %d is null", a);
      std::copy(src[a], src[a] + cd->n_triangles, m.begin() + (size_t)a * cd->n_triangles);
    }
    if ((rc = upload(&cs->mesh, m.data(), m.size()))) return rc;
    OL_CUDA(cudaMalloc(&cs->partials, (force_partial_rows(cd->n_triangles) * 9 + 16) * sizeof(double)));
  }
  cs->slot = c->free_slots.back();
  c->free_slots.pop_back();
  CaseDev cdv{};
  cdv.t = 0;
  cdv.u_target = cd->u_target;
  cdv.ramp_steps = cd->ramp_steps;
  cdv.async_depth = cs->async_depth;
  cdv.status = 0;
  OL_CUDA(cudaMemcpyAsync(c->d_cases + cs->slot, &cdv, sizeof(cdv), cudaMemcpyHostToDevice, c->stream));
  OL_CUDA(cudaStreamSynchronize(c->stream));
  cs->bytes = fp;
  cs->id = c->next_id++;
  c->used += fp;
  *case_id = cs->id;
  c->cases[cs->id] = std::move(cs);
  c->dirty = true;
  return OL_OK;
}

extern "C" int ol_ctx_case_remove(ol_ctx *c, int32_t id) {
  OL_CHECK_ARG(c, "ol_ctx_case_remove: null context");
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->cases.find(id);
  if (it == c->cases.end()) return set_error(OL_ERR_STATE, "ol_ctx_case_remove: unknown case %d", id);
  OL_CUDA(cudaStreamSynchronize(c->stream));
  NCase &cs = *it->second;
  for (auto &L : cs.levels) range_free(c, L.block_offset, L.n_blocks);
  free_case_meta(cs);
  c->free_slots.push_back(cs.slot);
  c->used -= cs.bytes;
  c->cases.erase(it);
  c->dirty = true;
  return OL_OK;
}

extern "C" int ol_ctx_step(ol_ctx *c, int32_t n) {
  OL_CHECK_ARG(c && n >= 0, "ol_ctx_step: bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  OL_CUDA(cudaSetDevice(c->device));
  if (c->dirty) {
    int rc = rebuild(c);
    if (rc) return rc;
  }
  if (!c->exec) return OL_OK;
  for (int i = 0; i < n; ++i) OL_CUDA(cudaGraphLaunch(c->exec, c->stream));
  c->launches += c->launches_per_step * n;
  for (auto &kv : c->cases) kv.second->steps += n;
  return OL_OK;
}

extern "C" int ol_ctx_case_step(ol_ctx *c, int32_t id, int32_t n, float u_in) {
  OL_CHECK_ARG(c && n >= 0, "ol_ctx_case_step: bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->cases.find(id);
  if (it == c->cases.end()) return set_error(OL_ERR_STATE, "ol_ctx_case_step: unknown case %d", id);
  OL_CUDA(cudaSetDevice(c->device));
  NCase &cs = *it->second;
  if (u_in >= 0.0f) {
    // a fixed inlet speed from now on: no ramp
    cs.u_target = u_in;
    cs.ramp_steps = 0;
    CaseDev *d = c->d_cases + cs.slot;
    const int32_t zero = 0;
    OL_CUDA(cudaMemcpyAsync(&d->u_target, &u_in, sizeof(float), cudaMemcpyHostToDevice, c->stream));
    OL_CUDA(cudaMemcpyAsync(&d->ramp_steps, &zero, sizeof(int32_t), cudaMemcpyHostToDevice,
                            c->stream));
    OL_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (n == 0) return OL_OK;
  // a plan (and graph) of this case alone, replayed n times; the next
  // ol_ctx_step rebuilds the plan of every resident case
  c->only_case = id;
  int rc = rebuild(c);
  if (rc == OL_OK && c->exec)
    for (int i = 0; i < n && rc == OL_OK; ++i) {
      const cudaError_t e = cudaGraphLaunch(c->exec, c->stream);
      if (e != cudaSuccess) rc = cuda_status(e, "cudaGraphLaunch");
    }
  c->only_case = -1;
  c->dirty = true;
  if (rc) return rc;
  c->launches += c->launches_per_step * n;
  cs.steps += n;
  return OL_OK;
}

extern "C" int ol_ctx_step_timed(ol_ctx *c, int32_t n, float *ms) {
  OL_CHECK_ARG(c && ms && n >= 0, "ol_ctx_step_timed: bad argument");
  {
    std::lock_guard<std::mutex> lk(c->mu);
    OL_CUDA(cudaSetDevice(c->device));
    if (c->dirty) {
      const int rc = rebuild(c);
      if (rc) return rc;
    }
  }
  cudaEvent_t e0, e1;
  OL_CUDA(cudaEventCreate(&e0));
  OL_CUDA(cudaEventCreate(&e1));
  OL_CUDA(cudaEventRecord(e0, c->stream));
  int rc = ol_ctx_step(c, n);
  if (rc == OL_OK) {
    OL_CUDA(cudaEventRecord(e1, c->stream));
    OL_CUDA(cudaEventSynchronize(e1));
    OL_CUDA(cudaEventElapsedTime(ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

extern "C" int ol_ctx_sync(ol_ctx *c) {
  OL_CHECK_ARG(c, "ol_ctx_sync: null context");
  OL_CUDA(cudaStreamSynchronize(c->stream));
  return OL_OK;
}

// Buffers holding the newest rho (written by the level's last sub-step) and
// the A half of vel (the reference's `level.vel`, surface.jl:788).
static void current_fields(ol_ctx *c, const NCase &cs, int lvl, float **rho, float **velA,
                           void **f) {
  const int64_t t = cs.steps;
  const int64_t last = t * ((int64_t)1 << lvl) + (((int64_t)1 << lvl) - 1);
  const bool even = (last & 1) == 0;
  *rho = t == 0 ? c->P.rhoA : (even ? c->P.rhoB : c->P.rhoA);
  *velA = c->P.velA;
  *f = t == 0 ? c->P.fA : (even ? c->P.fB : c->P.fA);
}

extern "C" int ol_ctx_case_forces(ol_ctx *c, int32_t id, double out[9]) {
  OL_CHECK_ARG(c && out, "ol_ctx_case_forces: null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->cases.find(id);
  if (it == c->cases.end()) return set_error(OL_ERR_STATE, "ol_ctx_case_forces: unknown case %d", id);
  NCase &cs = *it->second;
  for (int j = 0; j < 9; ++j) out[j] = 0.0;
  if (cs.n_tri == 0) return OL_OK;
  const int lvl = (int)cs.levels.size() - 1;
  const DevLevel &V = cs.levels[lvl];
  float *rho, *vel;
  void *f;
  current_fields(c, cs, lvl, &rho, &vel, &f);
  ForceDev D{};
  D.mesh.cx = cs.mesh; D.mesh.cy = cs.mesh + cs.n_tri; D.mesh.cz = cs.mesh + 2 * cs.n_tri;
  D.mesh.nx = cs.mesh + 3 * cs.n_tri; D.mesh.ny = cs.mesh + 4 * cs.n_tri;
  D.mesh.nz = cs.mesh + 5 * cs.n_tri; D.mesh.area = cs.mesh + 6 * cs.n_tri;
  D.mesh.n_triangles = cs.n_tri;
  D.rho = rho; D.vel = vel; D.obstacle = c->obst; D.bptr = V.bptr;
  D.block_offset = V.block_offset;
  D.dstride = c->capacity * BCELLS;
  D.fp = cs.force;
  D.fp.dim_x = V.dims[0]; D.fp.dim_y = V.dims[1]; D.fp.dim_z = V.dims[2];
  D.fp.tau_molecular = V.tau;
  D.partials = cs.partials;
  double *dev_out = cs.partials + force_partial_rows(cs.n_tri) * 9;
  launch_surface_forces(D, dev_out, c->stream);
  OL_LAUNCHED("ol_ctx_case_forces");
  OL_CUDA(cudaMemcpyAsync(out, dev_out, 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  OL_CUDA(cudaStreamSynchronize(c->stream));
  return OL_OK;
}

extern "C" int ol_ctx_case_coefficients(ol_ctx *c, int32_t id, const ol_coeff_ref *ref,
                                        double out[12]) {
  OL_CHECK_ARG(c && ref && out, "ol_ctx_case_coefficients: null argument");
  double raw[9];
  const int rc = ol_ctx_case_forces(c, id, raw);
  if (rc) return rc;
  coefficients_from_sums(raw, ref, out);
  return OL_OK;
}

extern "C" int ol_ctx_case_download(ol_ctx *c, int32_t id, int32_t level, float *rho, float *vel,
                                    float *f) {
  OL_CHECK_ARG(c, "ol_ctx_case_download: null context");
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->cases.find(id);
  if (it == c->cases.end()) return set_error(OL_ERR_STATE, "ol_ctx_case_download: unknown case %d", id);
  NCase &cs = *it->second;
  OL_CHECK_ARG(level >= 1 && level <= (int)cs.levels.size(), "ol_ctx_case_download: bad level");
  const DevLevel &V = cs.levels[level - 1];
  float *drho, *dvel;
  void *df;
  current_fields(c, cs, level - 1, &drho, &dvel, &df);
  OL_CUDA(cudaStreamSynchronize(c->stream));
  const size_t c0 = (size_t)V.block_offset * BCELLS, nc = (size_t)V.n_blocks * BCELLS;
  const size_t dstride = (size_t)c->capacity * BCELLS;
  if (rho) OL_CUDA(cudaMemcpy(rho, drho + c0, nc * 4, cudaMemcpyDeviceToHost));
  if (vel)
    for (int a = 0; a < 3; ++a)
      OL_CUDA(cudaMemcpy(vel + a * nc, dvel + c0 + a * dstride, nc * 4, cudaMemcpyDeviceToHost));
  if (f) {
    float *tmp = nullptr;
    OL_CUDA(cudaMalloc(&tmp, nc * 27 * 4));
    if (c->f16)
      k_decode_region<StoreF16S><<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(
          df, c0, nc, dstride, 1.0f / V.scale, tmp);
    else
      k_decode_region<StoreF32><<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(
          df, c0, nc, dstride, 1.0f, tmp);
    cudaError_t e = cudaMemcpyAsync(f, tmp, nc * 27 * 4, cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_status(e, "ol_ctx_case_download");
  }
  return OL_OK;
}

extern "C" int ol_ctx_case_download_thermal(ol_ctx *c, int32_t id, int32_t level, float *T,
                                            float *g) {
  OL_CHECK_ARG(c, "ol_ctx_case_download_thermal: null context");
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->cases.find(id);
  if (it == c->cases.end())
    return set_error(OL_ERR_STATE, "ol_ctx_case_download_thermal: unknown case %d", id);
  NCase &cs = *it->second;
  OL_CHECK_ARG(cs.ddf, "ol_ctx_case_download_thermal: case %d has no thermal DDF", id);
  OL_CHECK_ARG(level >= 1 && level <= (int)cs.levels.size(),
               "ol_ctx_case_download_thermal: bad level");
  const DevLevel &V = cs.levels[level - 1];
  // the last sub-step of the level wrote the same half of each A/B pair as rho and f
  const int64_t t = cs.steps;
  const int lv = level - 1;
  const int64_t last = t * ((int64_t)1 << lv) + (((int64_t)1 << lv) - 1);
  const bool even = (last & 1) == 0;
  float *dT = t == 0 ? c->P.TA : (even ? c->P.TB : c->P.TA);
  void *dg = t == 0 ? c->P.gA : (even ? c->P.gB : c->P.gA);
  OL_CUDA(cudaStreamSynchronize(c->stream));
  const size_t c0 = (size_t)V.block_offset * BCELLS, nc = (size_t)V.n_blocks * BCELLS;
  const size_t dstride = (size_t)c->capacity * BCELLS;
  if (T) OL_CUDA(cudaMemcpy(T, dT + c0, nc * 4, cudaMemcpyDeviceToHost));
  if (g) {
    float *tmp = nullptr;
    OL_CUDA(cudaMalloc(&tmp, nc * 27 * 4));
    if (c->f16)
      k_decode_region<StoreF16S><<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(
          dg, c0, nc, dstride, 1.0f / V.scale, tmp);
    else
      k_decode_region<StoreF32><<<(unsigned)((nc + 255) / 256), 256, 0, c->stream>>>(
          dg, c0, nc, dstride, 1.0f, tmp);
    cudaError_t e = cudaMemcpyAsync(g, tmp, nc * 27 * 4, cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_status(e, "ol_ctx_case_download_thermal");
  }
  return OL_OK;
}

extern "C" int ol_ctx_case_info(ol_ctx *c, int32_t id, int64_t *steps, int32_t *status) {
  OL_CHECK_ARG(c, "ol_ctx_case_info: null context");
  std::lock_guard<std::mutex> lk(c->mu);
  auto it = c->cases.find(id);
  if (it == c->cases.end()) return set_error(OL_ERR_STATE, "ol_ctx_case_info: unknown case %d", id);
  CaseDev cdv{};
  OL_CUDA(cudaMemcpyAsync(&cdv, c->d_cases + it->second->slot, sizeof(cdv), cudaMemcpyDeviceToHost,
                          c->stream));
  OL_CUDA(cudaStreamSynchronize(c->stream));
  if (steps) *steps = cdv.t;
  if (status) *status = cdv.status;
  return OL_OK;
}

extern "C" int ol_ctx_set_launch(ol_ctx *c, int32_t shape) {
  OL_CHECK_ARG(c, "ol_ctx_set_launch: null context");
  OL_CHECK_ARG(shape >= OL_LAUNCH_WS && shape <= 2, "ol_ctx_set_launch: unknown shape %d", shape);
  std::lock_guard<std::mutex> lk(c->mu);
  c->grid_mult = shape;
  for (auto &a : c->variant_shape)
    for (auto &b : a)
      for (auto &v : b) v = kShapeDefault;
  c->dirty = true;
  return OL_OK;
}

extern "C" int ol_ctx_get_launch(ol_ctx *c, int32_t *shape) {
  OL_CHECK_ARG(c && shape, "ol_ctx_get_launch: null argument");
  *shape = c->grid_mult;
  return OL_OK;
}

extern "C" int ol_ctx_get_variant_launch(ol_ctx *c, int32_t op, int32_t wale, int32_t ddf,
                                         int32_t *shape) {
  OL_CHECK_ARG(c && shape, "ol_ctx_get_variant_launch: null argument");
  OL_CHECK_ARG(op == OL_OP_CUMULANT || op == OL_OP_REGULARIZED_BGK,
               "ol_ctx_get_variant_launch: unknown operator %d", op);
  const int s = c->variant_shape[op][wale ? 1 : 0][ddf ? 1 : 0];
  *shape = s == kShapeDefault ? c->grid_mult : s;
  return OL_OK;
}

// Time `trials` coarse steps of the resident mix after one untimed step that
// rebuilds the plan and graph under the shapes just set.
static int time_mix(ol_ctx *c, int32_t trials, cudaEvent_t e0, cudaEvent_t e1, float *ms) {
  int rc = ol_ctx_step(c, 1);
  if (rc) return rc;
  OL_CUDA(cudaEventRecord(e0, c->stream));
  rc = ol_ctx_step(c, trials);
  if (rc) return rc;
  OL_CUDA(cudaEventRecord(e1, c->stream));
  OL_CUDA(cudaEventSynchronize(e1));
  OL_CUDA(cudaEventElapsedTime(ms, e0, e1));
  return OL_OK;
}

extern "C" int ol_ctx_autotune(ol_ctx *c, int32_t trials) {
  OL_CHECK_ARG(c && trials > 0, "ol_ctx_autotune: bad argument");
  const int cands[5] = {OL_LAUNCH_WS, OL_LAUNCH_PER_ITEM, 1, 2, OL_LAUNCH_PIPELINED};
  cudaEvent_t e0, e1;
  OL_CUDA(cudaEventCreate(&e0));
  OL_CUDA(cudaEventCreate(&e1));
  auto set = [&](auto &&apply) {
    std::lock_guard<std::mutex> lk(c->mu);
    apply();
    c->dirty = true;
  };
  auto reset_variants = [&]() {
    for (auto &x : c->variant_shape)
      for (auto &y : x)
        for (auto &v : y) v = kShapeDefault;
  };
  // one shape for the whole mix
  float best_ms = 1e30f;
  int best = c->grid_mult;
  int rc = OL_OK;
  for (int ci = 0; ci < 5 && !rc; ++ci) {
    set([&] { c->grid_mult = cands[ci]; reset_variants(); });
    float ms = 0.f;
    rc = time_mix(c, trials, e0, e1, &ms);
    if (!rc && ms < best_ms) { best_ms = ms; best = cands[ci]; }
  }
  if (!rc) set([&] { c->grid_mult = best; reset_variants(); });
  // then, when the mix holds more than one collision variant, each variant's
  // own shape with the others held (their time is the same in every trial)
  std::vector<std::array<int, 3>> keys;
  if (!rc) {
    std::lock_guard<std::mutex> lk(c->mu);
    for (const Launch &l : c->plan)
      if (l.kind == 0) {
        const std::array<int, 3> k{l.op & 1, l.wale ? 1 : 0, l.ddf ? 1 : 0};
        if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
      }
  }
  if (keys.size() > 1) {
    for (const auto &k : keys) {
      int &slot = c->variant_shape[k[0]][k[1]][k[2]];
      float kbest_ms = 1e30f;
      int kbest = best;
      for (int ci = 0; ci < 5 && !rc; ++ci) {
        set([&] { slot = cands[ci]; });
        float ms = 0.f;
        rc = time_mix(c, trials, e0, e1, &ms);
        if (!rc && ms < kbest_ms) { kbest_ms = ms; kbest = cands[ci]; }
      }
      if (rc) break;
      set([&] { slot = kbest; });
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

extern "C" int ol_ctx_stats(ol_ctx *c, size_t *used, size_t *budget, int32_t *n_cases,
                            int64_t *launches) {
  OL_CHECK_ARG(c, "ol_ctx_stats: null context");
  if (used) *used = c->used;
  if (budget) *budget = c->budget;
  if (n_cases) *n_cases = (int32_t)c->cases.size();
  if (launches) *launches = c->launches;
  return OL_OK;
}
