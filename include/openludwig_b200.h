/*
 * openludwig_b200.h -- C ABI of the B200 (sm_100a) lattice Boltzmann time step.
 *
 * Every entry point is plain C: raw pointers, sizes and POD structs, an int
 * status (0 = OL_OK) and a thread-local message from ol_last_error().  No
 * C++ types or exceptions cross this boundary and the library never frees
 * memory it did not allocate.
 *
 * Drop-in layer (ol_stream_collide, ol_bouzidi, ol_thermal, ol_surface_forces,
 * ol_init_equilibrium, ol_flow_stats): all pointers are DEVICE pointers to
 * buffers laid out exactly like the reference's Julia column-major CuArrays,
 * so `pointer(::CuArray)` can be handed over unchanged:
 *     f[x,y,z,b,k]  -> (x-1) + 8(y-1) + 64(z-1) + 512(b-1) + 512*nB*(k-1)
 *     vel[x,y,z,b,c]-> same with c in 1..3;  rho/obstacle/sponge/wall_dist[x,y,z,b]
 *     neighbor_table[b,dir] -> (b-1) + nB*(dir-1), dir=(dx+1)+3(dy+1)+9(dz+1)+1
 *     block_pointer[bx,by,bz] -> dense Int32 grid, bx fastest
 * Index VALUES stored inside those arrays keep the reference's 1-based
 * convention (block ids 1..nB, 0 = missing; Bouzidi cell x/y/z in 1..8).
 * The block edge is fixed at 8 cells (blocks.jl BLOCK_SIZE).
 *
 * Native layer (ol_ctx_*): the library owns a device block pool with FP32 or
 * FP16-shifted population storage and advances many cases of uneven size
 * together with persistent kernels replayed from a CUDA graph; ol_server_* /
 * ol_serve_* run the continuous-batching request loop over it (driven from
 * Python by openludwig_b200.serving, or from any caller of the C ABI).
 */
#ifndef OPENLUDWIG_B200_H
#define OPENLUDWIG_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OL_API __attribute__((visibility("default")))
#else
#define OL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define OL_OK 0
#define OL_ERR_ARG 1        /* bad argument (null pointer, size, enum)        */
#define OL_ERR_CUDA 2       /* a CUDA runtime call failed                      */
#define OL_ERR_NOMEM 3      /* allocation or HBM budget exceeded               */
#define OL_ERR_STATE 4      /* call out of order / unknown handle              */
#define OL_ERR_NUMERIC 5    /* device watchdog: NaN or rho below threshold     */

/* collision operators (physics_kernels.jl:35-45) */
#define OL_OP_CUMULANT 0
#define OL_OP_REGULARIZED_BGK 1
/* cumulant limiter (timestep.jl:46-47) */
#define OL_LIMITER_NONE 0
#define OL_LIMITER_FACTORED 1
#define OL_LIMITER_POSITIVITY 2

/* ------------------------------------------------------------------ */
/* Drop-in layer                                                        */
/* ------------------------------------------------------------------ */

/* One refinement level's device buffers (the BlockLevel fields the flow
 * kernel reads and writes, blocks.jl:138-196). */
typedef struct ol_level_view {
  float *f_out;                 /* [512*nB*27] written                        */
  const float *f_in;            /* [512*nB*27] read (pull source)             */
  float *f_post;                /* [512*nB*27] post-collision copy, or NULL    */
  float *rho;                   /* [512*nB]    written                         */
  float *vel_out;               /* [512*nB*3]  written                         */
  const float *vel_in;          /* [512*nB*3]  read (WALE gradients)           */
  const uint8_t *obstacle;      /* [512*nB]    Julia Bool                      */
  const float *sponge;          /* [512*nB]                                    */
  const float *wall_dist;       /* [512*nB]    may be NULL if no wall model    */
  const int32_t *neighbor_table;/* [nB*27]     1-based ids, 0 = missing        */
  const int32_t *map_x, *map_y, *map_z; /* [nB] 1-based block coordinates     */
  float *ghost;                 /* [ol_ghost_floats(nB)] scratch, or NULL (below) */
  int32_t n_blocks;
  /* Optional pairing of the two sub-steps a fine level takes per parent step
   * (temporal weights 0 and 1/2, solver_control.jl:65-97), with ghost set:
   * OL_GHOST_PAIR_FIRST on the weight-0 call also writes into ghost_next (a
   * second [ol_ghost_floats(nB)] scratch) the coarse-to-fine values of the
   * weight-1/2 call, reading each parent value once for both;
   * OL_GHOST_PAIR_SECOND on the weight-1/2 call, with ghost = that
   * ghost_next and the parent state unchanged since, evaluates only the
   * domain-boundary values.  OL_GHOST_UNPAIRED (0) computes every value in
   * every call.  Results are identical in all three modes. */
  float *ghost_next;
  int32_t ghost_mode;
  /* Optional [n_ghost_blocks] 0-based ids of the blocks the ghost pass visits
   * (NULL = every block; the pass skips blocks without an absent neighbour;
   * a non-NULL list with n_ghost_blocks = 0 launches no pass).  A list must
   * hold every block with an absent neighbour, or under OL_GHOST_PAIR_SECOND
   * every block with an absent neighbour not wholly inside the level's
   * domain; it saves the launch of the other blocks.  The pass visits the
   * list in order: listing blocks by their number of absent-neighbour
   * pulls, largest first (484 per absent face neighbour, 22 per edge, 1 per
   * corner), keeps the slowest blocks out of its last wave. */
  const int32_t *ghost_blocks;
  int32_t n_ghost_blocks;
} ol_level_view;

#define OL_GHOST_UNPAIRED 0
#define OL_GHOST_PAIR_FIRST 1
#define OL_GHOST_PAIR_SECOND 2

/* Size (floats) of the optional ol_level_view.ghost scratch.  No reference
 * counterpart: with ghost set, ol_stream_collide first evaluates, in a
 * separate pass over the blocks that have an absent neighbour, the boundary
 * values those pulls read (inlet/outlet equilibria, free-slip mirrors,
 * coarse-to-fine interpolation; kernel_cumulant.jl:117-159), then streams
 * them like neighbour data.  With ghost NULL the same values are computed
 * while the block is staged.  Results are identical either way. */
OL_API int64_t ol_ghost_floats(int32_t n_blocks);

/* Parent-level state for coarse-to-fine ghost interpolation
 * (physics_interpolation.jl:4-127).  Ignored when is_level_1 != 0. */
typedef struct ol_parent_view {
  const float *f, *rho, *vel;           /* parent state after its step        */
  const float *f_old, *rho_old, *vel_old; /* parent state before its step     */
  const int32_t *block_ptr;             /* [dim_x*dim_y*dim_z] 1-based ids    */
  int32_t dim_x, dim_y, dim_z;          /* size(block_ptr)                    */
  int32_t n_blocks;                     /* parent nB (array stride)           */
} ol_parent_view;

/* Every scalar argument of stream_collide_cumulant! (kernel_cumulant.jl:38-68);
 * the regularized-BGK kernel takes the same list (kernel_regularized_bgk.jl:13-41). */
typedef struct ol_step_params {
  int32_t op;                   /* OL_OP_*                                    */
  float tau_molecular, tau_parent, c_wale, nu_sgs_background;
  int32_t is_level_1, is_symmetric;
  int32_t nx_global, ny_global, nz_global;
  float u_inlet;
  int32_t wall_model_active, time_step_seed, store_post_collision;
  float inlet_turbulence, temporal_weight;
  int32_t use_temporal_interp, sponge_blend_distributions;
  float omega_bulk, omega_3, omega_4;
  int32_t adaptive_omega4;
  float lambda_param;
  int32_t limiter_type, compressible_corr;
} ol_step_params;

/* Fused pull-stream + collision of one level sub-step: one launch, grid of
 * one CTA per 8^3 block.  Replaces the kernel launch in perform_timestep_v2!
 * (timestep.jl:51-88, kernel_cumulant.jl:29-627 / kernel_regularized_bgk.jl:4-325).
 * `stream` is a cudaStream_t (NULL = legacy default stream). */
OL_API int ol_stream_collide(const ol_level_view *lv, const ol_parent_view *pv,
                      const ol_step_params *sp, void *stream);

/* Which kernel ol_stream_collide (and the block pool's stream-collide
 * launches) run; no reference counterpart (the reference has one kernel
 * launch shape).  OL_SC_KERNEL_BLOCK: one CTA per 8^3 block, synchronous
 * staging.  OL_SC_KERNEL_WS: one persistent CTA per SM whose producer warp
 * bulk-copies the next block while its consumer warps collide the current
 * one (cumulant operator, levels whose absent-neighbour values are ghost rows
 * or level-1 domain boundaries; other launches keep the per-block kernel).
 * The same choice applies to ol_thermal (FP32 thermal populations, two
 * blocks in flight per SM).
 * OL_SC_KERNEL_AUTO (default): OL_SC_KERNEL_WS for FP32 populations where
 * it applies and the level has at least two blocks per SM.  Both kernels
 * stage the same values and run the same cell-update code: rho and u agree
 * bit for bit; a few post-collision populations may differ in the last bit
 * (the compiler may fuse a multiply and an add differently in each).
 * max_ctas > 0 caps the persistent grid (each CTA then walks more blocks;
 * for tests of the stage hand-over), 0 = one CTA per SM.  Process-wide. */
#define OL_SC_KERNEL_AUTO 0
#define OL_SC_KERNEL_BLOCK 1
#define OL_SC_KERNEL_WS 2
OL_API int ol_set_stream_collide_kernel(int32_t choice, int32_t max_ctas);

/* Reads and clears the fault bits of the current device's warp-specialised
 * kernels: 1 = a consumer warp's wait for a staged block ran out, 2 = a
 * loader warp's wait for a free stage ran out (each wait is bounded at 2 s;
 * the kernel then ends early and its output is incomplete).  0 = none. */
OL_API int ol_pipeline_fault(int32_t *flags);

/* Host copies of the static staging tables (no GPU needed; for checking the
 * kernels' index arithmetic): the staging table of the one-CTA-per-block
 * kernel and the ghost pass, and the loader table of the warp-specialised
 * kernel (out-of-block pulls k | dir << 5 | source cell << 10 | pulling cell
 * << 19, face-halo velocity slots, then the FP32 stage slot of each pull).
 * sizes[4] = {halo entries, loader entries, stage plane slots, stage pad}; a
 * table is copied when its buffer is non-NULL and large enough. */
OL_API int ol_staging_tables(uint32_t *halo, int32_t halo_cap, uint32_t *ws, int32_t ws_cap,
                             int32_t *sizes);

/* Bouzidi interpolated bounce-back (bouzidi_kernel.jl:13-122).  q_map holds
 * IEEE binary16 bit patterns [512*nB*27]; cell_* are the sparse boundary-cell
 * lists (block 1-based Int32, x/y/z 1-based Int8).  Reads f_post, writes f_out. */
OL_API int ol_bouzidi(float *f_out, const float *f_post, const uint16_t *q_map,
               const int32_t *cell_block, const int8_t *cell_x,
               const int8_t *cell_y, const int8_t *cell_z, int32_t n_boundary,
               const int32_t *neighbor_table, int32_t n_blocks,
               float q_min_threshold, void *stream);

/* Same result as ol_bouzidi without a dense post-collision copy: f_out still
 * holds the post-collision values when it is called (the flow kernel ran with
 * store_post_collision = 0).  Phase 1 gathers every corrected link into
 * `scratch` (>= 27*n_boundary floats, caller-owned device memory), phase 2
 * scatters them, so no link reads a value another link already replaced.
 * Replaces the f_post_collision round trip of timestep.jl:71 + :90-98. */
OL_API int ol_bouzidi_sparse(float *f_out, const uint16_t *q_map,
                      const int32_t *cell_block, const int8_t *cell_x,
                      const int8_t *cell_y, const int8_t *cell_z,
                      int32_t n_boundary, const int32_t *neighbor_table,
                      int32_t n_blocks, float q_min_threshold, float *scratch,
                      void *stream);

/* A boundary link of the Bouzidi correction: level-local cell index
 * (b*512 + x + 8y + 64z, 0-based), q, direction k, and the cell x - c_k that
 * q < 1/2 reads (-1: absent neighbour block, or q >= 1/2). */
typedef struct ol_bouzidi_link {
  int32_t cell;
  int32_t far_cell;
  float q;
  int32_t k;
} ol_bouzidi_link;

/* Compacts the links of a level with q in (q_min, 1] (static for a level:
 * build once) into `links` (capacity 27 * n_boundary) and their number into
 * the device int *n_links_dev; arguments as ol_bouzidi_sparse.  No
 * reference counterpart: ol_bouzidi_apply_links then corrects only those
 * links each step instead of visiting all 27 directions of every boundary
 * cell. */
OL_API int ol_bouzidi_build_links(const uint16_t *q_map, const int32_t *cell_block,
                           const int8_t *cell_x, const int8_t *cell_y,
                           const int8_t *cell_z, int32_t n_boundary,
                           const int32_t *neighbor_table, int32_t n_blocks,
                           float q_min_threshold, ol_bouzidi_link *links,
                           int32_t *n_links_dev, void *stream);
/* The correction of ol_bouzidi_sparse (bouzidi_kernel.jl:13-92) over a link
 * list: every corrected value gathered into scratch (n_links floats), then
 * scattered.  The same values, bit for bit. */
OL_API int ol_bouzidi_apply_links(float *f_out, const ol_bouzidi_link *links, int32_t n_links,
                           int32_t n_blocks, float *scratch, void *stream);

/* Same correction as ol_bouzidi_sparse for callers that cannot allocate
 * device memory: callers whose memory is held by another allocator's pool
 * (CUDA.jl, PyTorch caching allocators) or loops that must not allocate.
 * No counterpart in the reference (it always allocates f_post_collision).
 * The scratch is a fixed library-owned device array sized for
 * OL_BOUZIDI_NOALLOC_MAX_CELLS boundary cells (27 floats each, 7 MB, held by
 * every device that loads the library until exit); larger n_boundary is
 * rejected with OL_ERR_ARG.  The call allocates nothing.  Its first call on
 * a device looks up the array's device address (once per device and CUDA
 * context, that device current; after a device reset or under another
 * context the next call looks it up again); make that first call before any
 * stream capture.  All calls share the one array: calls that overlap on the
 * GPU (other streams, other host threads) race on it. */
#define OL_BOUZIDI_NOALLOC_MAX_CELLS 65536
OL_API int ol_bouzidi_sparse_noalloc(float *f_out, const uint16_t *q_map,
                      const int32_t *cell_block, const int8_t *cell_x,
                      const int8_t *cell_y, const int8_t *cell_z,
                      int32_t n_boundary, const int32_t *neighbor_table,
                      int32_t n_blocks, float q_min_threshold, void *stream);

/* Thermal DDF level view + parameters (kernel_thermal.jl:14-40). */
typedef struct ol_thermal_view {
  float *g_out; const float *g_in; float *g_post;  /* g_post may be NULL     */
  float *temperature;            /* [512*nB] written                          */
  const float *vel;              /* flow kernel's vel_out of this sub-step    */
  const uint8_t *obstacle; const float *sponge;
  const int32_t *neighbor_table; const int32_t *map_x, *map_y, *map_z;
  int32_t n_blocks;
  /* parent (coarse-to-fine, physics_interpolation.jl:135-247) */
  const float *pg, *pT, *pvel, *pg_old, *pT_old, *pvel_old;
  const int32_t *p_block_ptr; int32_t p_dim_x, p_dim_y, p_dim_z, p_n_blocks;
  /* optional [ol_ghost_floats(nB)] scratch, as ol_level_view.ghost: the
   * boundary values of absent neighbours by a separate pass (same results) */
  float *ghost;
  float *ghost_next;             /* as ol_level_view.ghost_next / ghost_mode */
  int32_t ghost_mode;
  const int32_t *ghost_blocks;   /* as ol_level_view.ghost_blocks            */
  int32_t n_ghost_blocks;
} ol_thermal_view;

typedef struct ol_thermal_params {
  float tau_g, tau_g_parent;
  int32_t is_level_1, is_symmetric, nx_global, ny_global, nz_global;
  float u_inlet, T_inlet, T_wall;
  int32_t wall_bc_adiabatic, store_post_collision;
  float temporal_weight;
  int32_t use_temporal_interp, sponge_blend_distributions;
} ol_thermal_params;

/* Thermal DDF stream-collide (kernel_thermal.jl:14-202). */
OL_API int ol_thermal(const ol_thermal_view *tv, const ol_thermal_params *tp,
               void *stream);

/* Initial state of a level (main.jl:113-150): f = f_temp = w_k, and when
 * f_old != NULL also f_old = w_k, rho_old = 1, vel_old = 0. */
OL_API int ol_init_equilibrium(float *f, float *f_temp, float *f_old, float *rho_old,
                        float *vel_old, int32_t n_blocks, void *stream);

/* Surface mesh on the device (geometry.jl:24-33 GPUMesh). */
typedef struct ol_surface_mesh {
  const float *cx, *cy, *cz;     /* triangle centres (unrotated domain frame) */
  const float *nx, *ny, *nz;     /* unit normals                              */
  const float *area;
  int32_t n_triangles;
} ol_surface_mesh;

typedef struct ol_force_params {
  float dx;                              /* Float32(level.dx)                  */
  int32_t dim_x, dim_y, dim_z;           /* level grid_dim (size(block_ptr))   */
  float offset_x, offset_y, offset_z;    /* mesh_offset                        */
  float pressure_scale, stress_scale;    /* rho_phys * U_vs^2                  */
  float tau_molecular;
  int32_t search_radius;
  float c_wale, nu_sgs_bg;
  float ref_x, ref_y, ref_z;             /* moment centre                      */
} ol_force_params;

/* map_stresses_kernel! + integrate_forces_kernel! (surface.jl:350-507,
 * 702-762).  Writes the per-triangle maps (p, tau_x, tau_y, tau_z, device
 * arrays of n_triangles) and out[9] = {Fx_p, Fy_p, Fz_p, Fx_v, Fy_v, Fz_v,
 * Mx, My, Mz} summed in FP64 in a fixed order (deterministic; the
 * reference's FP32 atomics are not).  `partials` is caller device scratch of
 * >= ol_surface_forces_scratch_doubles(n_triangles) doubles. */
OL_API int ol_surface_forces(const ol_surface_mesh *mesh, const float *rho,
                      const float *vel, const uint8_t *obstacle,
                      const int32_t *block_ptr, int32_t n_blocks,
                      const ol_force_params *fp, float *p_map, float *sx_map,
                      float *sy_map, float *sz_map, double *partials,
                      double out[9], void *stream);
OL_API size_t ol_surface_forces_scratch_doubles(int32_t n_triangles);

/* Outputs of ol_surface_net_forces: device arrays of n_triangles floats.
 * The plus maps are force_data.pressure_map / shear_{x,y,z}_map, the minus
 * maps force_data.*_map_minus; each side's four are all given or all NULL. */
typedef struct ol_net_force_maps {
  float *p_plus, *sx_plus, *sy_plus, *sz_plus;
  float *p_minus, *sx_minus, *sy_minus, *sz_minus;
  float *net_fx, *net_fy, *net_fz;       /* per-triangle net force, required */
} ol_net_force_maps;

/* Two-sided per-triangle net force, replaces compute_net_aerodynamics!
 * (surface.jl:980-1034) with its kernels map_stresses_kernel! (:350-507),
 * map_minus_side_only_kernel! (:511-662) and
 * compute_net_triangle_forces_kernel! (:665-700):
 * net = -(p+ - p-) n A + (tau+ - tau-) A.  closed_body != 0 zeroes the minus
 * side without probing it (the reference's default).  One launch on `stream`,
 * asynchronous; results stay on the device. */
OL_API int ol_surface_net_forces(const ol_surface_mesh *mesh, const float *rho,
                          const float *vel, const uint8_t *obstacle,
                          const int32_t *block_ptr, int32_t n_blocks,
                          const ol_force_params *fp, int32_t closed_body,
                          const ol_net_force_maps *out, void *stream);

/* One level's part of the merged flow output (io_vtk.jl:6-129). */
typedef struct ol_output_level {
  const float *rho;                     /* [512*nB]                               */
  const float *vel;                     /* [512*nB*3]: vel or vel_temp, as the
                                           reference picks by step parity (io_vtk.jl:48) */
  const uint8_t *obstacle;              /* [512*nB]                               */
  const float *temperature;             /* [512*nB], or NULL without the DDF      */
  const int32_t *map_x, *map_y, *map_z; /* [nB] 1-based block coordinates         */
  const int32_t *blocks;                /* [n_export] 0-based ids (< nB) of the
                                           exported blocks, in export order        */
  int32_t n_export;
  int32_t n_blocks;                     /* level nB (array stride)                */
  int32_t level_id;                     /* 1-based, written to the level field    */
  float dx;                             /* Float32(level.dx)                      */
} ol_output_level;

/* Packed output arrays (device memory), N = total exported blocks; any may
 * be NULL to skip it.  Cell order is the block's own (x fastest), blocks
 * level after level in list order, as the reference's VTK writer lays them. */
typedef struct ol_output_fields {
  float *points;       /* [3 * 729 * N] x, y, z of the 9^3 corner points per block */
  float *rho;          /* [512 * N]                                             */
  float *vel;          /* [3 * 512 * N] ux, uy, uz per cell                     */
  float *vel_mag;      /* [512 * N]                                             */
  uint8_t *obstacle;   /* [512 * N] 0 / 1                                        */
  int32_t *level;      /* [512 * N] level id                                     */
  float *temperature;  /* [512 * N] (0 on levels without temperature)           */
} ol_output_fields;

/* Device part of export_merged_mesh_sync (io_vtk.jl:6-129): gathers the
 * exported blocks of up to 16 levels into the packed arrays, NaN / +-Inf
 * replaced by 0 (io_vtk.jl:111-115), velocity magnitude in Float32.  One
 * launch on `stream`, asynchronous; the caller copies the arrays back and
 * writes the file. */
OL_API int ol_pack_merged_fields(const ol_output_level *levels, int32_t n_levels,
                          const ol_output_fields *out, void *stream);

/* Flow statistics of a level in FP64 (diagnostics.jl:43-93):
 * out[0..6] = {n_fluid, rho_sum, rho_min, rho_max, v_max, kinetic_energy,
 * mass_all_cells}.  `partials` >= ol_flow_stats_scratch_doubles(nB). */
OL_API int ol_flow_stats(const float *rho, const float *vel, const uint8_t *obstacle,
                  int32_t n_blocks, double *partials, double out[7],
                  void *stream);
OL_API size_t ol_flow_stats_scratch_doubles(int32_t n_blocks);
/* The same statistics into out7_dev (7 doubles of device memory), enqueued
 * on `stream` without waiting: for a driver that reads them back
 * asynchronously (a copy to pinned memory it checks a step later). */
OL_API int ol_flow_stats_device(const float *rho, const float *vel, const uint8_t *obstacle,
                         int32_t n_blocks, double *partials, double *out7_dev,
                         void *stream);

/* ------------------------------------------------------------------ */
/* Native layer: device block pool, FP16-shifted storage, batched       */
/* multi-case stepping with persistent kernels and CUDA graphs.         */
/* ------------------------------------------------------------------ */

#define OL_STORE_F32 0
#define OL_STORE_F16 1   /* f stored as binary16 of (f_k - w_k) * scale / w_k */
#define OL_STORE_DDF 2   /* flag: the pool also holds thermal populations     */

typedef struct ol_ctx ol_ctx;

/* Host description of one refinement level of one case.  Arrays are HOST
 * memory in the drop-in layout above; the library copies them. */
typedef struct ol_level_desc {
  int32_t n_blocks;
  const int32_t *map_x, *map_y, *map_z;     /* [nB] 1-based                   */
  const int32_t *neighbor_table;            /* [nB*27]                         */
  const int32_t *block_ptr;                 /* [dim_x*dim_y*dim_z]             */
  int32_t dim_x, dim_y, dim_z;
  const uint8_t *obstacle;                  /* [512*nB]                        */
  const float *sponge;                      /* [512*nB]                        */
  const float *wall_dist;                   /* [512*nB] or NULL                */
  /* Bouzidi (dense q-map of binary16 bits + sparse cell list) or n_boundary=0 */
  int32_t n_boundary;
  const uint16_t *q_map;                    /* [512*nB*27]                     */
  const int32_t *cell_block; const int8_t *cell_x, *cell_y, *cell_z;
  float tau;                                /* tau of this level               */
  float tau_g;                              /* thermal tau (DDF cases)         */
  float store_scale;                        /* FP16 shift scale of this level  */
} ol_level_desc;

typedef struct ol_case_desc {
  int32_t n_levels;
  const ol_level_desc *levels;              /* [n_levels], coarsest first      */
  int32_t nx, ny, nz;                       /* coarse domain size in cells     */
  ol_step_params params;                    /* shared scalars (tau fields unused) */
  int32_t ddf;                              /* thermal DDF on                  */
  ol_thermal_params tparams;                /* thermal scalars (taus unused)   */
  /* surface mesh (host arrays, n_triangles entries) for Cd/Cl */
  int32_t n_triangles;
  const float *tri_cx, *tri_cy, *tri_cz, *tri_nx, *tri_ny, *tri_nz, *tri_area;
  ol_force_params force;                    /* finest-level force parameters   */
  float u_target;                           /* lattice inlet speed after ramp  */
  int32_t ramp_steps;                       /* cosine ramp (main.jl:217)       */
  int32_t async_depth;                      /* ramp batching (main.jl:210-218) */
  float q_min_threshold;                    /* Bouzidi q threshold             */
  float T_initial;                          /* initial temperature (DDF)       */
} ol_case_desc;

/* store_kind = OL_STORE_F32 or OL_STORE_F16, optionally | OL_STORE_DDF.
 * The block pool (hbm_budget_bytes * 15/16) is allocated here, once. */
OL_API int ol_ctx_create(ol_ctx **out, int device, size_t hbm_budget_bytes,
                  int store_kind);
OL_API int ol_ctx_destroy(ol_ctx *ctx);
/* bytes of device memory a case would take in this context */
OL_API int ol_ctx_case_footprint(ol_ctx *ctx, const ol_case_desc *cd, size_t *bytes);
OL_API int ol_ctx_case_add(ol_ctx *ctx, const ol_case_desc *cd, int32_t *case_id);
OL_API int ol_ctx_case_remove(ol_ctx *ctx, int32_t case_id);
/* Advance every resident case by n_coarse coarse steps (one graph replay
 * per coarse step).  Asynchronous on the context stream. */
OL_API int ol_ctx_step(ol_ctx *ctx, int32_t n_coarse);
OL_API int ol_ctx_sync(ol_ctx *ctx);
/* ol_ctx_step followed by a synchronize, timed with CUDA events recorded on
 * the context stream around the replays; *ms = device time of the n steps. */
OL_API int ol_ctx_step_timed(ol_ctx *ctx, int32_t n_coarse, float *ms);
/* Surface forces of one case on its finest level: out[9] as ol_surface_forces. */
OL_API int ol_ctx_case_forces(ol_ctx *ctx, int32_t case_id, double out[9]);

/* Reference values of the force coefficients (surface.jl:873-910): free-
 * stream density and speed, reference area and chord (physical units, as
 * the force sums), and whether the case is a half model (symmetric). */
typedef struct ol_coeff_ref {
  double rho_ref, u_ref, area_ref, chord_ref;
  int32_t symmetric;
} ol_coeff_ref;

/* The coefficient record of one case (compute_aerodynamics!, surface.jl:
 * 913-920, with the finishing of integrate_surface_forces!, :873-910):
 * out[12] = {Cd, Cl, Cs, Cmx, Cmy, Cmz, Fx, Fy, Fz, Mx, My, Mz} -- Cd along
 * x, Cl along z, Cs along y; forces are pressure + viscous, moments about
 * the moment centre, after symmetry doubling of a half model. */
OL_API int ol_ctx_case_coefficients(ol_ctx *ctx, int32_t case_id, const ol_coeff_ref *ref,
                                    double out[12]);

/* Advance ONE resident case by n_coarse coarse steps (the per-case
 * counterpart of ol_ctx_step; the reference steps its single case with
 * execute_timestep_batch!, solver_control.jl:199-218).  u_in >= 0 fixes
 * the case's inlet speed (lattice units) from now on, replacing its ramp;
 * u_in < 0 keeps the case's target and ramp.  The other resident cases do
 * not move.  It replays a graph of this case alone, so the next ol_ctx_step
 * rebuilds the graph of all cases. */
OL_API int ol_ctx_case_step(ol_ctx *ctx, int32_t case_id, int32_t n_coarse, float u_in);
/* Download a level's macroscopic fields (host buffers of 512*nB / 512*nB*3),
 * populations (host [512*nB*27] FP32, decoded), or NULL to skip. */
OL_API int ol_ctx_case_download(ol_ctx *ctx, int32_t case_id, int32_t level,
                         float *rho, float *vel, float *f);
/* The same for the thermal DDF of a DDF case: temperature [512*nB] and g
 * [27][512*nB] (decoded to FP32), either may be NULL. */
OL_API int ol_ctx_case_download_thermal(ol_ctx *ctx, int32_t case_id, int32_t level,
                                 float *temperature, float *g);
/* Coarse steps a case has done, and its device watchdog status. */
OL_API int ol_ctx_case_info(ol_ctx *ctx, int32_t case_id, int64_t *coarse_steps,
                     int32_t *status);
/* Launch shape of the context's stream-collide launches (no reference
 * counterpart):
 *   OL_LAUNCH_WS         warp-specialised persistent kernel, one CTA per SM
 *                        (FP32 cumulant launches without DDF; the other
 *                        variants take one CTA per work item) -- default;
 *   OL_LAUNCH_PIPELINED  software-pipelined persistent kernel (FP32 without
 *                        DDF), two CTAs per SM;
 *   OL_LAUNCH_PER_ITEM   one CTA per (case, level, block) work item;
 *   1, 2                 persistent grid of 1x / 2x the resident CTAs.
 * Every shape runs the same cell update on the same staged values. */
#define OL_LAUNCH_WS (-2)
#define OL_LAUNCH_PIPELINED (-1)
#define OL_LAUNCH_PER_ITEM 0
/* set_launch applies one shape to every collision variant (and clears the
 * per-variant shapes the autotuner may have set). */
OL_API int ol_ctx_set_launch(ol_ctx *ctx, int32_t shape);
OL_API int ol_ctx_get_launch(ol_ctx *ctx, int32_t *shape);
/* Shape of the stream-collide launches of one collision variant (operator,
 * WALE on/off, DDF on/off): the autotuner's choice for it, else the
 * context's shape. */
OL_API int ol_ctx_get_variant_launch(ol_ctx *ctx, int32_t op, int32_t wale, int32_t ddf,
                                     int32_t *shape);
/* Times `trials` coarse steps of the resident mix (CUDA events) under each
 * launch shape above and keeps the fastest for the whole mix; then, when the
 * mix holds more than one collision variant, tries each shape for one variant
 * at a time (the others held) and keeps each variant's fastest.  The timing
 * runs advance every resident case by 5 * (trials + 1) coarse steps, and by
 * 5 * (trials + 1) more per variant when there are several. */
OL_API int ol_ctx_autotune(ol_ctx *ctx, int32_t trials);
/* ------------------------------------------------------------------ */
/* Serving: continuous batching of solve requests over one context      */
/* ------------------------------------------------------------------ */
/* No reference counterpart beyond its sequential multi-case loop
 * (run_all_cases, main.jl:413-466).  Requests are admitted in arrival order
 * as soon as their footprint fits the context's budget; all resident cases
 * step together, check_every coarse steps per ol_serve_advance; a case
 * retires when |Cd(t) - Cd(t - window)| < tol after at least min_steps, on
 * its watchdog's non-finite flag, at max_steps, or when Cd is not finite. */
typedef struct ol_serve_rule {
  int32_t check_every;   /* coarse steps between Cd checks                */
  int32_t window;        /* convergence window, a multiple of check_every */
  double tol;            /* |Cd(t) - Cd(t - window)| bound                */
  int32_t max_steps;     /* retire anyway after this many coarse steps    */
  int32_t min_steps;     /* no convergence retirement before this         */
} ol_serve_rule;

/* One retired request.  Times on the server clock (seconds). */
typedef struct ol_serve_result {
  int32_t rid;
  int32_t steps;         /* coarse steps done                              */
  int32_t status;        /* device watchdog bits                           */
  int32_t converged;     /* 1 if retired by the convergence rule           */
  double arrival_s, admit_s, finish_s;
  double coeff[12];      /* last check's record, as ol_ctx_case_coefficients */
} ol_serve_result;

typedef struct ol_server ol_server;
OL_API int ol_server_create(ol_server **out, ol_ctx *ctx, const ol_serve_rule *rule);
/* Removes the cases still resident; the context stays. */
OL_API int ol_server_destroy(ol_server *srv);
/* Seconds since the server was created (steady clock). */
OL_API int ol_server_clock(ol_server *srv, double *now_s);
/* Queues a request arriving at arrival_s (server clock).  The descriptor and
 * the host arrays it points to must stay valid until the request's result
 * has been polled.  Fails with OL_ERR_NOMEM if the case can never fit. */
OL_API int ol_serve_submit(ol_server *srv, const ol_case_desc *cd, const ol_coeff_ref *ref,
                           double arrival_s, int32_t *rid);
/* One round: admit what has arrived and fits, then (if any case is
 * resident) step check_every coarse steps, check Cd, retire.  Synchronous.
 * Reports how many requests are resident and queued afterwards. */
OL_API int ol_serve_advance(ol_server *srv, int32_t *n_resident, int32_t *n_queued);
/* Up to `max` retired requests not yet polled, oldest first. */
OL_API int ol_serve_poll(ol_server *srv, ol_serve_result *out, int32_t max, int32_t *n);
/* The Cd check history of a retired request (*n = its length; up to `max`
 * values copied). */
OL_API int ol_serve_history(ol_server *srv, int32_t rid, double *cd, int32_t max, int32_t *n);

/* Bytes in use / budget / number of resident cases / kernel launches issued. */
OL_API int ol_ctx_stats(ol_ctx *ctx, size_t *used, size_t *budget, int32_t *n_cases,
                 int64_t *launches);

/* Fine-to-coarse restriction, opt-in; no counterpart in the reference, whose
 * levels are coupled coarse to fine only (physics_interpolation.jl).  After a
 * parent step and its two child sub-steps, every parent cell covered by a
 * child block gets the average of its 8 children: fbar = mean f, rho and u
 * from fbar, f = feq(rho, u) + (fbar - feq) * clamp((tau_c - 1/2) /
 * (tau_f - 1/2), 0.01, 100); rho and u are stored.  Parent cells that are
 * solid or have a solid child are left alone.  Column-major reference layout. */
typedef struct ol_restrict_view {
  const float *f_fine;              /* [512*nF*27] child's newest populations  */
  const uint8_t *obstacle_fine;     /* [512*nF]                                 */
  const int32_t *map_x, *map_y, *map_z; /* [nF] child block coordinates        */
  int32_t n_fine;
  float *f_coarse;                  /* [512*nC*27] parent's newest, updated     */
  float *rho_coarse, *vel_coarse;   /* [512*nC], [512*nC*3], updated            */
  const uint8_t *obstacle_coarse;   /* [512*nC]                                 */
  const int32_t *block_ptr;         /* parent block pointer grid                */
  int32_t dim_x, dim_y, dim_z, n_coarse;
  float tau_fine, tau_coarse;
  int32_t compressible;             /* O(u^4) equilibrium when nonzero          */
} ol_restrict_view;
OL_API int ol_restrict(const ol_restrict_view *v, void *stream);

/* ------------------------------------------------------------------------
 * Domain preprocessing on the device (the host build is the reference's
 * CPU path; these give the same bits).  All pointers are device memory:
 *   coords   [n_blocks][3] 1-based block coordinates (x, y, z) of the level
 *   tris     [n_tris][3][3] triangle vertices (mesh frame, FP64)
 *   tri_off  [n_blocks + 1], tri_list: per block, ascending 0-based ids of
 *            the triangles whose bounding box (+ margin) touches the block
 *   offset   host array, the mesh offset added to every vertex
 * ------------------------------------------------------------------------ */
/* Solid cells: some triangle overlaps the cell's box of half size
 * 0.75 dx * 1.001 (separating axes).  Replaces voxelize_blocks!
 * (domain_generation.jl:74-112 with the test of :10-32; margin 2 dx).
 * obstacle [512 n_blocks], 1 = solid (before the flood fill). */
OL_API int ol_voxelize(const int32_t *coords, int32_t n_blocks, const double *tris,
                       int32_t n_tris, const int32_t *tri_off, const int32_t *tri_list,
                       double dx, const double offset[3], uint8_t *obstacle, void *stream);
/* Bouzidi wall distances: per cell and link the nearest ray hit (Moller-
 * Trumbore, eps 1e-9) along the unit link direction, q = t / (dx |c_k|) kept
 * in (0, 1] as binary16 with its 1-based triangle id; has_link marks cells
 * with at least one kept link.  Replaces compute_bouzidi_qmap_sparse
 * (bouzidi_setup.jl:64-166, bouzidi_math.jl:9-101; margin 2.5 dx).
 * q_map / tri_map [27][512 n_blocks] (column-major [x,y,z,b,k]), has_link
 * [512 n_blocks]. */
OL_API int ol_bouzidi_qmap(const int32_t *coords, int32_t n_blocks, const double *tris,
                           int32_t n_tris, const int32_t *tri_off, const int32_t *tri_list,
                           double dx, const double offset[3], uint16_t *q_map,
                           int32_t *tri_map, uint8_t *has_link, void *stream);

/* ------------------------------------------------------------------------
 * FE load mapping: net triangle forces to structural nodes
 * (PREPOST/map_forces_to_nodes.jl).  Each triangle force, applied at its
 * centroid c, goes to the k = min(3, nodes of its object) nearest nodes of
 * the same object (squared distances in FP64, ties to the earlier node) as
 * the minimum-norm solution of
 *   sum_i F_i = F,   sum_i (p_i - c) x F_i = 0,   f = pinv(A) b
 * (A 6 x 3k, singular values at or below 6 eps sigma_max dropped, as
 * LinearAlgebra.pinv does; map_forces_to_nodes.jl:143-231); the nodal load is
 * the sum over triangles.  Nodes and triangles are grouped by object: object
 * o owns nodes [node_begin[o], node_begin[o+1]) and triangles [tri_begin[o],
 * tri_begin[o+1]); an object without nodes leaves its triangles unassigned
 * (node -1, force 0), as the reference skips it.  The sums are exact in
 * per-node fixed point (2^-40 of the node's largest contribution), so the
 * result does not depend on the order the GPU adds in.
 * All arrays are device memory; xyz triples are stored as three planes.
 * ------------------------------------------------------------------------ */
typedef struct ol_fe_map_view {
  const double *node_xyz;       /* [3 * n_nodes]                                   */
  const double *tri_xyz;        /* [3 * n_tris] centroids                         */
  const double *tri_force;      /* [3 * n_tris]                                   */
  const int32_t *node_begin;    /* [n_objects + 1], node_begin[0] = 0             */
  const int32_t *tri_begin;     /* [n_objects + 1], tri_begin[0] = 0              */
  int32_t n_nodes, n_tris, n_objects;
  int32_t *tri_nodes;           /* out [3 * n_tris]: node of slot j (nearest first) at j * n_tris + t, -1 unused */
  double *tri_node_force;       /* out [9 * n_tris]: component c of slot j at (3 j + c) * n_tris + t */
  double *nodal_force;          /* out [3 * n_nodes]                               */
  void *scratch;                /* ol_fe_map_scratch_bytes(n_nodes) bytes           */
} ol_fe_map_view;
/* Bytes of device scratch ol_fe_map_forces needs for n_nodes nodes. */
OL_API size_t ol_fe_map_scratch_bytes(int32_t n_nodes);
/* Map the forces on `stream` and wait for it.  *n_unconverged (host) = the
 * triangles whose SVD sweep limit was reached (their result is still the
 * last iterate).  OL_ERR_ARG for inconsistent sizes or more than 2^21
 * contributions to one node. */
OL_API int ol_fe_map_forces(const ol_fe_map_view *v, int32_t *n_unconverged, void *stream);

/* Message of the last failing call on this thread. */
OL_API const char *ol_last_error(void);
/* Library version string. */
OL_API const char *ol_version(void);

#ifdef __cplusplus
}
#endif
#endif /* OPENLUDWIG_B200_H */
