// Surface-stress forces (surface.jl:143-507 map, :702-762 integrate) and the
// FP64 flow statistics (diagnostics.jl:43-93).
//
// One thread per triangle probes the flow along +n, evaluates pressure and
// wall shear, and turns them into its force and moment contributions; the
// nine sums are reduced in FP64 with warp shuffles, then across CTAs in a
// fixed order by a single-CTA pass, so the result is bitwise reproducible
// (the reference accumulates FP32 atomics in arbitrary order).
#include "common.cuh"
#include "forces.cuh"

namespace ol {



// get_cell_at_position (surface.jl:192-222); 1-based global cell -> index
__device__ __forceinline__ bool cell_at(const ForceDev &D, int gx, int gy, int gz, size_t &ci) {
  if (gx < 1 || gy < 1 || gz < 1) return false;
  const int bx = (gx - 1) / BS + 1, by = (gy - 1) / BS + 1, bz = (gz - 1) / BS + 1;
  if (bx > D.fp.dim_x || by > D.fp.dim_y || bz > D.fp.dim_z) return false;
  const int b = D.bptr[(bx - 1) + D.fp.dim_x * ((by - 1) + D.fp.dim_y * (bz - 1))];
  if (b <= 0) return false;
  ci = (size_t)(D.block_offset + b - 1) * BCELLS + (gx - 1) % BS + BS * ((gy - 1) % BS) +
       BS * BS * ((gz - 1) % BS);
  return true;
}

// trilinear_sample_flow (surface.jl:224-346): fluid-only weights
__device__ bool trilinear_sample(const ForceDev &D, float px, float py, float pz, float &r,
                                 float &ux, float &uy, float &uz, float &wq) {
  const float dx = D.fp.dx;
  const float inv_dx = 1.0f / dx;
  const float fx = px * inv_dx - 0.5f, fy = py * inv_dx - 0.5f, fz = pz * inv_dx - 0.5f;
  const int ix0 = (int)floorf(fx) + 1, iy0 = (int)floorf(fy) + 1, iz0 = (int)floorf(fz) + 1;
  const float wx = fminf(fmaxf(fx - (float)(ix0 - 1), 0.0f), 1.0f);
  const float wy = fminf(fmaxf(fy - (float)(iy0 - 1), 0.0f), 1.0f);
  const float wz = fminf(fmaxf(fz - (float)(iz0 - 1), 0.0f), 1.0f);
  const float w0x = 1.0f - wx, w0y = 1.0f - wy, w0z = 1.0f - wz;
  float ra = 0.f, xa = 0.f, ya = 0.f, za = 0.f, wa = 0.f;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const int ox = s & 1, oy = (s >> 1) & 1, oz = s >> 2;
    const float wk = (ox ? wx : w0x) * (oy ? wy : w0y) * (oz ? wz : w0z);
    size_t ci;
    if (cell_at(D, ix0 + ox, iy0 + oy, iz0 + oz, ci) && !D.obstacle[ci]) {
      ra += wk * D.rho[ci];
      xa += wk * D.vel[ci];
      ya += wk * D.vel[ci + D.dstride];
      za += wk * D.vel[ci + 2 * D.dstride];
      wa += wk;
    }
  }
  if (wa > 0.01f) {
    const float iw = 1.0f / wa;
    r = ra * iw; ux = xa * iw; uy = ya * iw; uz = za * iw; wq = wa;
    return true;
  }
  r = 1.0f; ux = uy = uz = 0.0f; wq = 0.0f;
  return false;
}

// compute_stress_from_cell (surface.jl:143-190)
__device__ void stress_from_cell(const ol_force_params &fp, float rho, float ux, float uy,
                                 float uz, float nx, float ny, float nz, float d, float &p,
                                 float &tx, float &ty, float &tz) {
  p = (rho - 1.0f) / 3.0f * fp.pressure_scale;
  const float un = ux * nx + uy * ny + uz * nz;
  const float utx = ux - un * nx, uty = uy - un * ny, utz = uz - un * nz;
  const float ut = sqrtf(utx * utx + uty * uty + utz * utz);
  const float nu_mol = (fp.tau_molecular - 0.5f) / 3.0f;
  float nu_sgs = 0.0f;
  if (fp.c_wale > 0.0f && d > 0.01f && ut > 1e-10f) nu_sgs = (fp.c_wale * fp.c_wale) * (ut / d);
  nu_sgs = fmaxf(nu_sgs, fp.nu_sgs_bg);
  const float nu_eff = nu_mol + nu_sgs;
  tx = ty = tz = 0.0f;
  if (ut > 1e-10f && d > 0.01f) {
    const float tl = rho * nu_eff * ut / d;
    const float tph = tl * fp.stress_scale;
    tx = (utx / ut) * tph;
    ty = (uty / ut) * tph;
    tz = (utz / ut) * tph;
  }
}

// Flow sample on one side of a triangle centred at t with normal n.
// SIDE = +1: map_stresses_kernel! (surface.jl:380-483) -- ray-march along +n
// from 1.5 cells, first sample with fluid weight >= 0.5 wins, else the best
// one; failing that the nearest fluid cell with dot(c - t, n) > 0, shell by
// shell.  SIDE = -1: map_minus_side_only_kernel! (surface.jl:545-640) -- the
// same along -n, accepting dot < 0 with wall distance |dot| / dx.
template <int SIDE>
__device__ bool probe_side(const ForceDev &D, float tx, float ty, float tz, float nx, float ny,
                           float nz, float &br, float &bux, float &buy, float &buz, float &bd) {
  const ol_force_params &fp = D.fp;
  const float dx = fp.dx;
  br = 1.0f; bux = buy = buz = 0.f; bd = 1.0f;
  float bq = 0.0f;
  bool found = false;
  for (int pi = 1; pi <= fp.search_radius; ++pi) {
    const float dc = (float)pi + 0.5f;
    float px, py, pz;
    if constexpr (SIDE > 0) {
      px = tx + nx * dc * dx; py = ty + ny * dc * dx; pz = tz + nz * dc * dx;
    } else {
      px = tx - nx * dc * dx; py = ty - ny * dc * dx; pz = tz - nz * dc * dx;
    }
    float r, ux, uy, uz, wq;
    const bool ok = trilinear_sample(D, px, py, pz, r, ux, uy, uz, wq);
    if (ok && wq >= 0.5f) {
      br = r; bux = ux; buy = uy; buz = uz; bd = dc; bq = wq; found = true;
      break;
    } else if (ok && wq > bq) {
      br = r; bux = ux; buy = uy; buz = uz; bd = dc; bq = wq; found = true;
    }
  }
  if (found) return true;
  const int gx0 = (int)floorf(tx / dx) + 1, gy0 = (int)floorf(ty / dx) + 1,
            gz0 = (int)floorf(tz / dx) + 1;
  float best = 1e10f;
  for (int rad = 1; rad <= fp.search_radius && !found; ++rad) {
    for (int dz = -rad; dz <= rad; ++dz)
      for (int dy = -rad; dy <= rad; ++dy)
        for (int ddx = -rad; ddx <= rad; ++ddx) {
          if (!(abs(ddx) == rad || abs(dy) == rad || abs(dz) == rad)) continue;
          const int gx = gx0 + ddx, gy = gy0 + dy, gz = gz0 + dz;
          size_t ci;
          if (!cell_at(D, gx, gy, gz, ci) || D.obstacle[ci]) continue;
          const float ddxp = ((float)gx - 0.5f) * dx - tx;
          const float ddyp = ((float)gy - 0.5f) * dx - ty;
          const float ddzp = ((float)gz - 0.5f) * dx - tz;
          const float dn = ddxp * nx + ddyp * ny + ddzp * nz;
          if (SIDE > 0 ? dn <= 0.0f : dn >= 0.0f) continue;
          const float d2 = ddxp * ddxp + ddyp * ddyp + ddzp * ddzp;
          if (d2 < best) {
            best = d2;
            br = D.rho[ci];
            bux = D.vel[ci]; buy = D.vel[ci + D.dstride]; buz = D.vel[ci + 2 * D.dstride];
            bd = (SIDE > 0 ? dn : fabsf(dn)) / dx;
            found = true;
          }
        }
  }
  return found;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kForceThreads = 128;

__global__ void __launch_bounds__(kForceThreads) k_surface_forces(const __grid_constant__ ForceDev D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (i < D.mesh.n_triangles) {
    const ol_force_params &fp = D.fp;
    const float tx = D.mesh.cx[i] + fp.offset_x, ty = D.mesh.cy[i] + fp.offset_y,
                tz = D.mesh.cz[i] + fp.offset_z;
    const float nx = D.mesh.nx[i], ny = D.mesh.ny[i], nz = D.mesh.nz[i];
    float br, bux, buy, buz, bd;
    const bool found = probe_side<1>(D, tx, ty, tz, nx, ny, nz, br, bux, buy, buz, bd);
    float p = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
    if (found) stress_from_cell(fp, br, bux, buy, buz, nx, ny, nz, fmaxf(bd, 0.5f), p, sx, sy, sz);
    if (D.p_map) {
      D.p_map[i] = p; D.sx_map[i] = sx; D.sy_map[i] = sy; D.sz_map[i] = sz;
    }
    // integrate_forces_kernel! (surface.jl:702-762)
    const float A = D.mesh.area[i];
    const float fpx = -p * nx * A, fpy = -p * ny * A, fpz = -p * nz * A;
    const float fvx = sx * A, fvy = sy * A, fvz = sz * A;
    const float Fx = fpx + fvx, Fy = fpy + fvy, Fz = fpz + fvz;
    const float rx = tx - fp.ref_x, ry = ty - fp.ref_y, rz = tz - fp.ref_z;
    c[0] = fpx; c[1] = fpy; c[2] = fpz; c[3] = fvx; c[4] = fvy; c[5] = fvz;
    c[6] = ry * Fz - rz * Fy;
    c[7] = rz * Fx - rx * Fz;
    c[8] = rx * Fy - ry * Fx;
  }
  __shared__ double red[kForceThreads / 32][9];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    const double v = warp_sum(c[j]);
    if (lane == 0) red[wid][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double s = 0.0;
    for (int w = 0; w < kForceThreads / 32; ++w) s += red[w][threadIdx.x];
    D.partials[(size_t)blockIdx.x * 9 + threadIdx.x] = s;
  }
}

// Two-sided net force per triangle in one pass: compute_net_aerodynamics!
// (surface.jl:980-1034) runs the plus-side map, the minus-side map (open
// surfaces only; a closed body's minus maps are zero, surface.jl:987-997) and
// compute_net_triangle_forces_kernel! (surface.jl:665-700) as three launches
// over the triangles; here one thread does all three for its triangle, so the
// maps go to memory only when the caller asks for them.
__global__ void __launch_bounds__(kForceThreads)
    k_surface_net_forces(const __grid_constant__ ForceDev D,
                         const __grid_constant__ ol_net_force_maps M, int closed_body) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.mesh.n_triangles) return;
  const ol_force_params &fp = D.fp;
  const float tx = D.mesh.cx[i] + fp.offset_x, ty = D.mesh.cy[i] + fp.offset_y,
              tz = D.mesh.cz[i] + fp.offset_z;
  const float nx = D.mesh.nx[i], ny = D.mesh.ny[i], nz = D.mesh.nz[i];
  float br, bux, buy, buz, bd;
  float p = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
  if (probe_side<1>(D, tx, ty, tz, nx, ny, nz, br, bux, buy, buz, bd))
    stress_from_cell(fp, br, bux, buy, buz, nx, ny, nz, fmaxf(bd, 0.5f), p, sx, sy, sz);
  float pm = 0.f, sxm = 0.f, sym = 0.f, szm = 0.f;
  if (!closed_body && probe_side<-1>(D, tx, ty, tz, nx, ny, nz, br, bux, buy, buz, bd))
    stress_from_cell(fp, br, bux, buy, buz, -nx, -ny, -nz, fmaxf(bd, 0.5f), pm, sxm, sym, szm);
  if (M.p_plus) {
    M.p_plus[i] = p; M.sx_plus[i] = sx; M.sy_plus[i] = sy; M.sz_plus[i] = sz;
  }
  if (M.p_minus) {
    M.p_minus[i] = pm; M.sx_minus[i] = sxm; M.sy_minus[i] = sym; M.sz_minus[i] = szm;
  }
  const float pn = p - pm, snx = sx - sxm, sny = sy - sym, snz = sz - szm;
  const float A = D.mesh.area[i];
  M.net_fx[i] = -pn * nx * A + snx * A;
  M.net_fy[i] = -pn * ny * A + sny * A;
  M.net_fz[i] = -pn * nz * A + snz * A;
}

// Fixed-order sum of nvals-wide partial rows: out[j] = sum_b partials[b*nvals + j].
__global__ void k_sum_rows(const double *partials, int nrows, int nvals, double *out,
                           int mode_minmax) {
  __shared__ double sh[256];
  for (int j = 0; j < nvals; ++j) {
    const bool is_min = mode_minmax && j == 2;
    const bool is_max = mode_minmax && (j == 3 || j == 4);
    double s = is_min ? 1e300 : (is_max ? -1e300 : 0.0);
    for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
      const double v = partials[(size_t)r * nvals + j];
      s = is_min ? fmin(s, v) : (is_max ? fmax(s, v) : s + v);
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const double a = sh[threadIdx.x], b = sh[threadIdx.x + o];
        sh[threadIdx.x] = is_min ? fmin(a, b) : (is_max ? fmax(a, b) : a + b);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = sh[0];
    __syncthreads();
  }
}

// Per-block FP64 flow statistics: {n_fluid, rho_sum, rho_min, rho_max,
// v_max, kinetic_energy, mass_all}.
__global__ void __launch_bounds__(512) k_flow_stats(const float *rho, const float *vel,
                                                    const uint8_t *obs, int64_t block_offset,
                                                    int64_t dstride, double *partials) {
  const size_t ci = (size_t)(block_offset + blockIdx.x) * BCELLS + threadIdx.x;
  const double r = rho[ci];
  const double ux = vel[ci], uy = vel[ci + dstride], uz = vel[ci + 2 * dstride];
  const double v2 = ux * ux + uy * uy + uz * uz;
  const bool fluid = !obs[ci];
  double v[7] = {fluid ? 1.0 : 0.0, fluid ? r : 0.0, fluid ? r : 1e300, fluid ? r : -1e300,
                 fluid ? sqrt(v2) : 0.0, fluid ? 0.5 * r * v2 : 0.0, r};
  __shared__ double red[16][7];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    double x = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = j == 2 ? fmin(x, y) : ((j == 3 || j == 4) ? fmax(x, y) : x + y);
    }
    if (lane == 0) red[wid][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    const int j = threadIdx.x;
    double s = red[0][j];
    for (int w = 1; w < 16; ++w) {
      const double y = red[w][j];
      s = j == 2 ? fmin(s, y) : ((j == 3 || j == 4) ? fmax(s, y) : s + y);
    }
    partials[(size_t)blockIdx.x * 7 + j] = s;
  }
}

int launch_surface_forces(const ForceDev &D, double *dev_out9, cudaStream_t s) {
  const int nt = D.mesh.n_triangles;
  const int grid = (nt + kForceThreads - 1) / kForceThreads;
  if (grid == 0) return 0;
  k_surface_forces<<<grid, kForceThreads, 0, s>>>(D);
  k_sum_rows<<<1, 256, 0, s>>>(D.partials, grid, 9, dev_out9, 0);
  return 0;
}

int launch_flow_stats(const float *rho, const float *vel, const uint8_t *obs, int32_t nb,
                      int64_t block_offset, int64_t dstride, double *partials, double *dev_out7,
                      cudaStream_t s) {
  if (nb <= 0) return 0;
  k_flow_stats<<<nb, 512, 0, s>>>(rho, vel, obs, block_offset, dstride, partials);
  k_sum_rows<<<1, 256, 0, s>>>(partials, nb, 7, dev_out7, 1);
  return 0;
}

}  // namespace ol

using namespace ol;

extern "C" size_t ol_surface_forces_scratch_doubles(int32_t n_triangles) {
  const int grid = (n_triangles + kForceThreads - 1) / kForceThreads;
  return (size_t)grid * 9 + 16;
}

extern "C" int ol_surface_forces(const ol_surface_mesh *mesh, const float *rho, const float *vel,
                                 const uint8_t *obstacle, const int32_t *block_ptr,
                                 int32_t n_blocks, const ol_force_params *fp, float *p_map,
                                 float *sx_map, float *sy_map, float *sz_map, double *partials,
                                 double out[9], void *stream) {
  OL_CHECK_ARG(mesh && fp && out, "ol_surface_forces: null argument");
  OL_CHECK_ARG(mesh->n_triangles >= 0 && n_blocks > 0, "ol_surface_forces: bad sizes");
  for (int j = 0; j < 9; ++j) out[j] = 0.0;
  if (mesh->n_triangles == 0) return OL_OK;
  OL_CHECK_ARG(mesh->cx && mesh->cy && mesh->cz && mesh->nx && mesh->ny && mesh->nz &&
                   mesh->area && rho && vel && obstacle && block_ptr && partials,
               "ol_surface_forces: null device pointer");
  OL_CHECK_ARG(!p_map == !sx_map && !p_map == !sy_map && !p_map == !sz_map,
               "ol_surface_forces: stress maps must be all given or all null");
  ForceDev D = {};
  D.mesh = *mesh;
  D.rho = rho; D.vel = vel; D.obstacle = obstacle; D.bptr = block_ptr;
  D.block_offset = 0;
  D.dstride = (int64_t)BCELLS * n_blocks;
  D.fp = *fp;
  D.p_map = p_map; D.sx_map = sx_map; D.sy_map = sy_map; D.sz_map = sz_map;
  D.partials = partials;
  const int grid = (mesh->n_triangles + kForceThreads - 1) / kForceThreads;
  double *dev_out = partials + (size_t)grid * 9;
  cudaStream_t s = (cudaStream_t)stream;
  launch_surface_forces(D, dev_out, s);
  OL_LAUNCHED("ol_surface_forces");
  OL_CUDA(cudaMemcpyAsync(out, dev_out, 9 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OL_CUDA(cudaStreamSynchronize(s));
  return OL_OK;
}

extern "C" int ol_surface_net_forces(const ol_surface_mesh *mesh, const float *rho,
                                     const float *vel, const uint8_t *obstacle,
                                     const int32_t *block_ptr, int32_t n_blocks,
                                     const ol_force_params *fp, int32_t closed_body,
                                     const ol_net_force_maps *out, void *stream) {
  OL_CHECK_ARG(mesh && fp && out, "ol_surface_net_forces: null argument");
  OL_CHECK_ARG(mesh->n_triangles >= 0 && n_blocks > 0, "ol_surface_net_forces: bad sizes");
  if (mesh->n_triangles == 0) return OL_OK;
  OL_CHECK_ARG(mesh->cx && mesh->cy && mesh->cz && mesh->nx && mesh->ny && mesh->nz &&
                   mesh->area && rho && vel && obstacle && block_ptr && out->net_fx &&
                   out->net_fy && out->net_fz,
               "ol_surface_net_forces: null device pointer");
  OL_CHECK_ARG(!out->p_plus == !out->sx_plus && !out->p_plus == !out->sy_plus &&
                   !out->p_plus == !out->sz_plus && !out->p_minus == !out->sx_minus &&
                   !out->p_minus == !out->sy_minus && !out->p_minus == !out->sz_minus,
               "ol_surface_net_forces: each side's maps must be all given or all null");
  ForceDev D = {};
  D.mesh = *mesh;
  D.rho = rho; D.vel = vel; D.obstacle = obstacle; D.bptr = block_ptr;
  D.block_offset = 0;
  D.dstride = (int64_t)BCELLS * n_blocks;
  D.fp = *fp;
  const int grid = (mesh->n_triangles + kForceThreads - 1) / kForceThreads;
  k_surface_net_forces<<<grid, kForceThreads, 0, (cudaStream_t)stream>>>(D, *out,
                                                                          closed_body ? 1 : 0);
  OL_LAUNCHED("ol_surface_net_forces");
  return OL_OK;
}

extern "C" int ol_flow_stats_device(const float *rho, const float *vel, const uint8_t *obstacle,
                                    int32_t n_blocks, double *partials, double *out7_dev,
                                    void *stream) {
  OL_CHECK_ARG(n_blocks > 0 && rho && vel && obstacle && partials && out7_dev,
               "ol_flow_stats_device: bad argument");
  launch_flow_stats(rho, vel, obstacle, n_blocks, 0, (int64_t)BCELLS * n_blocks, partials,
                    out7_dev, (cudaStream_t)stream);
  OL_LAUNCHED("ol_flow_stats_device");
  return OL_OK;
}

extern "C" size_t ol_flow_stats_scratch_doubles(int32_t n_blocks) {
  return (size_t)(n_blocks > 0 ? n_blocks : 0) * 7 + 8;
}

extern "C" int ol_flow_stats(const float *rho, const float *vel, const uint8_t *obstacle,
                             int32_t n_blocks, double *partials, double out[7], void *stream) {
  OL_CHECK_ARG(out && n_blocks >= 0, "ol_flow_stats: bad argument");
  for (int j = 0; j < 7; ++j) out[j] = 0.0;
  if (n_blocks == 0) return OL_OK;
  OL_CHECK_ARG(rho && vel && obstacle && partials, "ol_flow_stats: null device pointer");
  cudaStream_t s = (cudaStream_t)stream;
  double *dev_out = partials + (size_t)n_blocks * 7;
  launch_flow_stats(rho, vel, obstacle, n_blocks, 0, (int64_t)BCELLS * n_blocks, partials,
                    dev_out, s);
  OL_LAUNCHED("ol_flow_stats");
  OL_CUDA(cudaMemcpyAsync(out, dev_out, 7 * sizeof(double), cudaMemcpyDeviceToHost, s));
  OL_CUDA(cudaStreamSynchronize(s));
  return OL_OK;
}
