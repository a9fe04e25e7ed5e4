// Sparse Bouzidi correction with library-owned scratch, for callers that
// cannot allocate device memory themselves.
//
// ol_bouzidi_sparse needs a caller-owned scratch buffer of 27 floats per
// boundary cell between its gather and scatter phases.  Some callers have no
// way to provide one: their device memory is entirely reserved by another
// allocator's pool (CUDA.jl's or PyTorch's caching allocator), where a raw
// cudaMalloc can fail even though the pool has room, or they run a loop that
// must not allocate at all.  This variant keeps the scratch in a file-scope
// device array of fixed size instead, so a call allocates nothing.
#include <cuda.h>  // driver types only; the entry points are fetched at run time

#include <mutex>

#include "bouzidi.cuh"
#include "common.cuh"

namespace ol {

// Resident on every device that loads the library, until process exit.
static __device__ __align__(256) float g_bouzidi_scratch[(size_t)OL_BOUZIDI_NOALLOC_MAX_CELLS * 27];

// Unique id of the calling thread's current CUDA context (0 when none is
// current yet), through the driver's cuCtxGetCurrent / cuCtxGetId, fetched
// from the runtime once (the library links only the static runtime).
static int current_context_id(unsigned long long *id) {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q{};
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent)p;
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetId)p;
  });
  if (!get_current || !get_id)
    return set_error(OL_ERR_CUDA, "ol_bouzidi_sparse_noalloc: driver context queries unavailable");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS)
    return set_error(OL_ERR_CUDA, "ol_bouzidi_sparse_noalloc: cuCtxGetCurrent failed");
  *id = 0;
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS)
    return set_error(OL_ERR_CUDA, "ol_bouzidi_sparse_noalloc: cuCtxGetId failed");
  return OL_OK;
}

// The array's name is only a host-side stand-in in host code; the kernels
// need its device address, looked up with the device current.  The address
// is kept per device together with the id of the context it belongs to and
// looked up again when the current context is another one (after a device
// reset, or a context the caller created itself).
static int noalloc_scratch(float **out) {
  static std::mutex mu;
  static float *per_dev[64] = {};
  static unsigned long long ctx_of[64] = {};
  int dev = 0;
  OL_CUDA(cudaGetDevice(&dev));
  OL_CHECK_ARG(dev >= 0 && dev < 64, "ol_bouzidi_sparse_noalloc: device id %d out of range", dev);
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(mu);
  if (!per_dev[dev] || id == 0 || ctx_of[dev] != id) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_bouzidi_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_bouzidi_scratch)");
    // the lookup makes the device's primary context current if none was
    if (id == 0 && (rc = current_context_id(&id))) return rc;
    per_dev[dev] = (float *)p;
    ctx_of[dev] = id;
  }
  *out = per_dev[dev];
  return OL_OK;
}

}  // namespace ol

using namespace ol;

extern "C" int ol_bouzidi_sparse_noalloc(float *f_out, const uint16_t *q_map,
                                         const int32_t *cell_block, const int8_t *cell_x,
                                         const int8_t *cell_y, const int8_t *cell_z,
                                         int32_t n_boundary, const int32_t *neighbor_table,
                                         int32_t n_blocks, float q_min_threshold, void *stream) {
  OL_CHECK_ARG(n_boundary >= 0 && n_blocks >= 0, "ol_bouzidi_sparse_noalloc: negative size");
  OL_CHECK_ARG(n_boundary <= OL_BOUZIDI_NOALLOC_MAX_CELLS,
               "ol_bouzidi_sparse_noalloc: %d boundary cells exceed the fixed scratch of %d cells; "
               "use ol_bouzidi_sparse with caller-owned scratch",
               n_boundary, OL_BOUZIDI_NOALLOC_MAX_CELLS);
  if (n_boundary == 0) return OL_OK;
  OL_CHECK_ARG(f_out && q_map && cell_block && cell_x && cell_y && cell_z && neighbor_table,
               "ol_bouzidi_sparse_noalloc: null device pointer");
  float *scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  BouzDev B{};
  B.f = f_out;
  B.src = f_out;
  B.q = q_map;
  B.dense_q = 1;
  B.cell_block = cell_block; B.cell_x = cell_x; B.cell_y = cell_y; B.cell_z = cell_z;
  B.n_boundary = n_boundary;
  B.nbr = neighbor_table; B.nbr_stride = n_blocks;
  B.block_offset = 0;
  B.dstride = (int64_t)BCELLS * n_blocks;
  B.q_min = q_min_threshold; B.scale = 1.0f; B.inv_scale = 1.0f;
  // Nothing here has to start at zero: the scatter phase reads exactly the
  // slots the gather phase of the same call has just written.
  B.scratch = scratch;
  launch_bouzidi(B, false, (cudaStream_t)stream);
  OL_LAUNCHED("ol_bouzidi_sparse_noalloc");
  return OL_OK;
}
