// qphix_gpu_blas_norm2_noalloc: squared norms of a spinor field that make no
// device (or pinned host) allocation at all.
//
// Some callers cannot let a library call cudaMalloc: host codes whose device
// memory is owned by another allocator that has already reserved the free HBM
// (an application that pre-allocates all device memory up front, or a
// framework's caching pool), and codes that must not add the device-wide
// synchronisation cudaMalloc / cudaFree can cause inside a latency-sensitive
// loop.  The regular qphix_gpu_blas_norm2 uses the lattice's reduction
// workspace (allocated with the lattice) and a pinned host mirror; this entry
// point instead takes its per-block partial sums from a fixed array in the
// library's own device memory (below) and writes the result to a device
// buffer the caller owns.
//
// Scratch: g_noalloc_scratch, QPX_NOALLOC_PARTIALS doubles (512 KiB), held
// by every GPU that loads the library until the process exits.  Under CUDA's lazy module loading
// (the default since CUDA 12.2) a device reserves the array at the first
// call made on it (the symbol lookup loads this file's module), so that
// first call belongs before the caller's allocator reserves the free HBM;
// CUDA_MODULE_LOADING=EAGER reserves it when the library is loaded.  A call needs
// ceil(volcb / 128) x nrhs partials; larger requests are rejected.
// Every call shares the array: each call's first kernel writes every partial
// its second kernel (the fold) reads, so nothing carries over from one call
// to the next, but calls whose kernels overlap on the GPU (different streams,
// or different host threads without ordering) race on it.
#include <mutex>

#include "qpx_finalize.cuh"
#include "qpx_host.h"

using namespace qpx;

namespace {

constexpr int QPX_NOALLOC_PARTIALS = 65536;
constexpr int QPX_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_scratch[QPX_NOALLOC_PARTIALS];

std::mutex g_mu;
double *g_scratch_addr[QPX_MAX_DEVICES] = {};

}  // namespace

// records the message returned by qphix_gpu_last_error() (capi.cu)
int qpx_set_last_error(const char *msg, int code);

// Declared in qphix_b200.h.  The first call on a device looks up the scratch
// array's device address (cudaGetSymbolAddress) with that device current;
// later calls reuse it.
extern "C" int qphix_gpu_blas_norm2_noalloc(qphix_gpu_field x, double *out_dev)
{
  if (!x || !out_dev) return qpx_set_last_error("null argument", QPHIX_GPU_EINVAL);
  if (x->kind != QPHIX_GPU_SPINOR) return qpx_set_last_error("x must be a spinor field", QPHIX_GPU_EINVAL);
  auto *lat = x->lat;
  // the field's device must be current
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, x->data) != cudaSuccess)
    return qpx_set_last_error("cannot query the field's device", QPHIX_GPU_ECUDA);
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return qpx_set_last_error("cudaGetDevice failed", QPHIX_GPU_ECUDA);
  if (attr.device != dev)
    return qpx_set_last_error("the field's device is not the current device", QPHIX_GPU_EINVAL);
  if (dev < 0 || dev >= QPX_MAX_DEVICES) return qpx_set_last_error("device ordinal too large", QPHIX_GPU_EINVAL);
  // the result is written by a kernel: out_dev must be device (or managed)
  // memory of this device, never a host buffer
  cudaPointerAttributes oattr;
  if (cudaPointerGetAttributes(&oattr, out_dev) != cudaSuccess) {
    cudaGetLastError();
    return qpx_set_last_error("out_dev is not a device pointer", QPHIX_GPU_EINVAL);
  }
  if ((oattr.type != cudaMemoryTypeDevice && oattr.type != cudaMemoryTypeManaged) || oattr.device != dev)
    return qpx_set_last_error("out_dev must be device or managed memory of the current device", QPHIX_GPU_EINVAL);
  const long long nblocks = (lat->vh + QPX_BLOCK - 1) / QPX_BLOCK;
  if (nblocks * x->nrhs > QPX_NOALLOC_PARTIALS)
    return qpx_set_last_error("qphix_gpu_blas_norm2_noalloc: ceil(volcb/128) * nrhs exceeds 65536 "
                              "(the fixed scratch size); use qphix_gpu_blas_norm2",
                              QPHIX_GPU_EINVAL);
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      cudaError_t e = cudaGetSymbolAddress((void **)&g_scratch_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        return qpx_set_last_error(cudaGetErrorString(e), QPHIX_GPU_ECUDA);
      }
    }
    scratch = g_scratch_addr[dev];
  }
  BlasArgs a;
  memset(&a, 0, sizeof(a));
  a.op = B_NORM2;
  a.vh = (int)lat->vh;
  a.nrhs = x->nrhs;
  a.x = x->sarg();
  a.red.mask = 0x1;
  a.red.nval = 1;
  a.red.fin = FIN_NONE;
  a.red.partials = scratch;
  a.red.result = out_dev;
  a.state = nullptr;
  try {
    launch_blas(x->prec, a, dim3((unsigned)nblocks, x->nrhs), lat->stream);
    launch_fold(a.red, nullptr, x->nrhs, (int)nblocks, lat->stream);
  } catch (const Error &err) {
    return qpx_set_last_error(err.what(), err.code);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return qpx_set_last_error(cudaGetErrorString(e), QPHIX_GPU_ECUDA);
  return QPHIX_GPU_OK;
}
