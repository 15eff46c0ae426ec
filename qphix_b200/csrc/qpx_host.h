// Host-side internals of the C ABI: handle structs, error plumbing and the
// kernel-dispatch entry points implemented by the per-precision .cu files.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qphix_b200.h"
#include "qpx_blas.cuh"
#include "qpx_dslash.cuh"
#include "qpx_layout.cuh"
#include "qpx_reduce.cuh"

namespace qpx {

// error raised inside the library, mapped to a status code at the C boundary
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define QPX_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw ::qpx::Error(e_ == cudaErrorMemoryAllocation ? QPHIX_GPU_ENOMEM : QPHIX_GPU_ECUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

#define QPX_REQUIRE(cond, msg)                                   \
  do {                                                           \
    if (!(cond)) throw ::qpx::Error(QPHIX_GPU_EINVAL, (msg));    \
  } while (0)

// per-precision element geometry of the device layouts
struct ChunkSpec {
  int nchunk;
  int chunk_bytes;
  int vpc;  // values per chunk
};
ChunkSpec spinor_spec(int prec);
ChunkSpec gauge_spec(int prec, int recon);
ChunkSpec clover_spec(int prec, int nreal);

}  // namespace qpx

struct qphix_gpu_lattice_s {
  int dims[4];
  int nxh;
  long long vh;
  long long stride;  // vh rounded up to a multiple of 64
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  int refs = 1;  // the creator's reference plus one per live field
  // fields of a lattice with a memory pool are allocated and freed in stream
  // order on its stream (no device-wide synchronisation); nullptr: cudaMalloc
  cudaMemPool_t mempool = nullptr;
  size_t field_bytes = 0;  // bytes of the live fields (pool temporaries included)
  size_t field_bytes_peak = 0;
  // reduction workspace (one in-flight reduction per stream at a time)
  double *partials = nullptr;
  size_t partials_len = 0;
  double *result = nullptr;       // device [QPX_MAX_RHS * QPX_MAX_RED]
  double *h_result = nullptr;     // pinned mirror
  qpx::SolverState *state = nullptr;   // device
  qpx::SolverState *h_state = nullptr; // pinned mirror
  void *grid_bar = nullptr;             // device GridBarrier of the persistent solvers (lazy)
  void *staging = nullptr;
  size_t staging_bytes = 0;
  // solver temporaries, reused across solves (they hold no lattice reference)
  std::vector<struct qphix_gpu_field_s *> pool_free, pool_all;
  // instantiated solver-iteration graphs, keyed by what they were captured on
  std::map<std::string, cudaGraphExec_t> graphs;
  std::map<std::string, unsigned long long> graph_nodes;
  std::vector<std::string> graph_order;
  qpx::Geom geom() const
  {
    qpx::Geom g;
    g.nx = dims[0];
    g.ny = dims[1];
    g.nz = dims[2];
    g.nt = dims[3];
    g.nxh = nxh;
    g.vh = (int)vh;
    g.div_nxh = qpx::make_divu(nxh);
    g.div_ny = qpx::make_divu(dims[1]);
    g.div_nz = qpx::make_divu(dims[2]);
    return g;
  }
};

struct qphix_gpu_field_s {
  qphix_gpu_lattice_s *lat;
  int kind, prec, recon, nrhs;
  unsigned long long serial = 0;  // unique per created field
  qpx::ChunkSpec spec;
  void *data = nullptr;
  float *norm = nullptr;
  size_t bytes = 0;
  bool pooled = false;  // allocated from the lattice's memory pool
  qpx::SpinorArg sarg() const
  {
    qpx::SpinorArg a;
    a.data = data;
    a.norm = norm;
    a.stride = lat->stride;
    a.rhs_stride_chunks = (long long)spec.nchunk * lat->stride;
    return a;
  }
  qpx::GaugeArg garg() const
  {
    qpx::GaugeArg a;
    a.data = data;
    a.stride = lat->stride;
    a.mu_stride = (long long)spec.nchunk * lat->stride;
    return a;
  }
  qpx::CloverArg carg() const
  {
    qpx::CloverArg a;
    a.data = data;
    a.stride = lat->stride;
    return a;
  }
};

struct qphix_gpu_eo_op_s {
  unsigned long long serial = 0;  // unique per created operator
  qphix_gpu_op_params p;
  qphix_gpu_field_s *gauge, *clov, *invclov, *finv0, *finv1;
  std::map<int, qphix_gpu_field_s *> tmp;  // by nrhs
  std::vector<int> pretuned;                // nrhs values whose Dslash shapes were tuned
};

namespace qpx {

}  // namespace qpx

// records `msg` as the calling thread's last error and returns `code`
int qpx_set_last_error(const char *msg, int code);

namespace qpx {

// ---- lattices for the serving layer ----------------------------------------
// A lattice whose fields come from `pool` in stream order (own stream).
int lattice_create_pooled(const int latt[4], cudaMemPool_t pool, qphix_gpu_lattice_s **out);
// Wait for the lattice's stream, then free its pooled solver temporaries and
// staging buffer and drop its cached iteration graphs.
void lattice_trim(qphix_gpu_lattice_s *L);

// ---- dispatch (implemented per precision) ----------------------------------
// Launch shape of the Dslash kernel: R right-hand sides per thread, SP
// lattice sites per thread, gen = the general path (direction mask, twisted
// boundary phases).  Grid: ceil(Vh / (QPX_BLOCK SP)) site blocks x nrhs / R.
struct DslashShape {
  int R = 1, SP = 1;
  bool gen = false;
  bool rl = false;  // with R = 1, SP = 2: two right-hand sides of one site in the float2 lanes
};
// a == nullptr: report only whether the shape is built for (prec, recon)
bool launch_dslash(int prec, int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                   cudaStream_t st);
void launch_blas(int prec, const BlasArgs &a, dim3 grid, cudaStream_t st);
// folds the block partials of the reducing launch just issued on `st` (nparts
// site blocks) and runs its finalize step (fold_kernel, blas.cu)
void launch_fold(const ReduceArg &ra, SolverState *state, int nrhs, int nparts, cudaStream_t st);
void launch_convert(int pdst, int psrc, int vh, SpinorArg src, SpinorArg dst, Coef scale, SolverState *state,
                    dim3 grid, cudaStream_t st, int accumulate = 0);
void launch_spinor_in(int prec, Geom g, HostLayout L, const void *host, SpinorArg f, int nrhs, dim3 grid,
                      cudaStream_t st);
void launch_spinor_out(int prec, Geom g, HostLayout L, void *host, SpinorArg f, int nrhs, dim3 grid,
                       cudaStream_t st);
void launch_gauge_in(int prec, Geom g, HostLayout L, const void *host, void *dev, long long stride,
                     long long slab_bytes, int vpc, int recon, int cb, int back, dim3 grid, cudaStream_t st);
void launch_clover_in(int prec, Geom g, HostLayout L, const void *host, void *dev, long long stride, int vpc,
                      int nr, dim3 grid, cudaStream_t st);
void launch_clover_out(int prec, Geom g, HostLayout L, void *host, const void *dev, long long stride, int vpc,
                       int nr, dim3 grid, cudaStream_t st);
void launch_mshift(int prec, const MShiftArgs &a, dim3 grid, cudaStream_t st);
void launch_clover_build(int recon, int prec_out, Geom geo, GaugeArg g, void *out, long long stride, int vpc, int cb,
                         double diag_mass, double cr, double ct, dim3 grid, cudaStream_t st);
void launch_clover_invert(int prec_in, int prec_out, Geom geo, const void *in, long long stride, int vpc_in, void *o0,
                          void *o1, int vpc_out, int mode, double mu, dim3 grid, cudaStream_t st, void *o2 = nullptr,
                          int vpc_out2 = 0, double eps = 0.0);
void launch_two_flav_clover(int prec, int vh, int npairs, SpinorArg out, SpinorArg in, CloverArg fa, CloverArg fb,
                            CloverArg c, cudaStream_t st);
void launch_clover_convert(int prec_in, int prec_out, Geom geo, const void *in, int vpc_in, void *out, int vpc_out,
                           long long stride, int nr, dim3 grid, cudaStream_t st);
// halo mode: copy the sites of one checkerboard of the slice `slice` along
// mu (face order of DslashArgs::halo) from `rows` chunk rows of src (row r at
// src + r * src_stride chunks) to dst ([row][face]); with nsrc, also nrows
// per-site norm rows to ndst ([row][face]); halo.cu
void launch_face_pack(const Geom &g, int mu, int slice, int cb, const void *src, long long src_stride, int rows,
                      int chunk_bytes, long long face, void *dst, const float *nsrc, float *ndst, int nrows,
                      cudaStream_t st);
// persistent CG kernel (qpx_persist.cuh) for (recon, Wilson or clover) with
// FP64 / FP32 storage and isign = +1; nullptr where none is built
const void *cg_persistent_kernel_f64(int recon, bool clover);
const void *cg_persistent_kernel_f32(int recon, bool clover);


}  // namespace qpx
