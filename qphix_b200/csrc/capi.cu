// C ABI implementation: lattices, fields, the Dslash family, the even-odd
// operators, BLAS and the Krylov solvers.  All device work of a lattice is
// ordered on its stream.  Solver iterations keep every scalar on the device
// (qpx_finalize.cuh) and are captured once per solve as a CUDA graph that is
// replayed until the device-side `done` flag is raised; the host only polls
// that flag every few iterations.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "qpx_finalize.cuh"
#include "qpx_host.h"
#include "qpx_persist.cuh"

using namespace qpx;

static thread_local std::string g_last_error;

int qpx_set_last_error(const char *msg, int code)
{
  g_last_error = msg;
  return code;
}

template <typename F>
static int guard(F &&f)
{
  try {
    f();
    return QPHIX_GPU_OK;
  } catch (const Error &e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return QPHIX_GPU_EINVAL;
  }
}

static int nblocks_for(long long n) { return (int)((n + QPX_BLOCK - 1) / QPX_BLOCK); }

static std::atomic<unsigned long long> g_launches{0};
static std::atomic<unsigned long long> g_serial{1};

static void check_launch()
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(QPHIX_GPU_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  g_launches++;
}

extern "C" int qphix_gpu_launch_count(unsigned long long *out)
{
  if (!out) return QPHIX_GPU_EINVAL;
  *out = g_launches.load();
  return QPHIX_GPU_OK;
}

static void lattice_release(qphix_gpu_lattice_s *L);
static void field_free(qphix_gpu_field_s *f);

// device memory of a lattice's fields: stream-ordered from its pool, or cudaMalloc
static cudaError_t dev_alloc(qphix_gpu_lattice_s *L, void **p, size_t bytes)
{
  if (L->mempool) return cudaMallocFromPoolAsync(p, bytes, L->mempool, L->stream);
  return cudaMalloc(p, bytes);
}

static void dev_free(qphix_gpu_lattice_s *L, bool pooled, void *p)
{
  if (!p) return;
  if (pooled)
    cudaFreeAsync(p, L->stream);
  else
    cudaFree(p);
}

static bool env_flag(const char *name)
{
  const char *v = getenv(name);
  return v && v[0] && v[0] != '0';
}

// ===========================================================================
// lattice
// ===========================================================================
extern "C" int qphix_gpu_version(void) { return 100; }
extern "C" const char *qphix_gpu_last_error(void) { return g_last_error.c_str(); }

extern "C" int qphix_gpu_init(int device)
{
  return guard([&] {
    int n = 0;
    QPX_CUDA(cudaGetDeviceCount(&n));
    QPX_REQUIRE(device >= 0 && device < n, "device index out of range");
    QPX_CUDA(cudaSetDevice(device));
  });
}

static void create_lattice(const int latt[4], cudaMemPool_t pool, qphix_gpu_lattice *out);

extern "C" int qphix_gpu_lattice_create(const int latt[4], qphix_gpu_lattice *out)
{
  return guard([&] { create_lattice(latt, nullptr, out); });
}

int qpx::lattice_create_pooled(const int latt[4], cudaMemPool_t pool, qphix_gpu_lattice_s **out)
{
  return guard([&] {
    QPX_REQUIRE(pool, "null memory pool");
    create_lattice(latt, pool, out);
  });
}

void qpx::lattice_trim(qphix_gpu_lattice_s *L)
{
  QPX_CUDA(cudaStreamSynchronize(L->stream));
  for (auto &kv : L->graphs) cudaGraphExecDestroy(kv.second);
  L->graphs.clear();
  L->graph_nodes.clear();
  L->graph_order.clear();
  for (auto *f : L->pool_all) field_free(f);
  L->pool_all.clear();
  L->pool_free.clear();
  if (L->staging) dev_free(L, L->mempool != nullptr, L->staging);
  L->staging = nullptr;
  L->staging_bytes = 0;
}

static void create_lattice(const int latt[4], cudaMemPool_t pool, qphix_gpu_lattice *out)
{
  {
    QPX_REQUIRE(latt && out, "null argument");
    for (int i = 0; i < 4; i++) QPX_REQUIRE(latt[i] >= 2, "every lattice extent must be >= 2");
    QPX_REQUIRE(latt[0] % 2 == 0, "Nx must be even (checkerboarding)");
    auto *L = new qphix_gpu_lattice_s();
    try {
      for (int i = 0; i < 4; i++) L->dims[i] = latt[i];
      L->nxh = latt[0] / 2;
      L->vh = (long long)L->nxh * latt[1] * latt[2] * latt[3];
      QPX_REQUIRE(L->vh < (1LL << 30), "lattice too large for 32-bit site indices");
      L->stride = (L->vh + 63) / 64 * 64;
      QPX_CUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
      L->owns_stream = true;
      L->mempool = pool;
      // per-block partials, plus 3 x QPX_MAX_RHS doubles at the end: the
      // Richardson per-rhs scale factors (last two) and the shifted CG's
      // per-rhs shifts (shift_coefs)
      L->partials_len = (size_t)nblocks_for(L->vh) * QPX_MAX_RHS * QPX_MAX_RED + 3 * QPX_MAX_RHS;
      QPX_CUDA(cudaMalloc(&L->partials, L->partials_len * sizeof(double)));
      QPX_CUDA(cudaMalloc(&L->result, QPX_MAX_RHS * QPX_MAX_RED * sizeof(double)));
      QPX_CUDA(cudaMallocHost(&L->h_result, QPX_MAX_RHS * QPX_MAX_RED * sizeof(double)));
      QPX_CUDA(cudaMalloc(&L->state, sizeof(SolverState)));
      QPX_CUDA(cudaMallocHost(&L->h_state, sizeof(SolverState)));
      memset(L->h_state, 0, sizeof(SolverState));
      QPX_CUDA(cudaMemset(L->state, 0, sizeof(SolverState)));
    } catch (...) {
      lattice_release(L);
      throw;
    }
    *out = L;
  }
}

static void lattice_release(qphix_gpu_lattice_s *L)
{
  if (!L) return;
  if (--L->refs > 0) return;
  if (L->stream) cudaStreamSynchronize(L->stream);
  for (auto &kv : L->graphs) cudaGraphExecDestroy(kv.second);
  for (auto *f : L->pool_all) field_free(f);
  if (L->staging) dev_free(L, L->mempool != nullptr, L->staging);
  if (L->stream) cudaStreamSynchronize(L->stream);
  cudaFree(L->partials);
  cudaFree(L->result);
  cudaFreeHost(L->h_result);
  cudaFree(L->state);
  cudaFreeHost(L->h_state);
  if (L->grid_bar) cudaFree(L->grid_bar);
  if (L->stream && L->owns_stream) cudaStreamDestroy(L->stream);
  delete L;
}

// The lattice stays alive until its last field is destroyed as well.
extern "C" int qphix_gpu_lattice_destroy(qphix_gpu_lattice L)
{
  return guard([&] { lattice_release(L); });
}

extern "C" int qphix_gpu_lattice_set_stream(qphix_gpu_lattice L, void *stream)
{
  return guard([&] {
    QPX_REQUIRE(L, "null lattice");
    QPX_REQUIRE(stream, "a non-default stream is required (iterations are graph-captured)");
    QPX_CUDA(cudaStreamSynchronize(L->stream));
    if (L->owns_stream) QPX_CUDA(cudaStreamDestroy(L->stream));
    L->stream = (cudaStream_t)stream;
    L->owns_stream = false;
  });
}

extern "C" int qphix_gpu_lattice_sync(qphix_gpu_lattice L)
{
  return guard([&] {
    QPX_REQUIRE(L, "null lattice");
    QPX_CUDA(cudaStreamSynchronize(L->stream));
  });
}

extern "C" long qphix_gpu_lattice_volcb(qphix_gpu_lattice L) { return L ? (long)L->vh : -1; }

static void *staging(qphix_gpu_lattice_s *L, size_t bytes)
{
  if (bytes > L->staging_bytes) {
    if (!L->mempool) QPX_CUDA(cudaStreamSynchronize(L->stream));
    dev_free(L, L->mempool != nullptr, L->staging);
    L->staging = nullptr;
    L->staging_bytes = 0;
    QPX_CUDA(dev_alloc(L, &L->staging, bytes));
    L->staging_bytes = bytes;
  }
  return L->staging;
}

// ===========================================================================
// fields
// ===========================================================================
extern "C" int qphix_gpu_field_create(qphix_gpu_lattice L, int kind, int prec, int recon, int nrhs,
                                      qphix_gpu_field *out)
{
  return guard([&] {
    QPX_REQUIRE(L && out, "null argument");
    QPX_REQUIRE(prec >= PREC_F64 && prec <= PREC_Q16F32, "bad precision");
    auto *f = new qphix_gpu_field_s();
    f->lat = L;
    f->serial = g_serial++;
    L->refs++;
    f->kind = kind;
    f->prec = prec;
    f->recon = 0;
    f->nrhs = 1;
    size_t rows = 0;
    switch (kind) {
    case QPHIX_GPU_SPINOR:
      QPX_REQUIRE(nrhs >= 1 && nrhs <= QPX_MAX_RHS, "nrhs must be in [1, 32]");
      f->nrhs = nrhs;
      f->spec = spinor_spec(prec);
      rows = (size_t)nrhs;
      break;
    case QPHIX_GPU_GAUGE:
      QPX_REQUIRE(recon == 12 || recon == 18, "gauge recon must be 12 or 18");
      f->recon = recon;
      f->spec = gauge_spec(prec, recon);
      rows = 8;  // [cb][mu]
      break;
    case QPHIX_GPU_CLOVER:
      f->spec = clover_spec(prec, 72);
      rows = 1;
      break;
    case QPHIX_GPU_FULLCLOVER:
      f->spec = clover_spec(prec, 144);
      rows = 1;
      break;
    default:
      L->refs--;
      delete f;
      throw Error(QPHIX_GPU_EINVAL, "bad field kind");
    }
    f->bytes = rows * f->spec.nchunk * (size_t)f->spec.chunk_bytes * L->stride;
    f->pooled = L->mempool != nullptr;
    cudaError_t e = dev_alloc(L, &f->data, f->bytes);
    if (e != cudaSuccess) {
      L->refs--;
      delete f;
      throw Error(QPHIX_GPU_ENOMEM, std::string("field allocation: ") + cudaGetErrorString(e));
    }
    cudaMemsetAsync(f->data, 0, f->bytes, L->stream);
    if (kind == QPHIX_GPU_SPINOR && prec >= PREC_F16) {
      void *nm = nullptr;
      e = dev_alloc(L, &nm, sizeof(float) * L->stride * f->nrhs);
      if (e != cudaSuccess) {
        dev_free(L, f->pooled, f->data);
        L->refs--;
        delete f;
        throw Error(QPHIX_GPU_ENOMEM, std::string("norm allocation: ") + cudaGetErrorString(e));
      }
      f->norm = static_cast<float *>(nm);
      cudaMemsetAsync(f->norm, 0, sizeof(float) * L->stride * f->nrhs, L->stream);
      f->bytes += sizeof(float) * L->stride * f->nrhs;
    }
    L->field_bytes += f->bytes;
    if (L->field_bytes > L->field_bytes_peak) L->field_bytes_peak = L->field_bytes;
    *out = f;
  });
}

static void field_free(qphix_gpu_field_s *f)
{
  qphix_gpu_lattice_s *L = f->lat;
  if (!f->pooled) cudaStreamSynchronize(L->stream);
  dev_free(L, f->pooled, f->data);
  dev_free(L, f->pooled, f->norm);
  L->field_bytes -= f->bytes;
  delete f;
}

extern "C" int qphix_gpu_field_destroy(qphix_gpu_field f)
{
  return guard([&] {
    if (!f) return;
    qphix_gpu_lattice_s *L = f->lat;
    field_free(f);
    lattice_release(L);
  });
}

extern "C" int qphix_gpu_field_bytes(qphix_gpu_field f, size_t *bytes)
{
  return guard([&] {
    QPX_REQUIRE(f && bytes, "null argument");
    *bytes = f->bytes;
  });
}

static HostLayout make_layout(const qphix_gpu_field_s *f, const qphix_gpu_host_layout *hl)
{
  HostLayout L{};
  QPX_REQUIRE(hl, "null host layout");
  L.kind = hl->kind;
  L.ft = hl->ft;
  QPX_REQUIRE(L.ft >= 0 && L.ft <= 2, "bad host element type");
  if (L.kind == HOST_CANONICAL) {
    QPX_REQUIRE(L.ft == HFT_F64, "canonical host arrays are FP64");
    return L;
  }
  if (L.kind == HOST_QDP) {
    QPX_REQUIRE(L.ft == HFT_F64 || L.ft == HFT_F32, "qdp host arrays are FP64 or FP32");
    QPX_REQUIRE(f->kind != QPHIX_GPU_FULLCLOVER, "qdp layout: full clover fields are not supported");
    L.cb = hl->cb;
    QPX_REQUIRE(f->kind == QPHIX_GPU_GAUGE || L.cb == 0 || L.cb == 1, "qdp layout: cb must be 0 or 1");
    return L;
  }
  QPX_REQUIRE(L.kind == HOST_QPHIX, "bad host layout kind");
  const auto *lat = f->lat;
  L.V = hl->veclen;
  L.S = hl->soalen;
  L.c12 = hl->compress12 ? 1 : 0;
  QPX_REQUIRE(L.V > 0 && L.S > 0 && L.V % L.S == 0, "soalen must divide veclen");
  QPX_REQUIRE(lat->nxh % L.S == 0, "Nx/2 must be divisible by soalen");
  L.nvecs = lat->nxh / L.S;
  L.ngy = L.V / L.S;
  QPX_REQUIRE(lat->dims[1] % L.ngy == 0, "Ny must be divisible by veclen/soalen");
  L.pxy = L.nvecs * lat->dims[1] + hl->pad_xy;
  L.pxyz = L.pxy * lat->dims[2] + hl->pad_xyz;
  return L;
}

static size_t host_elem_bytes(int ft) { return ft == HFT_F64 ? 8 : (ft == HFT_F32 ? 4 : 2); }

// number of host elements of a field transfer
static size_t host_elems(const qphix_gpu_field_s *f, const HostLayout &L, int nrhs)
{
  const auto *lat = f->lat;
  size_t vh = lat->vh;
  if (L.kind != HOST_QPHIX) {  // canonical, or the compacted qdp staging
    switch (f->kind) {
    case QPHIX_GPU_SPINOR: return (size_t)nrhs * vh * 24;
    case QPHIX_GPU_GAUGE: return 2 * 4 * vh * 18;
    case QPHIX_GPU_CLOVER: return vh * 72;
    default: return vh * 144;
    }
  }
  size_t nt = lat->dims[3];
  switch (f->kind) {
  case QPHIX_GPU_SPINOR: return (size_t)nrhs * L.pxyz * nt * 24 * L.S;
  case QPHIX_GPU_GAUGE: return (size_t)L.pxyz * nt * L.S / L.V * 8 * (L.c12 ? 2 : 3) * 3 * 2 * L.V;
  case QPHIX_GPU_CLOVER: return (size_t)L.pxyz * nt * L.S / L.V * 72 * L.V;
  default: return (size_t)L.pxyz * nt * L.S / L.V * 144 * L.V;
  }
}

// qdp layout: spinor and clover transfers move checkerboard L.cb of each
// full-lattice host array ([V] sites = 2 halves of vh) to / from a compacted
// staging buffer, one contiguous copy per right-hand side
static void qdp_half_copies(const qphix_gpu_field_s *f, const HostLayout &L, int nr, void *host, void *st,
                            bool to_device)
{
  size_t per = (f->kind == QPHIX_GPU_SPINOR ? 24 : 72) * (size_t)f->lat->vh * host_elem_bytes(L.ft);
  for (int i = 0; i < nr; i++) {
    char *h = (char *)host + (2 * (size_t)i + L.cb) * per;
    char *d = (char *)st + (size_t)i * per;
    if (to_device)
      QPX_CUDA(cudaMemcpyAsync(d, h, per, cudaMemcpyHostToDevice, f->lat->stream));
    else
      QPX_CUDA(cudaMemcpyAsync(h, d, per, cudaMemcpyDeviceToHost, f->lat->stream));
  }
}

static SpinorArg rhs_view(const qphix_gpu_field_s *f, int rhs)
{
  SpinorArg a = f->sarg();
  if (rhs > 0) {
    a.data = (char *)a.data + (size_t)rhs * a.rhs_stride_chunks * f->spec.chunk_bytes;
    if (a.norm) a.norm += (size_t)rhs * f->lat->stride;
  }
  return a;
}

extern "C" int qphix_gpu_field_upload(qphix_gpu_field f, const void *host, const qphix_gpu_host_layout *hl, int cb,
                                      int rhs)
{
  return guard([&] {
    QPX_REQUIRE(f && host, "null argument");
    auto *lat = f->lat;
    HostLayout L = make_layout(f, hl);
    Geom g = lat->geom();
    int nr = (f->kind == QPHIX_GPU_SPINOR) ? ((rhs < 0) ? f->nrhs : 1) : 1;
    QPX_REQUIRE(rhs < f->nrhs, "rhs index out of range");
    size_t bytes = host_elems(f, L, nr) * host_elem_bytes(L.ft);
    void *st = staging(lat, bytes);
    if (L.kind == HOST_QDP && f->kind != QPHIX_GPU_GAUGE) {
      QPX_REQUIRE(cb == -1 || cb == L.cb, "qdp layout: the checkerboard is given by layout->cb");
      qdp_half_copies(f, L, nr, const_cast<void *>(host), st, true);
    } else {
      QPX_CUDA(cudaMemcpyAsync(st, host, bytes, cudaMemcpyHostToDevice, lat->stream));
    }
    switch (f->kind) {
    case QPHIX_GPU_SPINOR: {
      SpinorArg a = rhs_view(f, rhs < 0 ? 0 : rhs);
      launch_spinor_in(f->prec, g, L, st, a, nr, dim3(nblocks_for(lat->vh), nr), lat->stream);
      break;
    }
    case QPHIX_GPU_GAUGE: {
      long long slab = (long long)f->spec.nchunk * f->spec.chunk_bytes * lat->stride;
      if (L.kind != HOST_QPHIX) {
        QPX_REQUIRE(cb == -1, "canonical / qdp gauge arrays hold both checkerboards (cb = -1)");
        for (int c = 0; c < 2; c++)
          launch_gauge_in(f->prec, g, L, st, f->data, lat->stride, slab, f->spec.vpc, f->recon, c, 0,
                          dim3(nblocks_for(lat->vh), 4), lat->stream);
      } else {
        QPX_REQUIRE(cb >= 0 && cb <= 3, "qphix gauge arrays: cb = 0/1 (forward links of that checkerboard) "
                                        "or 2/3 (all eight links of checkerboard cb - 2)");
        int c0 = cb & 1;
        launch_gauge_in(f->prec, g, L, st, f->data, lat->stride, slab, f->spec.vpc, f->recon, c0, 0,
                        dim3(nblocks_for(lat->vh), 4), lat->stream);
        if (cb >= 2)
          launch_gauge_in(f->prec, g, L, st, f->data, lat->stride, slab, f->spec.vpc, f->recon, c0, 1,
                          dim3(nblocks_for(lat->vh), 4), lat->stream);
      }
      break;
    }
    case QPHIX_GPU_CLOVER:
    case QPHIX_GPU_FULLCLOVER:
      launch_clover_in(f->prec, g, L, st, f->data, lat->stride, f->spec.vpc,
                       f->kind == QPHIX_GPU_CLOVER ? 72 : 144, dim3(nblocks_for(lat->vh)), lat->stream);
      break;
    }
    check_launch();
  });
}

extern "C" int qphix_gpu_field_download(qphix_gpu_field f, void *host, const qphix_gpu_host_layout *hl, int rhs)
{
  return guard([&] {
    QPX_REQUIRE(f && host, "null argument");
    auto *lat = f->lat;
    HostLayout L = make_layout(f, hl);
    Geom g = lat->geom();
    QPX_REQUIRE(rhs < f->nrhs, "rhs index out of range");
    int nr = (f->kind == QPHIX_GPU_SPINOR) ? ((rhs < 0) ? f->nrhs : 1) : 1;
    size_t bytes = host_elems(f, L, nr) * host_elem_bytes(L.ft);
    void *st = staging(lat, bytes);
    if (f->kind == QPHIX_GPU_SPINOR) {
      if (L.kind == HOST_QPHIX) QPX_CUDA(cudaMemsetAsync(st, 0, bytes, lat->stream));
      SpinorArg a = rhs_view(f, rhs < 0 ? 0 : rhs);
      launch_spinor_out(f->prec, g, L, st, a, nr, dim3(nblocks_for(lat->vh), nr), lat->stream);
    } else if (f->kind == QPHIX_GPU_CLOVER || f->kind == QPHIX_GPU_FULLCLOVER) {
      QPX_REQUIRE(L.kind != HOST_QPHIX, "clover download supports the canonical and qdp layouts");
      launch_clover_out(f->prec, g, L, st, f->data, lat->stride, f->spec.vpc, f->kind == QPHIX_GPU_CLOVER ? 72 : 144,
                        dim3(nblocks_for(lat->vh)), lat->stream);
    } else {
      throw Error(QPHIX_GPU_EUNSUPPORTED, "gauge download is not supported");
    }
    check_launch();
    if (L.kind == HOST_QDP)
      qdp_half_copies(f, L, nr, host, st, false);
    else
      QPX_CUDA(cudaMemcpyAsync(host, st, bytes, cudaMemcpyDeviceToHost, lat->stream));
    QPX_CUDA(cudaStreamSynchronize(lat->stream));
  });
}

static void convert_field(qphix_gpu_field_s *dst, qphix_gpu_field_s *src, Coef scale, SolverState *state,
                          int accumulate = 0)
{
  auto *lat = src->lat;
  launch_convert(dst->prec, src->prec, (int)lat->vh, src->sarg(), dst->sarg(), scale, state,
                 dim3(nblocks_for(lat->vh), src->nrhs), lat->stream, accumulate);
  check_launch();
}

extern "C" int qphix_gpu_field_convert(qphix_gpu_field dst, qphix_gpu_field src, double scale)
{
  return guard([&] {
    QPX_REQUIRE(dst && src, "null argument");
    QPX_REQUIRE(dst->kind == QPHIX_GPU_SPINOR && src->kind == QPHIX_GPU_SPINOR, "convert works on spinors");
    QPX_REQUIRE(dst->nrhs == src->nrhs && dst->lat == src->lat, "shape mismatch");
    Coef c{scale, 0, nullptr, nullptr};
    convert_field(dst, src, c, nullptr);
  });
}

// ===========================================================================
// Dslash launch plumbing
// ===========================================================================
static DslashArgs base_args(const qphix_gpu_op_params &p, qphix_gpu_lattice_s *lat, int isign, int cb, int nrhs)
{
  DslashArgs a;
  memset(&a, 0, sizeof(a));
  a.geom = lat->geom();
  a.cb = cb;
  a.isign = isign;
  a.nrhs = nrhs;
  a.dir_mask = 0xFFu;
  a.coeff_s = p.aniso_s;
  a.coeff_t = p.aniso_t;
  a.coeff_t_edge = p.aniso_t * p.t_boundary;
  a.tbc_mask = 0;
  for (int d = 0; d < 4; d++) {
    a.tbc[d][0] = 1.0;
    a.tbc[d][1] = 0.0;
    if (p.use_tbc[d]) {
      a.tbc_mask |= 1 << d;
      a.tbc[d][0] = p.tbc_phases[d][0];
      a.tbc[d][1] = p.tbc_phases[d][1];
    }
  }
  a.post = POST_STORE;
  return a;
}

namespace {
// scoped solver temporary taken from (and returned to) the lattice's pool;
// pool fields are allocated once and carry no lattice reference
struct Tmp {
  qphix_gpu_field f = nullptr;
  qphix_gpu_lattice_s *lat;
  Tmp(qphix_gpu_lattice_s *l, int prec, int nrhs) : lat(l)
  {
    for (size_t i = lat->pool_free.size(); i-- > 0;) {
      auto *c = lat->pool_free[i];
      if (c->prec == prec && c->nrhs == nrhs) {
        f = c;
        lat->pool_free.erase(lat->pool_free.begin() + i);
        return;
      }
    }
    int rc = qphix_gpu_field_create(lat, QPHIX_GPU_SPINOR, prec, 0, nrhs, &f);
    if (rc) throw Error(rc, g_last_error);
    lat->refs--;  // owned by the pool, freed with the lattice
    lat->pool_all.push_back(f);
  }
  ~Tmp() { lat->pool_free.push_back(f); }
  Tmp(const Tmp &) = delete;
  Tmp &operator=(const Tmp &) = delete;
  operator qphix_gpu_field_s *() const { return f; }
};

}  // namespace

// ---- Dslash launch shapes and their autotuner ------------------------------
// A shape (right-hand sides per thread R, sites per thread SP) is chosen per
// (precision, links, epilogue, lattice, nrhs) the first time that Dslash runs
// outside stream capture: every built shape is timed on a scratch output
// (one warm-up and three timed launches each, CUDA events on the lattice's
// stream) and the fastest is kept for the life of the process.  Launches
// that differ only in their fused solver updates or reductions share the
// entry.  QPHIX_GPU_TUNE=0 (or qphix_gpu_tune_enable(0)) switches timing off
// and uses the default shape; QPHIX_GPU_RHS_TILE / QPHIX_GPU_SITES_PER_THREAD
// force R / SP where that shape is built.
namespace {
struct TuneEntry {
  DslashShape sh;
  float us = 0.f;
  int candidates = 0;
};
std::mutex g_tune_mu;
std::map<std::string, TuneEntry> g_tune;
std::atomic<int> g_tune_on{-1};

bool tune_enabled()
{
  int v = g_tune_on.load();
  if (v < 0) {
    const char *e = getenv("QPHIX_GPU_TUNE");
    v = (e && atoi(e) == 0) ? 0 : 1;
    g_tune_on = v;
  }
  return v != 0;
}

dim3 dslash_grid(const qphix_gpu_lattice_s *lat, const DslashShape &sh, int nrhs)
{
  long long per = (long long)QPX_BLOCK * (sh.rl ? 1 : sh.SP);
  long long nsb = (lat->vh + per - 1) / per;
  return dim3((unsigned)(nsb * (nrhs / (sh.rl ? 2 : sh.R))));
}

bool shape_built(int prec, int recon, int epi, int achi, const DslashShape &sh, int nrhs)
{
  if (nrhs % sh.R) return false;
  if (sh.rl && nrhs % 2) return false;
  return launch_dslash(prec, recon, epi, achi, sh, nullptr, dim3(1), nullptr);
}

DslashShape default_shape(int prec, bool gen)
{
  DslashShape sh;
  sh.gen = gen;
  // FP32 arithmetic: two sites per thread in float2 lanes (paired FP32 ops)
  if (!gen && prec != PREC_F64) sh.SP = 2;
  return sh;
}

// the fused reductions that are timed with a configuration (the CG update's
// |r|^2 goes with its post op, which is not replayed when tuning)
int tuned_reductions(const DslashArgs &a) { return a.red.mask & ~RED_NORM_R; }

std::string tune_key(const qphix_gpu_lattice_s *lat, int prec, int recon, int epi, int achi, int nrhs, int red)
{
  char buf[160];
  snprintf(buf, sizeof(buf), "dslash p%d r%d e%d a%d %dx%dx%dx%d n%d", prec, recon, epi, achi, lat->dims[0],
           lat->dims[1], lat->dims[2], lat->dims[3], nrhs);
  std::string k = buf;
  if (red) k += " red" + std::to_string(red);
  return k;
}
}  // namespace

static DslashShape choose_shape(qphix_gpu_lattice_s *lat, int prec, int recon, int epi, int achi,
                                const DslashArgs &a)
{
  const bool gen = a.dir_mask != 0xFFu || a.tbc_mask != 0 || a.halo;
  if (is_two_flavour(epi, achi)) {  // both flavours of a site in one thread
    QPX_REQUIRE(!gen, "two-flavour twisted mass takes all hops without twisted boundary phases");
    DslashShape sh;
    sh.R = 2;
    return sh;
  }
  if (gen) return default_shape(prec, true);
  // forced shapes (experiments and tests): QPHIX_GPU_RHS_LANES=1 selects two
  // right-hand sides in the float2 lanes of one site
  const char *fr = getenv("QPHIX_GPU_RHS_TILE"), *fs = getenv("QPHIX_GPU_SITES_PER_THREAD");
  const char *fl = getenv("QPHIX_GPU_RHS_LANES");
  if (fl && atoi(fl) == 1) {
    DslashShape sh;
    sh.SP = 2;
    sh.rl = true;
    if (shape_built(prec, recon, epi, achi, sh, a.nrhs)) return sh;
  } else if (fr || fs) {
    DslashShape sh = default_shape(prec, false);
    if (fr) sh.R = atoi(fr);
    if (fs) sh.SP = atoi(fs);
    if (sh.R == 2 && !fs) sh.SP = 1;
    if (sh.R >= 1 && sh.SP >= 1 && shape_built(prec, recon, epi, achi, sh, a.nrhs)) return sh;
  }
  std::vector<DslashShape> cands;
  for (int sp = 1; sp <= 2; sp++)
    for (int r = 1; r <= 2; r++) {
      DslashShape sh;
      sh.R = r;
      sh.SP = sp;
      if (shape_built(prec, recon, epi, achi, sh, a.nrhs)) cands.push_back(sh);
    }
  {
    DslashShape sh;
    sh.SP = 2;
    sh.rl = true;
    if (shape_built(prec, recon, epi, achi, sh, a.nrhs)) cands.push_back(sh);
  }
  if (cands.size() <= 1) return cands.empty() ? default_shape(prec, false) : cands[0];
  const int red = tuned_reductions(a);
  const std::string key = tune_key(lat, prec, recon, epi, achi, a.nrhs, red);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second.sh;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  QPX_CUDA(cudaStreamIsCapturing(lat->stream, &cap));
  if (!tune_enabled() || cap != cudaStreamCaptureStatusNone) return default_shape(prec, false);

  // time every candidate writing a scratch field, with the configuration's
  // reductions (into the lattice's workspace) but no finalize, no fused
  // solver update and no solver state
  Tmp scratch(lat, prec, a.nrhs);
  DslashArgs t = a;
  t.out = static_cast<qphix_gpu_field_s *>(scratch)->sarg();
  t.post = POST_STORE;
  t.state = nullptr;
  t.red.mask = red;
  t.red.nval = red_nval(red);
  t.red.fin = FIN_NONE;
  t.red.partials = lat->partials;
  t.red.result = lat->result;
  cudaEvent_t e0, e1;
  QPX_CUDA(cudaEventCreate(&e0));
  QPX_CUDA(cudaEventCreate(&e1));
  TuneEntry best;
  best.us = 1e30f;
  best.candidates = (int)cands.size();
  struct PdlOff {
    PdlOff() { pdl_suspended() = true; }
    ~PdlOff() { pdl_suspended() = false; }
  } pdl_off;
  for (const auto &sh : cands) {
    dim3 grid = dslash_grid(lat, sh, a.nrhs);
    // a reducing launch is timed with the fold of its partials
    auto once = [&] {
      launch_dslash(prec, recon, epi, achi, sh, &t, grid, lat->stream);
      check_launch();
      if (red) {
        launch_fold(t.red, nullptr, a.nrhs, (int)(grid.x / (a.nrhs / (sh.rl ? 2 : sh.R))), lat->stream);
        check_launch();
      }
    };
    once();
    cudaEventRecord(e0, lat->stream);
    for (int i = 0; i < 3; i++) once();
    cudaEventRecord(e1, lat->stream);
    QPX_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    QPX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const float us = ms * 1000.f / 3.f;
    if (us < best.us) {
      best.us = us;
      best.sh = sh;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[key] = best;
  return best.sh;
}

extern "C" int qphix_gpu_tune_enable(int enable)
{
  return guard([&] { g_tune_on = enable ? 1 : 0; });
}

extern "C" int qphix_gpu_tune_entries(int *count)
{
  return guard([&] {
    QPX_REQUIRE(count, "null argument");
    std::lock_guard<std::mutex> g(g_tune_mu);
    *count = (int)g_tune.size();
  });
}

extern "C" int qphix_gpu_tune_entry(int index, char *key, size_t key_len, int *rhs_tile, int *sites_per_thread,
                                    double *launch_us)
{
  return guard([&] {
    std::lock_guard<std::mutex> g(g_tune_mu);
    QPX_REQUIRE(index >= 0 && index < (int)g_tune.size(), "tune entry index out of range");
    auto it = g_tune.begin();
    std::advance(it, index);
    if (key && key_len) snprintf(key, key_len, "%s", it->first.c_str());
    // the rhs-lanes shape reads as two right-hand sides on 0 sites per thread
    if (rhs_tile) *rhs_tile = it->second.sh.rl ? 2 : it->second.sh.R;
    if (sites_per_thread) *sites_per_thread = it->second.sh.rl ? 0 : it->second.sh.SP;
    if (launch_us) *launch_us = it->second.us;
  });
}

static void set_reduce(DslashArgs &a, qphix_gpu_lattice_s *lat, int mask, int fin, SolverState *st)
{
  a.red.mask = mask;
  a.red.nval = red_nval(mask);
  a.red.fin = fin;
  a.red.partials = lat->partials;
  a.red.result = lat->result;
  a.state = st;
}

// While set (on this thread), Dslash launches are recorded instead of issued:
// the persistent solvers take the arguments of one iteration's launches from
// the regular code path and run them inside their own kernel.
struct CapturedDslash {
  int prec, recon, epi, achi;
  DslashArgs a;
};
static thread_local std::vector<CapturedDslash> *g_dslash_capture = nullptr;

static void dslash_launch(qphix_gpu_lattice_s *lat, int prec, int recon, int epi, int achi, DslashArgs &a)
{
  if (g_dslash_capture) {
    if (a.red.mask) {
      a.red.partials = lat->partials;
      a.red.result = lat->result;
      a.red.nval = red_nval(a.red.mask);
    }
    g_dslash_capture->push_back(CapturedDslash{prec, recon, epi, achi, a});
    return;
  }
  DslashShape sh = choose_shape(lat, prec, recon, epi, achi, a);
  if (a.red.mask) {
    a.red.partials = lat->partials;
    a.red.result = lat->result;
    a.red.nval = red_nval(a.red.mask);
  }
  const dim3 grid = dslash_grid(lat, sh, a.nrhs);
  if (!launch_dslash(prec, recon, epi, achi, sh, &a, grid, lat->stream))
    throw Error(QPHIX_GPU_EINVAL, "no Dslash kernel built for this precision / link / shape combination");
  check_launch();
  if (a.red.mask) {  // the blocks' partials: one per (site block, rhs, value)
    const int ntiles = a.nrhs / (sh.rl ? 2 : sh.R);
    launch_fold(a.red, a.state, a.nrhs, (int)(grid.x / ntiles), lat->stream);
    check_launch();
  }
}

static void require_spinor(const qphix_gpu_field_s *f, const char *what)
{
  if (!f || f->kind != QPHIX_GPU_SPINOR) throw Error(QPHIX_GPU_EINVAL, std::string(what) + " must be a spinor field");
}

// Fields combine if their lattices have the same shape (a field of one
// lattice object, e.g. a resident gauge field, can serve operators whose
// work runs on another lattice object's stream and workspace).
static bool same_shape(const qphix_gpu_lattice_s *a, const qphix_gpu_lattice_s *b)
{
  return a == b || (a->dims[0] == b->dims[0] && a->dims[1] == b->dims[1] && a->dims[2] == b->dims[2] &&
                    a->dims[3] == b->dims[3]);
}

static void require_same(const qphix_gpu_field_s *a, const qphix_gpu_field_s *b)
{
  if (!same_shape(a->lat, b->lat)) throw Error(QPHIX_GPU_EINVAL, "fields belong to lattices of different shape");
  if (a->prec != b->prec) throw Error(QPHIX_GPU_EINVAL, "fields have different precisions");
}

static void tm_derived(const qphix_gpu_op_params &p, double &dmu, double &dmu_inv)
{
  // include/qphix/tm_dslash_body.h:32-34
  double alpha = 4.0 + p.mass;
  dmu = p.twisted_mass / alpha;
  dmu_inv = alpha / (p.twisted_mass * p.twisted_mass + alpha * alpha);
}

// res = EPI(D psi) on checkerboard cb
// ---- halo mode ---------------------------------------------------------------
// t slabs (qphix_gpu_halo_faces) are the cut {t} of the general mode.
struct HaloSpec {
  int cut = 0;
  const void *psi_fwd[4] = {}, *psi_bwd[4] = {}, *links_bwd[4] = {};
  int global_first_t = 0, global_last_t = 0;
};

static size_t face_sites(const qphix_gpu_lattice_s *lat) { return (size_t)lat->nxh * lat->dims[1] * lat->dims[2]; }

// sites of one checkerboard of a slice along mu
static size_t face_sites_dir(const qphix_gpu_lattice_s *lat, int mu)
{
  const size_t nxh = lat->nxh, ny = lat->dims[1], nz = lat->dims[2], nt = lat->dims[3];
  switch (mu) {
  case 0: return ny * nz * nt / 2;
  case 1: return nxh * nz * nt;
  case 2: return nxh * ny * nt;
  default: return nxh * ny * nz;
  }
}

static size_t halo_spinor_bytes(const qphix_gpu_field_s *f, int mu = 3)
{
  const size_t face = face_sites_dir(f->lat, mu);
  return (size_t)f->nrhs * face * ((size_t)f->spec.nchunk * f->spec.chunk_bytes + (f->norm ? sizeof(float) : 0));
}

static size_t halo_link_bytes(const qphix_gpu_field_s *g, int mu = 3)
{
  return 2 * face_sites_dir(g->lat, mu) * (size_t)g->spec.nchunk * g->spec.chunk_bytes;
}

// a cut along mu needs an even local extent along mu (block offsets even, so
// local and global checkerboards agree) and, for x, an even Ny (x faces take
// every other y)
static void require_face_extents(const qphix_gpu_lattice_s *lat, int mu)
{
  QPX_REQUIRE(lat->dims[mu] % 2 == 0, "halo mode needs an even local extent along every cut direction");
  QPX_REQUIRE(mu != 0 || lat->dims[1] % 2 == 0, "a cut along x needs an even local Ny");
}

// the ghost-face arguments of a halo-mode launch hopping field psi with links gauge
static void set_halo(DslashArgs &a, const qphix_gpu_op_params &p, const qphix_gpu_field_s *psi,
                     const qphix_gpu_field_s *gauge, int cb, const HaloSpec &h)
{
  QPX_REQUIRE(h.cut > 0 && h.cut < 16, "halo: the cut mask takes bits 0-3 (x, y, z, t)");
  QPX_REQUIRE(a.tbc_mask == 0, "halo mode takes no twisted boundary phases");
  const auto *lat = psi->lat;
  for (int mu = 0; mu < 4; mu++) {
    if (!((h.cut >> mu) & 1)) continue;
    require_face_extents(lat, mu);
    QPX_REQUIRE(h.psi_fwd[mu] && h.psi_bwd[mu] && h.links_bwd[mu], "halo faces: null buffer");
    const long long face = (long long)face_sites_dir(lat, mu);
    QPX_REQUIRE(face % 4 == 0, "halo mode needs every face size divisible by 4");
    auto ghost = [&](const void *buf) {
      SpinorArg g;
      g.data = const_cast<void *>(buf);
      g.stride = face;
      g.rhs_stride_chunks = (long long)psi->spec.nchunk * face;
      g.norm = psi->norm ? reinterpret_cast<float *>(static_cast<char *>(g.data) +
                                                     (size_t)psi->nrhs * face * psi->spec.nchunk *
                                                         psi->spec.chunk_bytes)
                         : nullptr;
      return g;
    };
    a.ghost_fwd[mu] = ghost(h.psi_fwd[mu]);
    a.ghost_bwd[mu] = ghost(h.psi_bwd[mu]);
    // the backward hop onto checkerboard cb reads U_mu of the other checkerboard
    a.ghost_link[mu].data = static_cast<const char *>(h.links_bwd[mu]) +
                            (size_t)(1 - cb) * face * gauge->spec.nchunk * gauge->spec.chunk_bytes;
    a.ghost_link[mu].stride = face;
    a.ghost_link[mu].mu_stride = (long long)gauge->spec.nchunk * face;
  }
  a.halo = h.cut;
  // without a t cut the block holds both global t edges
  const bool tcut = (h.cut >> 3) & 1;
  a.coeff_t_edge = p.aniso_t * ((!tcut || h.global_last_t) ? p.t_boundary : 1.0);
  a.coeff_t_bwd_edge = p.aniso_t * ((!tcut || h.global_first_t) ? p.t_boundary : 1.0);
}

static HaloSpec halo_of(const qphix_gpu_halo_faces &f)
{
  HaloSpec h;
  h.cut = 8;
  h.psi_fwd[3] = f.psi_fwd;
  h.psi_bwd[3] = f.psi_bwd;
  h.links_bwd[3] = f.links_bwd;
  h.global_first_t = f.global_first;
  h.global_last_t = f.global_last;
  return h;
}

static HaloSpec halo_of(const qphix_gpu_halo_faces4 &f)
{
  HaloSpec h;
  h.cut = f.cut;
  for (int mu = 0; mu < 4; mu++) {
    h.psi_fwd[mu] = f.psi_fwd[mu];
    h.psi_bwd[mu] = f.psi_bwd[mu];
    h.links_bwd[mu] = f.links_bwd[mu];
  }
  h.global_first_t = f.global_first_t;
  h.global_last_t = f.global_last_t;
  return h;
}

extern "C" int qphix_gpu_halo_face_sites(qphix_gpu_lattice lat, int mu, size_t *sites)
{
  return guard([&] {
    QPX_REQUIRE(lat && sites, "null argument");
    QPX_REQUIRE(mu >= 0 && mu < 4, "mu must be in [0, 4)");
    *sites = face_sites_dir(lat, mu);
  });
}

extern "C" int qphix_gpu_halo_spinor_bytes_dir(qphix_gpu_field psi, int mu, size_t *bytes)
{
  return guard([&] {
    QPX_REQUIRE(psi && bytes, "null argument");
    require_spinor(psi, "psi");
    QPX_REQUIRE(mu >= 0 && mu < 4, "mu must be in [0, 4)");
    *bytes = halo_spinor_bytes(psi, mu);
  });
}

extern "C" int qphix_gpu_halo_link_bytes_dir(qphix_gpu_field gauge, int mu, size_t *bytes)
{
  return guard([&] {
    QPX_REQUIRE(gauge && bytes && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
    QPX_REQUIRE(mu >= 0 && mu < 4, "mu must be in [0, 4)");
    *bytes = halo_link_bytes(gauge, mu);
  });
}

// [rhs][chunk][face] rows, then [rhs][face] norms
extern "C" int qphix_gpu_halo_pack_spinor_dir(qphix_gpu_field psi, int mu, int side, int cb, void *dst)
{
  return guard([&] {
    QPX_REQUIRE(psi && dst, "null argument");
    require_spinor(psi, "psi");
    QPX_REQUIRE(mu >= 0 && mu < 4, "mu must be in [0, 4)");
    QPX_REQUIRE(side == 0 || side == 1, "side must be 0 (first slice) or 1 (last slice)");
    QPX_REQUIRE(cb == 0 || cb == 1, "cb must be 0 or 1");
    auto *lat = psi->lat;
    require_face_extents(lat, mu);
    const long long face = (long long)face_sites_dir(lat, mu);
    const int rows = psi->nrhs * psi->spec.nchunk;
    float *ndst = psi->norm ? reinterpret_cast<float *>(static_cast<char *>(dst) +
                                                        (size_t)rows * face * psi->spec.chunk_bytes)
                            : nullptr;
    launch_face_pack(lat->geom(), mu, side ? lat->dims[mu] - 1 : 0, cb, psi->data, lat->stride, rows,
                     psi->spec.chunk_bytes, face, dst, psi->norm, ndst, psi->nrhs, lat->stream);
    check_launch();
  });
}

// U_mu on the last slice along mu, checkerboard 0 then 1, [chunk][face] rows each
extern "C" int qphix_gpu_halo_pack_links_dir(qphix_gpu_field gauge, int mu, void *dst)
{
  return guard([&] {
    QPX_REQUIRE(gauge && dst && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
    QPX_REQUIRE(mu >= 0 && mu < 4, "mu must be in [0, 4)");
    auto *lat = gauge->lat;
    require_face_extents(lat, mu);
    const long long face = (long long)face_sites_dir(lat, mu);
    const size_t cbytes = gauge->spec.chunk_bytes, nch = gauge->spec.nchunk;
    const size_t mu_stride = nch * lat->stride;
    for (int c = 0; c < 2; c++)
      launch_face_pack(lat->geom(), mu, lat->dims[mu] - 1, c,
                       static_cast<const char *>(gauge->data) + (c * 4 + mu) * mu_stride * cbytes, lat->stride,
                       (int)nch, (int)cbytes, face, static_cast<char *>(dst) + c * nch * face * cbytes, nullptr,
                       nullptr, 0, lat->stream);
    check_launch();
  });
}

extern "C" int qphix_gpu_halo_spinor_bytes(qphix_gpu_field psi, size_t *bytes)
{
  return guard([&] {
    QPX_REQUIRE(psi && bytes, "null argument");
    require_spinor(psi, "psi");
    *bytes = halo_spinor_bytes(psi);
  });
}

extern "C" int qphix_gpu_halo_link_bytes(qphix_gpu_field gauge, size_t *bytes)
{
  return guard([&] {
    QPX_REQUIRE(gauge && bytes && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
    *bytes = halo_link_bytes(gauge);
  });
}

// [rhs][chunk][face] rows, then [rhs][face] norms: one strided copy each
extern "C" int qphix_gpu_halo_pack_spinor(qphix_gpu_field psi, int side, void *dst)
{
  return guard([&] {
    QPX_REQUIRE(psi && dst, "null argument");
    require_spinor(psi, "psi");
    QPX_REQUIRE(side == 0 || side == 1, "side must be 0 (first slice) or 1 (last slice)");
    auto *lat = psi->lat;
    const size_t face = face_sites(lat), cbytes = psi->spec.chunk_bytes;
    const size_t s0 = side ? (size_t)(lat->dims[3] - 1) * face : 0;
    const size_t rows = (size_t)psi->nrhs * psi->spec.nchunk;
    QPX_CUDA(cudaMemcpy2DAsync(dst, face * cbytes, static_cast<const char *>(psi->data) + s0 * cbytes,
                               (size_t)lat->stride * cbytes, face * cbytes, rows, cudaMemcpyDeviceToDevice,
                               lat->stream));
    if (psi->norm)
      QPX_CUDA(cudaMemcpy2DAsync(static_cast<char *>(dst) + rows * face * cbytes, face * sizeof(float),
                                 psi->norm + s0, (size_t)lat->stride * sizeof(float), face * sizeof(float),
                                 (size_t)psi->nrhs, cudaMemcpyDeviceToDevice, lat->stream));
  });
}

// U_t on the last slice, checkerboard 0 then 1, [chunk][face] rows each
extern "C" int qphix_gpu_halo_pack_links(qphix_gpu_field gauge, void *dst)
{
  return guard([&] {
    QPX_REQUIRE(gauge && dst && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
    auto *lat = gauge->lat;
    const size_t face = face_sites(lat), cbytes = gauge->spec.chunk_bytes, nch = gauge->spec.nchunk;
    const size_t s0 = (size_t)(lat->dims[3] - 1) * face, mu_stride = nch * lat->stride;
    for (int c = 0; c < 2; c++)
      QPX_CUDA(cudaMemcpy2DAsync(static_cast<char *>(dst) + c * nch * face * cbytes, face * cbytes,
                                 static_cast<const char *>(gauge->data) + ((c * 4 + 3) * mu_stride + s0) * cbytes,
                                 (size_t)lat->stride * cbytes, face * cbytes, nch, cudaMemcpyDeviceToDevice,
                                 lat->stream));
  });
}

static void dslash_core(const qphix_gpu_op_params &p, qphix_gpu_field_s *res, qphix_gpu_field_s *psi,
                        qphix_gpu_field_s *gauge, qphix_gpu_field_s *aux, qphix_gpu_field_s *aux2, int isign,
                        int cb, unsigned dir_mask = 0xFFu, qphix_gpu_field_s *aux3 = nullptr,
                        const HaloSpec *faces = nullptr, SolverState *state = nullptr)
{
  require_spinor(res, "res");
  require_spinor(psi, "psi");
  QPX_REQUIRE(gauge && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
  require_same(res, psi);
  require_same(res, gauge);
  QPX_REQUIRE(res->nrhs == psi->nrhs, "rhs count mismatch");
  QPX_REQUIRE(res != psi, "res and psi must be different fields");
  QPX_REQUIRE(isign == 1 || isign == -1, "isign must be +1 or -1");
  QPX_REQUIRE(cb == 0 || cb == 1, "cb must be 0 or 1");
  auto *lat = res->lat;
  DslashArgs a = base_args(p, lat, isign, cb, res->nrhs);
  a.dir_mask = dir_mask;
  a.out = res->sarg();
  a.in = psi->sarg();
  a.gauge = gauge->garg();
  int epi = EPI_NONE;
  switch (p.kind) {
  case QPHIX_GPU_WILSON:
    break;
  case QPHIX_GPU_CLOVER_OP:
    QPX_REQUIRE(aux && aux->kind == QPHIX_GPU_CLOVER, "clover dslash needs A^-1 (clover field)");
    require_same(res, aux);
    a.clov = aux->carg();
    epi = EPI_CLOV;
    break;
  case QPHIX_GPU_TM:
    tm_derived(p, a.mu, a.mu_inv);
    epi = EPI_TMINV;
    break;
  case QPHIX_GPU_TMCLOVER: {
    qphix_gpu_field_s *f = (isign == 1) ? aux : aux2;  // tm_clov_dslash_body.h:352
    QPX_REQUIRE(f && f->kind == QPHIX_GPU_FULLCLOVER, "tm clover dslash needs the two full inverses");
    require_same(res, f);
    a.clov = f->carg();
    epi = EPI_FCLOV;
    break;
  }
  case QPHIX_GPU_NDTM: {  // include/qphix/ndtm_reuse_operator.h:76-96
    QPX_REQUIRE(res->nrhs % 2 == 0, "two-flavour fields hold an even number of right-hand sides (up, down pairs)");
    const double alpha = 4.0 + p.mass, mu = p.twisted_mass, eps = p.epsilon;
    const double mu_inv = 1.0 / (alpha * alpha + mu * mu - eps * eps);
    a.alpha = alpha * mu_inv;
    a.mu = -isign * mu * mu_inv;
    a.eps = eps * mu_inv;
    epi = EPI_NDTM;
    break;
  }
  case QPHIX_GPU_NDTMCLOVER: {  // include/qphix/ndtm_reuse_operator_clover.h:121-126
    QPX_REQUIRE(res->nrhs % 2 == 0, "two-flavour fields hold an even number of right-hand sides (up, down pairs)");
    QPX_REQUIRE(aux && aux2 && aux->kind == QPHIX_GPU_FULLCLOVER && aux2->kind == QPHIX_GPU_FULLCLOVER,
                "two-flavour clover dslash needs the two full flavour-diagonal inverses");
    QPX_REQUIRE(aux3 && aux3->kind == QPHIX_GPU_CLOVER, "two-flavour clover dslash needs the off-diagonal inverse");
    require_same(res, aux);
    require_same(res, aux2);
    require_same(res, aux3);
    // isign swaps the flavour-diagonal inverses (tm_clov_dslash_body.h:1193-1200)
    a.clov = (isign == 1 ? aux : aux2)->carg();
    a.clov2 = (isign == 1 ? aux2 : aux)->carg();
    a.clov3 = aux3->carg();
    epi = EPI_NDFCLOV;
    break;
  }
  default:
    throw Error(QPHIX_GPU_EINVAL, "bad operator kind");
  }
  if (faces) {
    QPX_REQUIRE(!is_two_flavour(epi, ACHI_NONE), "halo mode is not provided for the two-flavour operators");
    set_halo(a, p, psi, gauge, cb, *faces);
  }
  // inside a solver iteration: a state whose solve is done makes the launch
  // return at once (graph replays after convergence, before the host sees it)
  a.state = state;
  dslash_launch(lat, res->prec, gauge->recon, epi, ACHI_NONE, a);
}

// options for the second (achimbdpsi) kernel of an operator application
static const double *fetch_result(qphix_gpu_lattice_s *lat, int nrhs, int nval);

struct ApplyOpts {
  int post = POST_STORE;
  int red_mask = 0;
  int fin = FIN_NONE;
  SolverState *state = nullptr;
  const qphix_gpu_field_s *w = nullptr, *r = nullptr, *x = nullptr, *p = nullptr;
};

static void achi_core(const qphix_gpu_op_params &p, qphix_gpu_field_s *res, qphix_gpu_field_s *psi,
                      qphix_gpu_field_s *chi, qphix_gpu_field_s *gauge, qphix_gpu_field_s *aux, double alpha,
                      double beta, int isign, int cb, double musign, const ApplyOpts &o,
                      const HaloSpec *faces = nullptr)
{
  require_spinor(res, "res");
  require_spinor(psi, "psi");
  require_spinor(chi, "chi");
  QPX_REQUIRE(gauge && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
  require_same(res, psi);
  require_same(res, chi);
  require_same(res, gauge);
  QPX_REQUIRE(res->nrhs == psi->nrhs && res->nrhs == chi->nrhs, "rhs count mismatch");
  QPX_REQUIRE(res != psi, "res and psi must be different fields");
  QPX_REQUIRE(isign == 1 || isign == -1, "isign must be +1 or -1");
  QPX_REQUIRE(cb == 0 || cb == 1, "cb must be 0 or 1");
  auto *lat = res->lat;
  DslashArgs a = base_args(p, lat, isign, cb, res->nrhs);
  a.out = res->sarg();
  a.in = psi->sarg();
  a.chi = chi->sarg();
  a.gauge = gauge->garg();
  a.alpha = alpha;
  a.beta = beta;
  int achi = ACHI_ALPHA;
  switch (p.kind) {
  case QPHIX_GPU_WILSON:
    break;
  case QPHIX_GPU_CLOVER_OP:
  case QPHIX_GPU_TMCLOVER:
    QPX_REQUIRE(aux && aux->kind == QPHIX_GPU_CLOVER, "clover achimbdpsi needs the clover term A");
    require_same(res, aux);
    a.clov = aux->carg();
    a.rho = p.prec_mass_rho;
    achi = ACHI_CLOV;
    break;
  case QPHIX_GPU_TM: {
    double dmu, dmu_inv;
    tm_derived(p, dmu, dmu_inv);
    a.mu = musign * dmu;
    achi = ACHI_TM;
    break;
  }
  case QPHIX_GPU_NDTM:  // include/qphix/tm_dslash_body.h:1174-1207
    QPX_REQUIRE(res->nrhs % 2 == 0, "two-flavour fields hold an even number of right-hand sides (up, down pairs)");
    a.mu = p.twisted_mass / (4.0 + p.mass);
    a.eps = p.epsilon;
    achi = ACHI_NDTM;
    break;
  case QPHIX_GPU_NDTMCLOVER:  // include/qphix/tm_clov_dslash_body.h:1345-1365
    QPX_REQUIRE(res->nrhs % 2 == 0, "two-flavour fields hold an even number of right-hand sides (up, down pairs)");
    QPX_REQUIRE(aux && aux->kind == QPHIX_GPU_CLOVER, "two-flavour clover achimbdpsi needs the clover term A");
    require_same(res, aux);
    a.clov = aux->carg();
    a.rho = p.twisted_mass;  // the up flavour's; the down flavour's is -rho (:983)
    a.eps = p.epsilon;
    achi = ACHI_NDCLOV;
    break;
  default:
    throw Error(QPHIX_GPU_EINVAL, "bad operator kind");
  }
  if (faces) {
    QPX_REQUIRE(!is_two_flavour(EPI_NONE, achi), "halo mode is not provided for the two-flavour operators");
    QPX_REQUIRE(!o.red_mask && o.post == POST_STORE, "halo launches take no fused solver updates");
    set_halo(a, p, psi, gauge, cb, *faces);
  }
  a.post = o.post;
  if (o.w) a.w = o.w->sarg();
  if (o.r) a.r = o.r->sarg();
  if (o.x) a.x = o.x->sarg();
  if (o.p) a.p = o.p->sarg();
  a.state = o.state;
  if (o.red_mask) set_reduce(a, lat, o.red_mask, o.fin, o.state);
  dslash_launch(lat, res->prec, gauge->recon, EPI_NONE, achi, a);
}

static qphix_gpu_op_params wilson_params_of(const qphix_gpu_op_params &p)
{
  qphix_gpu_op_params q = p;
  q.kind = QPHIX_GPU_WILSON;
  return q;
}

extern "C" int qphix_gpu_dslash(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                qphix_gpu_field gauge, qphix_gpu_field aux, qphix_gpu_field aux2, int isign, int cb)
{
  return guard([&] {
    QPX_REQUIRE(p, "null params");
    QPX_REQUIRE(p->kind != QPHIX_GPU_NDTMCLOVER, "the two-flavour clover hop is qphix_gpu_dslash_two_flav_clover");
    dslash_core(*p, res, psi, gauge, aux, aux2, isign, cb);
  });
}

extern "C" int qphix_gpu_dslash_two_flav_clover(const qphix_gpu_op_params *p, qphix_gpu_field res,
                                                qphix_gpu_field psi, qphix_gpu_field gauge,
                                                qphix_gpu_field finv_up, qphix_gpu_field finv_dn,
                                                qphix_gpu_field clov_odiag, int isign, int cb)
{
  return guard([&] {
    QPX_REQUIRE(p, "null params");
    qphix_gpu_op_params q = *p;
    q.kind = QPHIX_GPU_NDTMCLOVER;
    dslash_core(q, res, psi, gauge, finv_up, finv_dn, isign, cb, 0xFFu, clov_odiag);
  });
}

extern "C" int qphix_gpu_dslash_achimbdpsi(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                           qphix_gpu_field chi, qphix_gpu_field gauge, qphix_gpu_field aux,
                                           double alpha, double beta, int isign, int cb, double musign)
{
  return guard([&] {
    QPX_REQUIRE(p, "null params");
    achi_core(*p, res, psi, chi, gauge, aux, alpha, beta, isign, cb, musign, ApplyOpts());
  });
}

extern "C" int qphix_gpu_dslash_achimbdpsi_norms(const qphix_gpu_op_params *p, qphix_gpu_field res,
                                                 qphix_gpu_field psi, qphix_gpu_field chi, qphix_gpu_field gauge,
                                                 qphix_gpu_field aux, double alpha, double beta, int isign, int cb,
                                                 double musign, qphix_gpu_field w, double *out)
{
  return guard([&] {
    QPX_REQUIRE(p, "null params");
    if (w) {
      require_spinor(w, "w");
      require_same(res, w);
      QPX_REQUIRE(w->nrhs == res->nrhs, "rhs count mismatch");
    }
    ApplyOpts o;
    o.red_mask = RED_NORM_OUT | RED_DOT_OUT_CHI | (w ? RED_DOT_W_OUT : 0);
    o.fin = FIN_NONE;
    o.w = w;
    achi_core(*p, res, psi, chi, gauge, aux, alpha, beta, isign, cb, musign, o);
    if (out) {
      const int nval = red_nval(o.red_mask);
      const double *h = fetch_result(res->lat, res->nrhs, nval);
      for (int i = 0; i < res->nrhs * nval; i++) out[i] = h[i];
    }
  });
}

extern "C" int qphix_gpu_dslash_halo(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                     qphix_gpu_field gauge, qphix_gpu_field aux, qphix_gpu_field aux2, int isign,
                                     int cb, const qphix_gpu_halo_faces *faces)
{
  return guard([&] {
    QPX_REQUIRE(p && faces, "null argument");
    const HaloSpec h = halo_of(*faces);
    dslash_core(*p, res, psi, gauge, aux, aux2, isign, cb, 0xFFu, nullptr, &h);
  });
}

extern "C" int qphix_gpu_dslash_halo4(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                      qphix_gpu_field gauge, qphix_gpu_field aux, qphix_gpu_field aux2, int isign,
                                      int cb, const qphix_gpu_halo_faces4 *faces)
{
  return guard([&] {
    QPX_REQUIRE(p && faces, "null argument");
    const HaloSpec h = halo_of(*faces);
    dslash_core(*p, res, psi, gauge, aux, aux2, isign, cb, 0xFFu, nullptr, &h);
  });
}

extern "C" int qphix_gpu_dslash_achimbdpsi_halo(const qphix_gpu_op_params *p, qphix_gpu_field res,
                                                qphix_gpu_field psi, qphix_gpu_field chi, qphix_gpu_field gauge,
                                                qphix_gpu_field aux, double alpha, double beta, int isign, int cb,
                                                double musign, const qphix_gpu_halo_faces *faces)
{
  return guard([&] {
    QPX_REQUIRE(p && faces, "null argument");
    const HaloSpec h = halo_of(*faces);
    achi_core(*p, res, psi, chi, gauge, aux, alpha, beta, isign, cb, musign, ApplyOpts(), &h);
  });
}

extern "C" int qphix_gpu_dslash_achimbdpsi_halo4(const qphix_gpu_op_params *p, qphix_gpu_field res,
                                                 qphix_gpu_field psi, qphix_gpu_field chi, qphix_gpu_field gauge,
                                                 qphix_gpu_field aux, double alpha, double beta, int isign, int cb,
                                                 double musign, const qphix_gpu_halo_faces4 *faces)
{
  return guard([&] {
    QPX_REQUIRE(p && faces, "null argument");
    const HaloSpec h = halo_of(*faces);
    achi_core(*p, res, psi, chi, gauge, aux, alpha, beta, isign, cb, musign, ApplyOpts(), &h);
  });
}

extern "C" int qphix_gpu_dslash_dir(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                    qphix_gpu_field gauge, int cb, int dir)
{
  return guard([&] {
    QPX_REQUIRE(p, "null params");
    QPX_REQUIRE(dir >= 0 && dir < 8, "dir must be in [0, 8)");
    // include/qphix/dslash_body.h:1075-1157: isign +1; dir = 2 mu (+0) takes
    // the forward-neighbour hop, 2 mu + 1 the backward one
    int mu = dir / 2;
    unsigned bit = (dir % 2 == 0) ? (1u << (2 * mu + 1)) : (1u << (2 * mu));
    dslash_core(wilson_params_of(*p), res, psi, gauge, nullptr, nullptr, 1, cb, bit);
  });
}

extern "C" int qphix_gpu_clover_apply(qphix_gpu_field res, qphix_gpu_field chi, qphix_gpu_field clov)
{
  return guard([&] {
    require_spinor(res, "res");
    require_spinor(chi, "chi");
    QPX_REQUIRE(clov && clov->kind == QPHIX_GPU_CLOVER, "clov must be a clover field");
    require_same(res, chi);
    require_same(res, clov);
    QPX_REQUIRE(res->nrhs == chi->nrhs, "rhs count mismatch");
    // A chi = the clover achimbdpsi kernel with beta = 0, rho = 0 and no hops
    auto *lat = res->lat;
    qphix_gpu_op_params p{};
    p.kind = QPHIX_GPU_CLOVER_OP;
    p.aniso_s = p.aniso_t = 1.0;
    p.t_boundary = 1.0;
    DslashArgs a = base_args(p, lat, 1, 0, res->nrhs);
    a.dir_mask = 0;
    a.out = res->sarg();
    a.in = chi->sarg();
    a.chi = chi->sarg();
    a.clov = clov->carg();
    a.beta = 0.0;
    a.rho = 0.0;
    // dir_mask = 0 means no gauge access: any recon is fine
    a.gauge.data = nullptr;
    dslash_launch(lat, res->prec, 18, EPI_NONE, ACHI_CLOV, a);
  });
}

// ===========================================================================
// clover term construction / inversion on the device (clover_build.cu)
// ===========================================================================
extern "C" int qphix_gpu_clover_build(qphix_gpu_field clov, qphix_gpu_field gauge, int cb, double diag_mass,
                                      double csw_r, double csw_t)
{
  return guard([&] {
    QPX_REQUIRE(clov && clov->kind == QPHIX_GPU_CLOVER, "clov must be a clover field");
    QPX_REQUIRE(gauge && gauge->kind == QPHIX_GPU_GAUGE && gauge->prec == PREC_F64,
                "the clover term is built from an FP64 gauge field");
    QPX_REQUIRE(same_shape(clov->lat, gauge->lat), "fields belong to lattices of different shape");
    QPX_REQUIRE(cb == 0 || cb == 1, "cb must be 0 or 1");
    auto *lat = clov->lat;
    // tests/clover_term_qdp_w.h:133-137: the coefficients enter multiplied by 1/2
    launch_clover_build(gauge->recon, clov->prec, lat->geom(), gauge->garg(), clov->data, lat->stride, clov->spec.vpc,
                        cb, diag_mass, 0.5 * csw_r, 0.5 * csw_t, dim3((unsigned)((lat->vh + 63) / 64)), lat->stream);
    check_launch();
  });
}

extern "C" int qphix_gpu_clover_invert(qphix_gpu_field dst, qphix_gpu_field src)
{
  return guard([&] {
    QPX_REQUIRE(dst && src && dst->kind == QPHIX_GPU_CLOVER && src->kind == QPHIX_GPU_CLOVER,
                "dst and src must be clover fields");
    QPX_REQUIRE(same_shape(dst->lat, src->lat) && dst != src, "distinct fields of one lattice shape required");
    auto *lat = src->lat;
    launch_clover_invert(src->prec, dst->prec, lat->geom(), src->data, lat->stride, src->spec.vpc, dst->data, nullptr,
                         dst->spec.vpc, 0, 0.0, dim3((unsigned)((lat->vh + 63) / 64)), lat->stream);
    check_launch();
  });
}

extern "C" int qphix_gpu_two_flav_clover_apply(qphix_gpu_field res, qphix_gpu_field psi, qphix_gpu_field finv_up,
                                               qphix_gpu_field finv_dn, qphix_gpu_field clov_odiag, int isign)
{
  return guard([&] {
    require_spinor(res, "res");
    require_spinor(psi, "psi");
    require_same(res, psi);
    QPX_REQUIRE(res != psi, "res and psi must be different fields");
    QPX_REQUIRE(res->nrhs == psi->nrhs && psi->nrhs % 2 == 0, "two-flavour fields hold (up, down) pairs");
    QPX_REQUIRE(finv_up && finv_dn && finv_up->kind == QPHIX_GPU_FULLCLOVER && finv_dn->kind == QPHIX_GPU_FULLCLOVER,
                "the flavour-diagonal inverses must be full clover fields");
    QPX_REQUIRE(clov_odiag && clov_odiag->kind == QPHIX_GPU_CLOVER, "the off-diagonal inverse must be a clover field");
    require_same(res, finv_up);
    require_same(res, finv_dn);
    require_same(res, clov_odiag);
    QPX_REQUIRE(isign == 1 || isign == -1, "isign must be +1 or -1");
    auto *lat = res->lat;
    // isign swaps the flavour-diagonal inverses (tm_clov_dslash_body.h:1193-1200)
    const auto *fa = isign == 1 ? finv_up : finv_dn, *fb = isign == 1 ? finv_dn : finv_up;
    launch_two_flav_clover(res->prec, (int)lat->vh, res->nrhs / 2, res->sarg(), psi->sarg(), fa->carg(), fb->carg(),
                           clov_odiag->carg(), lat->stream);
    check_launch();
  });
}

extern "C" int qphix_gpu_clover_invert_ndtm(qphix_gpu_field finv_up, qphix_gpu_field finv_dn,
                                            qphix_gpu_field clov_odiag, qphix_gpu_field src, double mu, double eps)
{
  return guard([&] {
    QPX_REQUIRE(finv_up && finv_dn && clov_odiag && src, "null argument");
    QPX_REQUIRE(finv_up->kind == QPHIX_GPU_FULLCLOVER && finv_dn->kind == QPHIX_GPU_FULLCLOVER,
                "flavour-diagonal inverses must be full clover fields");
    QPX_REQUIRE(clov_odiag->kind == QPHIX_GPU_CLOVER && src->kind == QPHIX_GPU_CLOVER,
                "src and the off-diagonal inverse must be clover fields");
    QPX_REQUIRE(finv_up->prec == finv_dn->prec && finv_up->prec == clov_odiag->prec,
                "destinations must share a precision");
    QPX_REQUIRE(same_shape(finv_up->lat, src->lat) && same_shape(finv_dn->lat, src->lat) &&
                    same_shape(clov_odiag->lat, src->lat),
                "fields belong to lattices of different shape");
    QPX_REQUIRE(clov_odiag != src, "distinct fields required");
    auto *lat = src->lat;
    launch_clover_invert(src->prec, finv_up->prec, lat->geom(), src->data, lat->stride, src->spec.vpc,
                         finv_up->data, finv_dn->data, finv_up->spec.vpc, 2, mu,
                         dim3((unsigned)((lat->vh + 63) / 64)), lat->stream, clov_odiag->data, clov_odiag->spec.vpc,
                         eps);
    check_launch();
  });
}

extern "C" int qphix_gpu_clover_invert_twisted(qphix_gpu_field dst_plus, qphix_gpu_field dst_minus,
                                               qphix_gpu_field src, double mu)
{
  return guard([&] {
    QPX_REQUIRE(dst_plus && dst_minus && src, "null argument");
    QPX_REQUIRE(dst_plus->kind == QPHIX_GPU_FULLCLOVER && dst_minus->kind == QPHIX_GPU_FULLCLOVER,
                "destinations must be full clover fields");
    QPX_REQUIRE(src->kind == QPHIX_GPU_CLOVER, "src must be a clover field");
    QPX_REQUIRE(dst_plus->prec == dst_minus->prec, "destinations must share a precision");
    QPX_REQUIRE(same_shape(dst_plus->lat, src->lat) && same_shape(dst_minus->lat, src->lat),
                "fields belong to lattices of different shape");
    auto *lat = src->lat;
    launch_clover_invert(src->prec, dst_plus->prec, lat->geom(), src->data, lat->stride, src->spec.vpc,
                         dst_plus->data, dst_minus->data, dst_plus->spec.vpc, 1, mu,
                         dim3((unsigned)((lat->vh + 63) / 64)), lat->stream);
    check_launch();
  });
}

extern "C" int qphix_gpu_clover_convert(qphix_gpu_field dst, qphix_gpu_field src)
{
  return guard([&] {
    QPX_REQUIRE(dst && src && dst->kind == src->kind &&
                    (src->kind == QPHIX_GPU_CLOVER || src->kind == QPHIX_GPU_FULLCLOVER),
                "dst and src must be clover fields of the same kind");
    QPX_REQUIRE(same_shape(dst->lat, src->lat), "fields belong to lattices of different shape");
    auto *lat = dst->lat;
    launch_clover_convert(src->prec, dst->prec, lat->geom(), src->data, src->spec.vpc, dst->data, dst->spec.vpc,
                          lat->stride, src->kind == QPHIX_GPU_CLOVER ? 72 : 144, dim3(nblocks_for(lat->vh)),
                          lat->stream);
    check_launch();
  });
}

// ===========================================================================
// even-odd operators
// ===========================================================================
extern "C" int qphix_gpu_eo_op_create(const qphix_gpu_op_params *p, qphix_gpu_field gauge, qphix_gpu_field clov,
                                      qphix_gpu_field invclov, qphix_gpu_field finv0, qphix_gpu_field finv1,
                                      qphix_gpu_eo_op *out)
{
  return guard([&] {
    QPX_REQUIRE(p && out, "null argument");
    QPX_REQUIRE(gauge && gauge->kind == QPHIX_GPU_GAUGE, "gauge must be a gauge field");
    if (p->kind == QPHIX_GPU_CLOVER_OP) QPX_REQUIRE(clov && invclov, "clover operator needs clov and invclov");
    if (p->kind == QPHIX_GPU_TMCLOVER) QPX_REQUIRE(clov && finv0 && finv1, "tm clover operator needs clov, finv0/1");
    if (p->kind == QPHIX_GPU_NDTMCLOVER)
      QPX_REQUIRE(clov && invclov && finv0 && finv1,
                  "two-flavour clover operator needs clov, invclov (off-diagonal inverse) and finv0/1");
    auto *op = new qphix_gpu_eo_op_s();
    op->serial = g_serial++;
    op->p = *p;
    op->gauge = gauge;
    op->clov = clov;
    op->invclov = invclov;
    op->finv0 = finv0;
    op->finv1 = finv1;
    *out = op;
  });
}

extern "C" int qphix_gpu_eo_op_destroy(qphix_gpu_eo_op op)
{
  return guard([&] {
    if (!op) return;
    for (auto &kv : op->tmp) qphix_gpu_field_destroy(kv.second);
    delete op;
  });
}

// the operator's temporary, created on the lattice (stream) of the first
// field it is applied to
static qphix_gpu_field_s *op_tmp(qphix_gpu_eo_op_s *op, int nrhs, qphix_gpu_lattice_s *lat = nullptr)
{
  auto it = op->tmp.find(nrhs);
  if (it != op->tmp.end()) return it->second;
  qphix_gpu_field f = nullptr;
  int rc = qphix_gpu_field_create(lat ? lat : op->gauge->lat, QPHIX_GPU_SPINOR, op->gauge->prec, 0, nrhs, &f);
  if (rc) throw Error(rc, g_last_error);
  op->tmp[nrhs] = f;
  return f;
}

// M_oo in = [diag] in - beta D_{target,other} [inv-diag] D_{other,target} in
static void eo_apply(qphix_gpu_eo_op_s *op, qphix_gpu_field_s *res, qphix_gpu_field_s *in, int isign, int target_cb,
                     const ApplyOpts &o)
{
  require_spinor(in, "in");
  qphix_gpu_field_s *tmp = op_tmp(op, in->nrhs, in->lat);
  const auto &p = op->p;
  int other = 1 - target_cb;
  switch (p.kind) {
  case QPHIX_GPU_WILSON: {  // include/qphix/wilson.h:49-65
    double alpha = 4.0 + p.mass, beta = 0.25 / alpha;
    dslash_core(p, tmp, in, op->gauge, nullptr, nullptr, isign, other, 0xFFu, nullptr, nullptr, o.state);
    achi_core(p, res, tmp, in, op->gauge, nullptr, alpha, beta, isign, target_cb, 1.0, o);
    break;
  }
  case QPHIX_GPU_CLOVER_OP:  // include/qphix/clover.h:162-172
    dslash_core(p, tmp, in, op->gauge, op->invclov, nullptr, isign, other, 0xFFu, nullptr, nullptr, o.state);
    achi_core(p, res, tmp, in, op->gauge, op->clov, 0.0, 0.25, isign, target_cb, 1.0, o);
    break;
  case QPHIX_GPU_TM: {  // include/qphix/twisted_mass.h:62-77
    double alpha = 4.0 + p.mass;
    dslash_core(p, tmp, in, op->gauge, nullptr, nullptr, isign, other, 0xFFu, nullptr, nullptr, o.state);
    achi_core(p, res, tmp, in, op->gauge, nullptr, alpha, 0.25, isign, target_cb, 1.0, o);
    break;
  }
  case QPHIX_GPU_NDTM:  // include/qphix/ndtm_reuse_operator.h:68-110
    dslash_core(p, tmp, in, op->gauge, nullptr, nullptr, isign, other, 0xFFu, nullptr, nullptr, o.state);
    achi_core(p, res, tmp, in, op->gauge, nullptr, 4.0 + p.mass, 0.25, isign, target_cb, 1.0, o);
    break;
  case QPHIX_GPU_TMCLOVER:  // include/qphix/twisted_mass_clover.h:92-102
    dslash_core(p, tmp, in, op->gauge, op->finv0, op->finv1, isign, other, 0xFFu, nullptr, nullptr, o.state);
    achi_core(p, res, tmp, in, op->gauge, op->clov, 0.0, 0.25, isign, target_cb, 1.0, o);
    break;
  case QPHIX_GPU_NDTMCLOVER:  // include/qphix/ndtm_reuse_operator_clover.h:117-128
    dslash_core(p, tmp, in, op->gauge, op->finv0, op->finv1, isign, other, 0xFFu, op->invclov, nullptr,
                o.state);
    achi_core(p, res, tmp, in, op->gauge, op->clov, 0.0, 0.25, isign, target_cb, 1.0, o);
    break;
  default:
    throw Error(QPHIX_GPU_EINVAL, "bad operator kind");
  }
}

// Times the operator's Dslash shapes (autotuner) outside stream capture, on
// scratch fields, once per operator, nrhs and set of fused reductions: for an
// operator whose first applications would otherwise happen inside a captured
// solver iteration.  `opts` are the applications' options; their finalize
// steps and solver state are dropped (reductions land in the workspace only).
static void pretune_op(qphix_gpu_eo_op_s *op, qphix_gpu_lattice_s *lat, int nrhs, int isign, int cb,
                       std::vector<ApplyOpts> opts)
{
  if (!tune_enabled()) return;
  int tag = nrhs;
  for (size_t i = 0; i < opts.size(); i++) tag = tag * 64 + opts[i].red_mask;
  for (int n : op->pretuned)
    if (n == tag) return;
  // the input's values do not matter for timing (pool fields hold finite data)
  Tmp a(lat, op->gauge->prec, nrhs), b(lat, op->gauge->prec, nrhs);
  for (auto o : opts) {
    o.fin = FIN_NONE;
    o.state = nullptr;
    o.post = POST_STORE;
    eo_apply(op, b, a, isign, cb, o);
  }
  QPX_CUDA(cudaStreamSynchronize(lat->stream));
  op->pretuned.push_back(tag);
}

extern "C" int qphix_gpu_eo_op_apply(qphix_gpu_eo_op op, qphix_gpu_field res, qphix_gpu_field in, int isign,
                                     int target_cb)
{
  return guard([&] {
    QPX_REQUIRE(op, "null operator");
    eo_apply(op, res, in, isign, target_cb, ApplyOpts());
  });
}

// ===========================================================================
// BLAS
// ===========================================================================
static Coef cval(double re, double im = 0.0) { return Coef{re, im, nullptr, nullptr}; }
static Coef cslot(SolverState *st, int slot_re, int slot_im = -1)
{
  return Coef{0, 0, st->v[slot_re], slot_im >= 0 ? st->v[slot_im] : nullptr};
}

struct BlasCall {
  int op;
  const qphix_gpu_field_s *x = nullptr, *y = nullptr, *z = nullptr, *w = nullptr, *v = nullptr;
  Coef a{0, 0, nullptr, nullptr}, b{0, 0, nullptr, nullptr};
  int slots = 0;  // reduction slot set
  int fin = FIN_NONE;
  SolverState *state = nullptr;
};

// Site blocks of a BLAS launch: one site per thread.  (Four sites per thread
// on the 16^3x32, 8-rhs solve cut the following fold from 13.6 to 6.3 us but
// slowed the pass from 18.8 to 20.2 us, and the changed summation order
// moved the mixed solve's inner iteration count; the kernel takes any grid.)
static int blas_blocks(long long vh, int nrhs)
{
  (void)nrhs;
  return nblocks_for(vh);
}

static void blas_launch(qphix_gpu_lattice_s *lat, int prec, int nrhs, const BlasCall &c)
{
  BlasArgs a;
  memset(&a, 0, sizeof(a));
  a.op = c.op;
  a.vh = (int)lat->vh;
  a.nrhs = nrhs;
  if (c.x) a.x = c.x->sarg();
  if (c.y) a.y = c.y->sarg();
  if (c.z) a.z = c.z->sarg();
  if (c.w) a.w = c.w->sarg();
  if (c.v) a.v = c.v->sarg();
  a.a = c.a;
  a.b = c.b;
  a.state = c.state;
  if (c.slots) {
    a.red.mask = c.slots;
    a.red.nval = __builtin_popcount(c.slots);
    a.red.fin = c.fin;
    a.red.partials = lat->partials;
    a.red.result = lat->result;
  }
  const int nb = blas_blocks(lat->vh, nrhs);
  launch_blas(prec, a, dim3(nb, nrhs), lat->stream);
  check_launch();
  if (c.slots) {
    launch_fold(a.red, c.state, nrhs, nb, lat->stream);
    check_launch();
  }
}

// fetch the last reduction result (nrhs x nval) to the host
static const double *fetch_result(qphix_gpu_lattice_s *lat, int nrhs, int nval)
{
  QPX_CUDA(cudaMemcpyAsync(lat->h_result, lat->result, sizeof(double) * nrhs * nval, cudaMemcpyDeviceToHost,
                           lat->stream));
  QPX_CUDA(cudaStreamSynchronize(lat->stream));
  return lat->h_result;
}

static std::vector<double> norm2_host(const qphix_gpu_field_s *x)
{
  BlasCall c;
  c.op = B_NORM2;
  c.x = x;
  c.slots = 0x1;
  c.fin = FIN_NONE;
  blas_launch(x->lat, x->prec, x->nrhs, c);
  const double *r = fetch_result(x->lat, x->nrhs, 1);
  return std::vector<double>(r, r + x->nrhs);
}

extern "C" int qphix_gpu_blas_norm2(qphix_gpu_field x, double *out)
{
  return guard([&] {
    require_spinor(x, "x");
    QPX_REQUIRE(out, "null out");
    auto v = norm2_host(x);
    for (int r = 0; r < x->nrhs; r++) out[r] = v[r];
  });
}

extern "C" int qphix_gpu_blas_inner_product(qphix_gpu_field x, qphix_gpu_field y, double *out)
{
  return guard([&] {
    require_spinor(x, "x");
    require_spinor(y, "y");
    require_same(x, y);
    QPX_REQUIRE(out, "null out");
    BlasCall c;
    c.op = B_DOT;
    c.x = x;
    c.y = y;
    c.slots = 0x3;
    blas_launch(x->lat, x->prec, x->nrhs, c);
    const double *r = fetch_result(x->lat, x->nrhs, 2);
    for (int i = 0; i < 2 * x->nrhs; i++) out[i] = r[i];
  });
}

// y = a x + b y, out[r] = |y_r|^2 (axpyNorm2, include/qphix/blas_new_c.h:312-343)
extern "C" int qphix_gpu_blas_caxpby_norm2(const double a[2], qphix_gpu_field x, const double b[2],
                                           qphix_gpu_field y, double *out)
{
  return guard([&] {
    require_spinor(x, "x");
    require_spinor(y, "y");
    require_same(x, y);
    QPX_REQUIRE(a && b && out, "null argument");
    BlasCall c;
    c.op = B_CAXPBY_NORM;
    c.x = x;
    c.y = y;
    c.a = cval(a[0], a[1]);
    c.b = cval(b[0], b[1]);
    c.slots = 0x1;
    blas_launch(x->lat, x->prec, x->nrhs, c);
    const double *r = fetch_result(x->lat, x->nrhs, 1);
    for (int i = 0; i < x->nrhs; i++) out[i] = r[i];
  });
}

// z = x - y, out[r] = |z_r|^2 (xmyNorm2Spinor, blas_new_c.h:345-358; z may be y:
// xmy2Norm2Spinor, :360-395)
extern "C" int qphix_gpu_blas_xmy_norm2(qphix_gpu_field x, qphix_gpu_field y, qphix_gpu_field z, double *out)
{
  return guard([&] {
    require_spinor(x, "x");
    require_spinor(y, "y");
    require_spinor(z, "z");
    require_same(x, y);
    require_same(x, z);
    QPX_REQUIRE(out, "null out");
    BlasCall c;
    c.op = B_XMY_NORM;
    c.x = x;
    c.y = y;
    c.z = z;
    c.slots = 0x1;
    blas_launch(x->lat, x->prec, x->nrhs, c);
    const double *r = fetch_result(x->lat, x->nrhs, 1);
    for (int i = 0; i < x->nrhs; i++) out[i] = r[i];
  });
}

// out[3 r .. 3 r + 2] = Re <x, y>, Im <x, y>, |x|^2 (innerProductNorm, blas_new_c.h:573-625)
extern "C" int qphix_gpu_blas_inner_product_norm(qphix_gpu_field x, qphix_gpu_field y, double *out)
{
  return guard([&] {
    require_spinor(x, "x");
    require_spinor(y, "y");
    require_same(x, y);
    QPX_REQUIRE(out, "null out");
    BlasCall c;
    c.op = B_DOTNORM;
    c.x = x;
    c.y = y;
    c.slots = 0x7;
    blas_launch(x->lat, x->prec, x->nrhs, c);
    const double *r = fetch_result(x->lat, x->nrhs, 3);
    for (int i = 0; i < 3 * x->nrhs; i++) out[i] = r[i];
  });
}

extern "C" int qphix_gpu_blas_caxpby(const double a[2], qphix_gpu_field x, const double b[2], qphix_gpu_field y)
{
  return guard([&] {
    require_spinor(x, "x");
    require_spinor(y, "y");
    require_same(x, y);
    QPX_REQUIRE(a && b, "null coefficient");
    BlasCall c;
    c.op = B_CAXPBY;
    c.x = x;
    c.y = y;
    c.a = cval(a[0], a[1]);
    c.b = cval(b[0], b[1]);
    blas_launch(x->lat, x->prec, x->nrhs, c);
  });
}

extern "C" int qphix_gpu_blas_copy(qphix_gpu_field dst, qphix_gpu_field src)
{
  return guard([&] {
    require_spinor(dst, "dst");
    require_spinor(src, "src");
    QPX_REQUIRE(dst->nrhs == src->nrhs && dst->lat == src->lat, "shape mismatch");
    if (dst->prec == src->prec) {
      BlasCall c;
      c.op = B_COPY;
      c.x = src;
      c.y = dst;
      blas_launch(src->lat, src->prec, src->nrhs, c);
    } else {
      convert_field(dst, src, cval(1.0), nullptr);
    }
  });
}

extern "C" int qphix_gpu_blas_zero(qphix_gpu_field x)
{
  return guard([&] {
    require_spinor(x, "x");
    BlasCall c;
    c.op = B_ZERO;
    c.x = x;
    blas_launch(x->lat, x->prec, x->nrhs, c);
  });
}

// ===========================================================================
// solvers
// ===========================================================================
namespace {

std::string fkey(const qphix_gpu_field_s *f) { return f ? std::to_string(f->serial) : std::string("-"); }

// push the host copy of the solver state to the device
void state_upload(qphix_gpu_lattice_s *lat)
{
  QPX_CUDA(cudaMemcpyAsync(lat->state, lat->h_state, sizeof(SolverState), cudaMemcpyHostToDevice, lat->stream));
  QPX_CUDA(cudaStreamSynchronize(lat->stream));
}

void state_download(qphix_gpu_lattice_s *lat)
{
  QPX_CUDA(cudaMemcpyAsync(lat->h_state, lat->state, sizeof(SolverState), cudaMemcpyDeviceToHost, lat->stream));
  QPX_CUDA(cudaStreamSynchronize(lat->stream));
}

SolverState &state_reset(qphix_gpu_lattice_s *lat, int nrhs, int max_iter)
{
  SolverState &s = *lat->h_state;
  memset(&s, 0, sizeof(SolverState));
  s.nrhs = nrhs;
  s.max_iter = max_iter;
  return s;
}

// Replays `step` (one solver iteration, kernels only) until the device raises
// state->done.  The step is captured once into a CUDA graph.
// `key` names everything the captured launches depend on (solver, operator
// and field serial numbers, isign, cb); a graph captured under the same key
// is replayed instead of captured again.
template <typename Step>
void run_iterations(qphix_gpu_lattice_s *lat, Step &&step, int max_iter, const std::string &key)
{
  const int check = 8;
  bool use_graph = !env_flag("QPHIX_GPU_NO_GRAPH");
  cudaGraphExec_t exec = nullptr;
  unsigned long long nodes = 0;
  bool cached = false;
  if (use_graph && !key.empty()) {
    auto it = lat->graphs.find(key);
    if (it != lat->graphs.end()) {
      exec = it->second;
      nodes = lat->graph_nodes[key];
      cached = true;
    }
  }
  if (use_graph && !cached) {
    cudaGraph_t graph = nullptr;
    unsigned long long before = g_launches.load();
    QPX_CUDA(cudaStreamBeginCapture(lat->stream, cudaStreamCaptureModeThreadLocal));
    try {
      step();
    } catch (...) {
      cudaStreamEndCapture(lat->stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    QPX_CUDA(cudaStreamEndCapture(lat->stream, &graph));
    nodes = g_launches.load() - before;  // captured, not run: counted per replay below
    g_launches -= nodes;
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) throw Error(QPHIX_GPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    if (!key.empty()) {
      if (lat->graph_order.size() >= 64) {  // bounded cache: drop the oldest
        const std::string &old_key = lat->graph_order.front();
        cudaGraphExecDestroy(lat->graphs[old_key]);
        lat->graphs.erase(old_key);
        lat->graph_nodes.erase(old_key);
        lat->graph_order.erase(lat->graph_order.begin());
      }
      lat->graphs[key] = exec;
      lat->graph_nodes[key] = nodes;
      lat->graph_order.push_back(key);
      cached = true;
    }
  }
  int launched = 0;
  try {
    while (true) {
      for (int i = 0; i < check; i++) {
        if (use_graph) {
          QPX_CUDA(cudaGraphLaunch(exec, lat->stream));
          g_launches += nodes;
        } else
          step();
        launched++;
      }
      QPX_CUDA(cudaMemcpyAsync(&lat->h_state->done, &lat->state->done, sizeof(int), cudaMemcpyDeviceToHost,
                               lat->stream));
      QPX_CUDA(cudaStreamSynchronize(lat->stream));
      if (lat->h_state->done) break;
      if (launched > max_iter + 2 * check) break;  // the device enforces max_iter; belt and braces
    }
  } catch (...) {
    if (exec && !cached) cudaGraphExecDestroy(exec);
    throw;
  }
  if (exec && !cached) QPX_CUDA(cudaGraphExecDestroy(exec));
  state_download(lat);
}

double elapsed(cudaEvent_t a, cudaEvent_t b)
{
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms * 1e-3;
}

struct Timer {
  cudaEvent_t t0, t1;
  qphix_gpu_lattice_s *lat;
  explicit Timer(qphix_gpu_lattice_s *l) : lat(l)
  {
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, lat->stream);
  }
  double stop()
  {
    cudaEventRecord(t1, lat->stream);
    cudaEventSynchronize(t1);
    return elapsed(t0, t1);
  }
  ~Timer()
  {
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
  }
};

// An operator's fields may belong to other lattice objects of the same shape
// (a resident gauge field shared by many solves): their streams are
// synchronised once, so that the fields are complete before a solve's work,
// which all runs on the stream of x's lattice, reads them.
void sync_op_fields(const qphix_gpu_eo_op_s *op, const qphix_gpu_lattice_s *lat)
{
  const qphix_gpu_field_s *fs[5] = {op->gauge, op->clov, op->invclov, op->finv0, op->finv1};
  const qphix_gpu_lattice_s *done[5];
  int nd = 0;
  for (const auto *f : fs) {
    if (!f || f->lat == lat) continue;
    QPX_REQUIRE(same_shape(f->lat, lat), "operator fields belong to a lattice of different shape");
    bool seen = false;
    for (int i = 0; i < nd; i++) seen = seen || done[i] == f->lat;
    if (seen) continue;
    QPX_CUDA(cudaStreamSynchronize(f->lat->stream));
    done[nd++] = f->lat;
  }
}

static bool two_flavour_kind(int kind) { return kind == QPHIX_GPU_NDTM || kind == QPHIX_GPU_NDTMCLOVER; }

void check_solver_fields(qphix_gpu_eo_op_s *op, qphix_gpu_field_s *x, qphix_gpu_field_s *rhs,
                         bool two_flavour_ok = false)
{
  QPX_REQUIRE(op, "null operator");
  QPX_REQUIRE(two_flavour_ok || !two_flavour_kind(op->p.kind),
              "two-flavour operators are solved with CG (the flavour pair as one system)");
  require_spinor(x, "x");
  require_spinor(rhs, "rhs");
  require_same(x, rhs);
  require_same(x, op->gauge);
  QPX_REQUIRE(x->nrhs == rhs->nrhs, "rhs count mismatch");
  sync_op_fields(op, x->lat);
}

// true residual |b - M x|^2 per rhs (and relative), t: scratch
void true_residual(qphix_gpu_eo_op_s *op, qphix_gpu_field_s *x, qphix_gpu_field_s *rhs, qphix_gpu_field_s *t,
                   qphix_gpu_field_s *r, int isign, int cb, bool normal_eq, const std::vector<double> &bnorm,
                   std::vector<double> &abs2, std::vector<double> &rel)
{
  if (normal_eq) {
    eo_apply(op, r, x, isign, cb, ApplyOpts());
    eo_apply(op, t, r, -isign, cb, ApplyOpts());
  } else {
    eo_apply(op, t, x, isign, cb, ApplyOpts());
  }
  BlasCall c;
  c.op = B_XMY_NORM;
  c.x = rhs;
  c.y = t;
  c.z = r;
  c.slots = 0x1;
  blas_launch(x->lat, x->prec, x->nrhs, c);
  const double *h = fetch_result(x->lat, x->nrhs, 1);
  abs2.assign(h, h + x->nrhs);
  rel.resize(x->nrhs);
  for (int i = 0; i < x->nrhs; i++) rel[i] = bnorm[i] > 0 ? std::sqrt(abs2[i] / bnorm[i]) : 0.0;
}

// ---------------------------------------------------------------------------
// CG on M^dag M (include/qphix/invcg.h:88-456)
// two-flavour systems: the values of right-hand sides 2k and 2k+1 summed
void pair_sum(std::vector<double> &v)
{
  for (size_t r = 0; r + 1 < v.size(); r += 2) v[r] = v[r + 1] = v[r] + v[r + 1];
}

// ---------------------------------------------------------------------------
// Persistent-kernel CG (qpx_persist.cuh): the whole iteration loop in one
// cooperative launch, for lattices whose Dslash launches are too small to
// fill the GPU.  QPHIX_GPU_PERSISTENT=1 uses it wherever it is built (Wilson
// and clover operators, FP64 / FP32 storage, isign = +1, no twisted boundary
// phases) and Vh x nrhs stays within kPersistentSites; unset or 0, solves
// replay the captured iteration graph.  It is not the default: on B200 a
// grid barrier costs about as much as a kernel boundary of the graph
// (~2 us), and at 8^4 the graph replay measured slightly faster (0.98
// against 1.01 ms per FP64 Wilson CG solve).
constexpr long long kPersistentSites = 32768;

static bool persistent_cg_wanted(qphix_gpu_eo_op_s *op, qphix_gpu_lattice_s *lat, int prec, int nrhs, int isign,
                                 bool coupled)
{
  const char *e = std::getenv("QPHIX_GPU_PERSISTENT");
  const int mode = (e && *e) ? std::atoi(e) : -1;
  if (mode != 1 || coupled || isign != 1) return false;
  if (prec != PREC_F64 && prec != PREC_F32) return false;
  if (op->p.kind != QPHIX_GPU_WILSON && op->p.kind != QPHIX_GPU_CLOVER_OP) return false;
  if (op->gauge->recon != 12 && op->gauge->recon != 18) return false;
  return lat->vh * nrhs <= kPersistentSites;
}

// Runs the iterations of solve_cg from the state already on the device, with
// the four Dslash launches of one iteration as captured; false when the
// launches need the general Dslash path (twisted phases, direction masks,
// halo faces) or the device cannot hold a block of the kernel, and the caller
// iterates with the captured graph instead.
static bool run_cg_persistent(qphix_gpu_lattice_s *lat, const std::vector<CapturedDslash> &cap,
                              qphix_gpu_field_s *r, qphix_gpu_field_s *p, int nrhs)
{
  if (cap.size() != 4) return false;
  for (const auto &c : cap)
    if (c.a.tbc_mask || c.a.dir_mask != 0xFFu || c.a.halo) return false;
  const bool clover = cap[0].epi == EPI_CLOV;
  if (!(clover ? (cap[1].achi == ACHI_CLOV) : (cap[0].epi == EPI_NONE && cap[1].achi == ACHI_ALPHA))) return false;
  const void *fn = cap[0].prec == PREC_F64 ? cg_persistent_kernel_f64(cap[0].recon, clover)
                                           : cg_persistent_kernel_f32(cap[0].recon, clover);
  if (!fn) return false;
  int dev = 0, nsm = 0, per_sm = 0, coop = 0;
  QPX_CUDA(cudaGetDevice(&dev));
  QPX_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  QPX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  QPX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, QPX_BLOCK, 0));
  if (!coop || per_sm < 1) return false;
  CgPersistArgs pa;
  memset(&pa, 0, sizeof(pa));
  for (int i = 0; i < 4; i++) pa.d[i] = cap[i].a;
  // phases 1 and 3 leave g5 M x: with it phases 2 and 3 apply M^+ = g5 M g5
  // through the isign = +1 kernel bodies (qpx_persist.cuh)
  pa.d[1].g5_out = 1;
  pa.d[3].g5_out = 1;
  QPX_REQUIRE(!(pa.d[1].red.mask & RED_DOT_OUT_CHI) && !(pa.d[3].red.mask & RED_DOT_OUT_CHI),
              "persistent CG: unexpected <out, chi> reduction");
  pa.r = r->sarg();
  pa.p = p->sarg();
  pa.state = lat->state;
  pa.nrhs = nrhs;
  pa.vh = (int)lat->vh;
  pa.nsb = nblocks_for(lat->vh);
  if (!lat->grid_bar) QPX_CUDA(cudaMalloc(&lat->grid_bar, sizeof(GridBarrier)));
  pa.bar = static_cast<GridBarrier *>(lat->grid_bar);
  const int grid = (int)std::min<long long>((long long)per_sm * nsm, (long long)pa.nsb * nrhs);
  QPX_CUDA(cudaMemsetAsync(pa.bar, 0, sizeof(GridBarrier), lat->stream));
  void *args[] = {&pa};
  QPX_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(QPX_BLOCK), args, 0, lat->stream));
  check_launch();
  GridBarrier hb;
  QPX_CUDA(cudaMemcpyAsync(&hb, pa.bar, sizeof(GridBarrier), cudaMemcpyDeviceToHost, lat->stream));
  state_download(lat);
  QPX_CUDA(cudaStreamSynchronize(lat->stream));
  if (hb.error)
    throw Error(QPHIX_GPU_ECUDA, "persistent CG: a grid barrier timed out (phase " + std::to_string(hb.where) + ")");
  return true;
}

// the per-rhs shift coefficients of a shifted CG solve (device, QPX_MAX_RHS)
static double *shift_coefs(qphix_gpu_lattice_s *lat) { return lat->partials + lat->partials_len - 3 * QPX_MAX_RHS; }

// r -= s_i x_i per rhs with |r|^2 on the host: the shift term of a shifted
// system's residual b - (M^+M + s) x (the per-rhs -s_i already in
// shift_coefs(lat))
static std::vector<double> sub_shift_norm(qphix_gpu_lattice_s *lat, int prec, int nr, qphix_gpu_field_s *x,
                                          qphix_gpu_field_s *r)
{
  BlasCall c;
  c.op = B_CAXPBY_NORM;
  c.x = x;
  c.y = r;
  c.a = Coef{0, 0, shift_coefs(lat), nullptr};
  c.b = cval(1.0);
  c.slots = 0x1;
  blas_launch(lat, prec, nr, c);
  const double *h = fetch_result(lat, nr, 1);
  return std::vector<double>(h, h + nr);
}

// shifts == nullptr: CG on M^+M.  Otherwise CG on M^+M + s_i for right-hand
// side i (shifted systems solved side by side, e.g. the refinement of a
// multishift solve); the iteration then stores M^+M p and updates r and x
// in a BLAS pass (B_CG_RX: r -= a (M^+M p + s p)), and the p update's fold
// keeps |p|^2 for d = <p, (M^+M + s) p> = |Mp|^2 + s |p|^2.
void solve_cg(qphix_gpu_eo_op_s *op, qphix_gpu_field_s *x, qphix_gpu_field_s *rhs, const double *rsd,
              int max_iters, int isign, int cb, qphix_gpu_solve_info *info, bool final_resid = true,
              const double *shifts = nullptr)
{
  check_solver_fields(op, x, rhs, true);
  auto *lat = x->lat;
  const int nr = x->nrhs, prec = x->prec;
  // two-flavour operator: each (up, down) pair is one system whose inner
  // products sum over both flavours (include/qphix/invcg.h with num_flav = 2)
  const bool coupled = two_flavour_kind(op->p.kind);
  QPX_REQUIRE(!coupled || nr % 2 == 0, "two-flavour fields hold (up, down) pairs");
  QPX_REQUIRE(!shifts || !coupled, "shifted CG takes single-flavour operators");
  if (shifts) {
    std::vector<double> ns(nr);
    for (int i = 0; i < nr; i++) {
      QPX_REQUIRE(shifts[i] >= 0.0, "shifts must be non-negative");
      ns[i] = -shifts[i];
    }
    QPX_CUDA(cudaMemcpyAsync(shift_coefs(lat), ns.data(), sizeof(double) * nr, cudaMemcpyHostToDevice,
                             lat->stream));
  }
  Timer timer(lat);
  Tmp mp(lat, prec, nr), mmp(lat, prec, nr), r(lat, prec, nr), p(lat, prec, nr);
  std::vector<double> chi = norm2_host(rhs);
  if (coupled) pair_sum(chi);
  eo_apply(op, mp, x, isign, cb, ApplyOpts());
  eo_apply(op, mmp, mp, -isign, cb, ApplyOpts());
  BlasCall c;
  c.op = B_XMY_NORM;
  c.x = rhs;
  c.y = mmp;
  c.z = r;
  c.slots = 0x1;
  blas_launch(lat, prec, nr, c);
  const double *h = fetch_result(lat, nr, 1);
  std::vector<double> cp(h, h + nr);
  if (shifts) cp = sub_shift_norm(lat, prec, nr, x, r);
  if (coupled) pair_sum(cp);
  SolverState &S = state_reset(lat, nr, max_iters + 1);
  S.coupled = coupled ? 1 : 0;
  bool all = true;
  for (int i = 0; i < nr; i++) {
    if (shifts) {
      S.v[S_AUX3][i] = shifts[i];
      S.v[S_AUX4][i] = cp[i];  // |p|^2 with p = r
    }
    S.v[S_RSD][i] = rsd[i] * rsd[i] * chi[i];
    S.v[S_C][i] = cp[i];
    S.v[S_RNORM][i] = cp[i];
    if (cp[i] <= S.v[S_RSD][i]) {
      S.rhs_done[i] = 1;
      S.rhs_iter[i] = 0;
    }
    all = all && S.rhs_done[i];
  }
  S.done = all ? 1 : 0;
  state_upload(lat);
  SolverState *ds = lat->state;
  unsigned long mv = 2;
  if (!all) {
    BlasCall cpy;
    cpy.op = B_COPY;
    cpy.x = r;
    cpy.y = p;
    blas_launch(lat, prec, nr, cpy);
    auto apply_both = [&] {
      ApplyOpts o1;
      o1.red_mask = RED_NORM_OUT;
      o1.fin = FIN_CG_A;
      o1.state = ds;
      eo_apply(op, mp, p, isign, cb, o1);
      ApplyOpts o2;
      o2.post = POST_CG;
      o2.red_mask = RED_NORM_R;
      o2.fin = FIN_CG_R;
      o2.state = ds;
      o2.r = r;
      o2.x = x;
      o2.p = p;
      eo_apply(op, mmp, mp, -isign, cb, o2);
    };
    auto step = [&] {
      apply_both();
      BlasCall pu;
      pu.op = B_CG_P;
      pu.x = r;
      pu.y = p;
      pu.a = cslot(ds, S_B);
      pu.state = ds;
      blas_launch(lat, prec, nr, pu);
    };
    auto step_shifted = [&] {
      ApplyOpts o1;
      o1.red_mask = RED_NORM_OUT;
      o1.fin = FIN_CG_A;
      o1.state = ds;
      eo_apply(op, mp, p, isign, cb, o1);
      ApplyOpts o2;
      o2.state = ds;
      eo_apply(op, mmp, mp, -isign, cb, o2);
      BlasCall u;
      u.op = B_CG_RX;
      u.x = x;
      u.y = r;
      u.z = mmp;
      u.v = p;
      u.a = cslot(ds, S_A);
      u.b = cslot(ds, S_AUX3);
      u.slots = 0x1;
      u.fin = FIN_CG_R;
      u.state = ds;
      blas_launch(lat, prec, nr, u);
      BlasCall pu;
      pu.op = B_CG_P;
      pu.x = r;
      pu.y = p;
      pu.a = cslot(ds, S_B);
      pu.slots = 0x1;
      pu.fin = FIN_CG_P;
      pu.state = ds;
      blas_launch(lat, prec, nr, pu);
    };
    bool done = false;
    if (shifts) {
      ApplyOpts t1;
      t1.red_mask = RED_NORM_OUT;
      pretune_op(op, lat, nr, isign, cb, {t1});
      std::string key = "cgs/" + std::to_string(op->serial) + "/" + fkey(x) + "/" + fkey(mp) + fkey(mmp) +
                        fkey(r) + fkey(p) + "/" + std::to_string(isign) + std::to_string(cb);
      run_iterations(lat, step_shifted, max_iters + 1, key);
      done = true;
    } else if (persistent_cg_wanted(op, lat, prec, nr, isign, coupled)) {
      std::vector<CapturedDslash> cap;
      g_dslash_capture = &cap;
      try {
        apply_both();
      } catch (...) {
        g_dslash_capture = nullptr;
        throw;
      }
      g_dslash_capture = nullptr;
      done = run_cg_persistent(lat, cap, r, p, nr);
    }
    if (!done) {
      std::string key = "cg/" + std::to_string(op->serial) + "/" + fkey(x) + "/" + fkey(mp) + fkey(mmp) +
                        fkey(r) + fkey(p) + "/" + std::to_string(isign) + std::to_string(cb);
      run_iterations(lat, step, max_iters + 1, key);
    }
    mv += 2ul * lat->h_state->iter;
  }
  // true residual (not counted in mv_apps: the reference's own recompute is
  // compiled out, include/qphix/invcg.h:342-403)
  std::vector<double> abs2(nr, -1.0), rel(nr, -1.0);
  if (final_resid) {
    true_residual(op, x, rhs, mmp, r, isign, cb, true, chi, abs2, rel);
    if (shifts) {
      abs2 = sub_shift_norm(lat, prec, nr, x, r);
      for (int i = 0; i < nr; i++) rel[i] = chi[i] > 0 ? std::sqrt(abs2[i] / chi[i]) : 0.0;
    }
    if (coupled) {
      pair_sum(abs2);
      for (int i = 0; i < nr; i++) rel[i] = chi[i] > 0 ? std::sqrt(abs2[i] / chi[i]) : 0.0;
    }
  }
  const SolverState &H = *lat->h_state;
  double secs = timer.stop();
  for (int i = 0; i < nr; i++) {
    info[i].n_iters = H.rhs_done[i] ? H.rhs_iter[i] : max_iters;
    info[i].rsd_sq_final = abs2[i];
    info[i].mv_apps = mv;
    info[i].site_flops = (unsigned long)(4 * 12 + 6 * 12 + H.iter * (4 * 12 + 12 * 12 + 4 * 12) + 6 * 12);
    info[i].status = H.rhs_done[i] == 2 ? 2 : (H.rhs_done[i] ? 0 : 1);
    info[i].true_rel_resid = rel[i];
    info[i].seconds = secs;
  }
}

// ---------------------------------------------------------------------------
// BiCGStab (include/qphix/invbicgstab.h:80-263)
void solve_bicgstab(qphix_gpu_eo_op_s *op, qphix_gpu_field_s *x, qphix_gpu_field_s *rhs, const double *rsd,
                    int max_iters, int isign, int cb, qphix_gpu_solve_info *info, bool final_resid = true)
{
  check_solver_fields(op, x, rhs);
  auto *lat = x->lat;
  const int nr = x->nrhs, prec = x->prec;
  Timer timer(lat);
  Tmp r0(lat, prec, nr), r(lat, prec, nr), p(lat, prec, nr), v(lat, prec, nr), t(lat, prec, nr);
  std::vector<double> bn = norm2_host(rhs);
  eo_apply(op, r0, x, isign, cb, ApplyOpts());
  BlasCall c;
  c.op = B_XMY_NORM;
  c.x = rhs;
  c.y = r0;
  c.z = r0;
  c.slots = 0x1;
  blas_launch(lat, prec, nr, c);
  const double *h = fetch_result(lat, nr, 1);
  std::vector<double> rn(h, h + nr);
  SolverState &S = state_reset(lat, nr, max_iters);
  bool all = true;
  for (int i = 0; i < nr; i++) {
    S.v[S_RSD][i] = rsd[i] * rsd[i] * bn[i];
    S.v[S_RNORM][i] = rn[i];
    S.v[S_RHO_RE][i] = rn[i];  // rho_1 = <r0, r> with r = r0
    S.v[S_RHOP_RE][i] = 1.0;
    S.v[S_ALPHA_RE][i] = 1.0;
    S.v[S_OMEGA_RE][i] = 1.0;
    S.v[S_BETA_RE][i] = rn[i];  // (rho / 1) (1 / 1)
    if (rn[i] < S.v[S_RSD][i] || bn[i] == 0.0) {
      S.rhs_done[i] = 1;
      S.rhs_iter[i] = -1;  // reported as 0
      S.v[S_BETA_RE][i] = 0;
      S.v[S_ALPHA_RE][i] = 0;
      S.v[S_OMEGA_RE][i] = 0;
    }
    all = all && S.rhs_done[i];
  }
  S.done = all ? 1 : 0;
  state_upload(lat);
  SolverState *ds = lat->state;
  unsigned long mv = 1;
  if (!all) {
    BlasCall cpy;
    cpy.op = B_COPY;
    cpy.x = r0;
    cpy.y = r;
    blas_launch(lat, prec, nr, cpy);
    BlasCall z;
    z.op = B_ZERO;
    z.x = p;
    blas_launch(lat, prec, nr, z);
    z.x = v;
    blas_launch(lat, prec, nr, z);
    auto step = [&] {
      BlasCall pu;
      pu.op = B_BICG_P;
      pu.x = r;
      pu.y = p;
      pu.z = v;
      pu.a = cslot(ds, S_BETA_RE, S_BETA_IM);
      pu.b = cslot(ds, S_OMEGA_RE, S_OMEGA_IM);
      pu.state = ds;
      blas_launch(lat, prec, nr, pu);
      ApplyOpts o1;
      o1.red_mask = RED_DOT_W_OUT;
      o1.fin = FIN_BICG_ALPHA;
      o1.state = ds;
      o1.w = r0;
      eo_apply(op, v, p, isign, cb, o1);
      BlasCall su;
      su.op = B_BICG_S;
      su.x = r;
      su.y = v;
      su.a = cslot(ds, S_ALPHA_RE, S_ALPHA_IM);
      su.state = ds;
      blas_launch(lat, prec, nr, su);
      ApplyOpts o2;
      o2.red_mask = RED_NORM_OUT | RED_DOT_OUT_CHI;
      o2.fin = FIN_BICG_OMEGA;
      o2.state = ds;
      eo_apply(op, t, r, isign, cb, o2);
      BlasCall rx;
      rx.op = B_BICG_RX;
      rx.x = x;
      rx.y = r;
      rx.z = t;
      rx.v = p;
      rx.w = r0;
      rx.a = cslot(ds, S_OMEGA_RE, S_OMEGA_IM);
      rx.b = cslot(ds, S_ALPHA_RE, S_ALPHA_IM);
      rx.slots = 0x7;
      rx.fin = FIN_BICG_RX;
      rx.state = ds;
      blas_launch(lat, prec, nr, rx);
    };
    std::string key = "bicg/" + std::to_string(op->serial) + "/" + fkey(x) + "/" + fkey(r0) + fkey(r) + fkey(p) +
                      fkey(v) + fkey(t) + "/" + std::to_string(isign) + std::to_string(cb);
    run_iterations(lat, step, max_iters, key);
    mv += 2ul * lat->h_state->iter;
  }
  std::vector<double> abs2(nr, -1.0), rel(nr, -1.0);
  if (final_resid) true_residual(op, x, rhs, t, r, isign, cb, false, bn, abs2, rel);
  const SolverState &H = *lat->h_state;
  double secs = timer.stop();
  for (int i = 0; i < nr; i++) {
    // the reference reports its loop counter after the final increment
    info[i].n_iters = H.rhs_done[i] ? H.rhs_iter[i] + 1 : max_iters + 1;
    if (H.rhs_done[i] == 2) info[i].n_iters = H.rhs_iter[i];
    info[i].rsd_sq_final = H.v[S_RNORM][i];
    info[i].mv_apps = mv;
    info[i].site_flops = (unsigned long)(4 * 12 + 24 + H.iter * (8 * 12 + 16 * 12 + 8 * 12 + 8 * 12 + 4 * 12 +
                                                                  8 * 12 + 28 * 12));
    info[i].status = H.rhs_done[i] == 2 ? 2 : (H.rhs_done[i] ? 0 : 1);
    info[i].true_rel_resid = rel[i];
    info[i].seconds = secs;
  }
}

// ---------------------------------------------------------------------------
// MR (include/qphix/invmr.h:62-210), terminating on the relative residual
// terminate = false: InvMRSmoother, exactly max_iters iterations with no
// residual test (include/qphix/invmr.h:302-354, terminateOnResiduum false)
void solve_mr(qphix_gpu_eo_op_s *op, qphix_gpu_field_s *x, qphix_gpu_field_s *rhs, const double *rsd, int max_iters,
              double omega, int isign, int cb, qphix_gpu_solve_info *info, bool final_resid = true,
              bool terminate = true)
{
  check_solver_fields(op, x, rhs);
  auto *lat = x->lat;
  const int nr = x->nrhs, prec = x->prec;
  Timer timer(lat);
  if (max_iters == 0) {
    for (int i = 0; i < nr; i++) {
      info[i] = qphix_gpu_solve_info{};
      info[i].rsd_sq_final = -1;
    }
    return;
  }
  Tmp r(lat, prec, nr), Mr(lat, prec, nr);
  std::vector<double> bn = norm2_host(rhs);
  eo_apply(op, r, x, isign, cb, ApplyOpts());
  BlasCall c;
  c.op = B_XMY_NORM;
  c.x = rhs;
  c.y = r;
  c.z = r;
  c.slots = 0x1;
  blas_launch(lat, prec, nr, c);
  const double *h = fetch_result(lat, nr, 1);
  std::vector<double> cp(h, h + nr);
  SolverState &S = state_reset(lat, nr, max_iters);
  bool all = true;
  for (int i = 0; i < nr; i++) {
    S.v[S_RSD][i] = terminate ? rsd[i] * rsd[i] * bn[i] : -1.0;  // |r|^2 > -1 always: no residual stop
    S.v[S_RNORM][i] = cp[i];
    S.v[S_AUX0][i] = omega;
    if (terminate && (cp[i] < S.v[S_RSD][i] || bn[i] == 0.0)) {
      S.rhs_done[i] = 1;
      S.rhs_iter[i] = 0;
    }
    all = all && S.rhs_done[i];
  }
  S.done = all ? 1 : 0;
  state_upload(lat);
  SolverState *ds = lat->state;
  unsigned long mv = 1;
  if (!all) {
    auto step = [&] {
      ApplyOpts o;
      o.red_mask = RED_NORM_OUT | RED_DOT_OUT_CHI;
      o.fin = FIN_MR_A;
      o.state = ds;
      eo_apply(op, Mr, r, isign, cb, o);
      BlasCall u;
      u.op = B_MR_RX;
      u.x = x;
      u.y = r;
      u.z = Mr;
      u.a = cslot(ds, S_ALPHA_RE, S_ALPHA_IM);
      u.slots = 0x1;
      u.fin = FIN_MR_R;
      u.state = ds;
      blas_launch(lat, prec, nr, u);
    };
    std::string key = "mr/" + std::to_string(op->serial) + "/" + fkey(x) + "/" + fkey(r) + fkey(Mr) + "/" +
                      std::to_string(isign) + std::to_string(cb);
    run_iterations(lat, step, max_iters, key);
    mv += lat->h_state->iter;
  }
  std::vector<double> abs2(nr, -1.0), rel(nr, -1.0);
  if (final_resid) {
    Tmp t(lat, prec, nr), rr(lat, prec, nr);
    true_residual(op, x, rhs, t, rr, isign, cb, false, bn, abs2, rel);
  }
  const SolverState &H = *lat->h_state;
  double secs = timer.stop();
  for (int i = 0; i < nr; i++) {
    info[i].n_iters = H.rhs_done[i] ? H.rhs_iter[i] : H.iter;
    info[i].rsd_sq_final = terminate ? H.v[S_RNORM][i] / bn[i] : -1.0;
    info[i].mv_apps = mv;
    info[i].site_flops = (unsigned long)(24 + 8 * 12 + H.iter * (12 * 12 + 2 * 8 * 12 + 4 * 12));
    info[i].status = (H.rhs_done[i] || !terminate) ? 0 : 1;
    info[i].true_rel_resid = rel[i];
    info[i].seconds = secs;
  }
}

// ---------------------------------------------------------------------------
// Richardson defect correction (include/qphix/inv_richardson_multiprec.h:42-239)
void solve_richardson(qphix_gpu_eo_op_s *op, qphix_gpu_eo_op_s *opi, int inner, qphix_gpu_field_s *x,
                      qphix_gpu_field_s *rhs, double rsd, double delta, int max_iters, int inner_max, int isign,
                      int cb, qphix_gpu_solve_info *info)
{
  check_solver_fields(op, x, rhs);
  QPX_REQUIRE(opi, "null inner operator");
  auto *lat = x->lat;
  // the inner operator's fields may live on another lattice object of the
  // same shape (QPhiX gives the inner solver its own Geometry): that stream
  // is synchronised once, so the fields are complete, and every step of the
  // solve, inner temporaries included, then runs on x's lattice and stream
  QPX_REQUIRE(same_shape(opi->gauge->lat, lat), "inner and outer lattices differ");
  sync_op_fields(opi, lat);
  auto *lati = lat;
  const int nr = x->nrhs, prec = x->prec, iprec = opi->gauge->prec;
  Timer timer(lat);
  Tmp r(lat, prec, nr), tmp(lat, prec, nr), dx(lat, prec, nr);
  Tmp rin(lati, iprec, nr), dxin(lati, iprec, nr);
  std::vector<double> bn = norm2_host(rhs);
  std::vector<double> rsd_t(nr);
  for (int i = 0; i < nr; i++) rsd_t[i] = rsd * rsd * bn[i];
  eo_apply(op, tmp, x, isign, cb, ApplyOpts());
  BlasCall c;
  c.op = B_XMY_NORM;
  c.x = rhs;
  c.y = tmp;
  c.z = r;
  c.slots = 0x1;
  blas_launch(lat, prec, nr, c);
  const double *h = fetch_result(lat, nr, 1);
  std::vector<double> rn(h, h + nr);
  unsigned long mv_outer = 1, mv_inner = 0;
  std::vector<int> done(nr, 0);
  bool all = true;
  for (int i = 0; i < nr; i++) {
    done[i] = rn[i] < rsd_t[i] || bn[i] == 0.0;
    all = all && done[i];
  }
  int iter = 0;
  // per-rhs scale factors live in the state's AUX slots between inner solves
  std::vector<double> scale_dn(nr), scale_up(nr), inner_rsd(nr);
  // the two per-rhs scale vectors live at the end of the reduction workspace
  double *d_scales = lat->partials + lat->partials_len - 2 * QPX_MAX_RHS;
  std::vector<qphix_gpu_solve_info> ii(nr);
  try {
    if (!all) {
      for (iter = 1; iter < max_iters; iter++) {
        for (int i = 0; i < nr; i++) {
          double dfin = std::sqrt(rsd_t[i] / rn[i]);
          inner_rsd[i] = done[i] ? 1.0 : (dfin > delta ? dfin : delta);
          double rnorm = std::sqrt(rn[i]);
          scale_dn[i] = done[i] ? 0.0 : 1.0 / rnorm;
          scale_up[i] = done[i] ? 0.0 : rnorm;
        }
        std::vector<double> sc(2 * QPX_MAX_RHS, 0.0);
        for (int i = 0; i < nr; i++) {
          sc[i] = scale_dn[i];
          sc[QPX_MAX_RHS + i] = scale_up[i];
        }
        QPX_CUDA(cudaMemcpyAsync(d_scales, sc.data(), sizeof(double) * 2 * QPX_MAX_RHS, cudaMemcpyHostToDevice,
                                 lat->stream));
        convert_field(rin, r, Coef{0, 0, d_scales, nullptr}, nullptr);
        BlasCall z;
        z.op = B_ZERO;
        z.x = dxin;
        blas_launch(lat, iprec, nr, z);
        if (inner == QPHIX_GPU_SOLVER_BICGSTAB)
          solve_bicgstab(opi, dxin, rin, inner_rsd.data(), inner_max, isign, cb, ii.data(), false);
        else if (inner == QPHIX_GPU_SOLVER_MR)
          solve_mr(opi, dxin, rin, inner_rsd.data(), inner_max, 1.0, isign, cb, ii.data(), false);
        else
          solve_cg(opi, dxin, rin, inner_rsd.data(), inner_max, isign, cb, ii.data(), false);
        mv_inner += ii[0].mv_apps;
        convert_field(dx, dxin, Coef{0, 0, d_scales + QPX_MAX_RHS, nullptr}, nullptr);
        eo_apply(op, tmp, dx, isign, cb, ApplyOpts());
        mv_outer++;
        BlasCall u;
        u.op = B_RICH_RX;
        u.x = x;
        u.y = r;
        u.z = dx;
        u.w = tmp;
        u.slots = 0x1;
        blas_launch(lat, prec, nr, u);
        h = fetch_result(lat, nr, 1);
        all = true;
        for (int i = 0; i < nr; i++) {
          rn[i] = h[i];
          if (!done[i] && rn[i] < rsd_t[i]) done[i] = 1;
          all = all && done[i];
        }
        if (all) break;
      }
    }
  } catch (...) {
    throw;
  }
  std::vector<double> abs2, rel;
  true_residual(op, x, rhs, tmp, r, isign, cb, false, bn, abs2, rel);
  mv_outer++;
  double secs = timer.stop();
  for (int i = 0; i < nr; i++) {
    info[i].n_iters = iter;
    info[i].rsd_sq_final = bn[i] > 0 ? abs2[i] / bn[i] : 0.0;  // relative, as the reference reports
    info[i].mv_apps = mv_outer + mv_inner;
    info[i].site_flops = 0;
    info[i].status = done[i] ? 0 : 1;
    info[i].true_rel_resid = rel[i];
    info[i].seconds = secs;
  }
}

// ---------------------------------------------------------------------------
// BiCGStab with reliable updates (no counterpart in the reference): the
// Krylov iteration runs on op_lo (16-bit or FP32 storage, FP32 arithmetic)
// and is never restarted; the low-precision solution increment is folded into
// the FP64 solution and r is replaced by the FP64 true residual b - M x
// whenever a right-hand side's iterated residual has dropped by `delta`
// since its last update (or reaches the target).  Convergence is decided on
// the true residual only.
void solve_bicgstab_mixed(qphix_gpu_eo_op_s *op, qphix_gpu_eo_op_s *opl, qphix_gpu_field_s *x,
                          qphix_gpu_field_s *rhs, double rsd, double delta, int max_iters, int isign, int cb,
                          qphix_gpu_solve_info *info)
{
  check_solver_fields(op, x, rhs);
  QPX_REQUIRE(opl, "null low-precision operator");
  auto *lat = x->lat;
  // the low-precision operator's fields may live on another lattice object of
  // the same shape: that stream is synchronised once, and every step of the
  // solve then runs on x's lattice and stream
  QPX_REQUIRE(same_shape(opl->gauge->lat, lat), "the two operators' lattices differ");
  sync_op_fields(opl, lat);
  auto *latl = lat;
  const int nr = x->nrhs, prec = x->prec, lp = opl->gauge->prec;
  Timer timer(lat);
  Tmp rh(lat, prec, nr), th(lat, prec, nr);
  Tmp r0(latl, lp, nr), r(latl, lp, nr), p(latl, lp, nr), v(latl, lp, nr), t(latl, lp, nr), xl(latl, lp, nr);
  std::vector<double> bn = norm2_host(rhs);
  // true residual in FP64 -> rh, |rh|^2
  auto true_r = [&]() {
    eo_apply(op, th, x, isign, cb, ApplyOpts());
    BlasCall c;
    c.op = B_XMY_NORM;
    c.x = rhs;
    c.y = th;
    c.z = rh;
    c.slots = 0x1;
    blas_launch(lat, prec, nr, c);
    const double *h = fetch_result(lat, nr, 1);
    return std::vector<double>(h, h + nr);
  };
  std::vector<double> rn = true_r();
  unsigned long mv_hi = 1, updates = 0;
  std::vector<int> conv(nr, 0);
  bool all = true;
  for (int i = 0; i < nr; i++) {
    conv[i] = (rn[i] < rsd * rsd * bn[i]) || bn[i] == 0.0;
    all = all && conv[i];
  }
  int low_iters = 0;
  if (!all) {
    // r = r0 = convert(rh); xl = p = v = 0
    convert_field(r, rh, cval(1.0), nullptr);
    BlasCall cpy;
    cpy.op = B_COPY;
    cpy.x = r;
    cpy.y = r0;
    blas_launch(latl, lp, nr, cpy);
    BlasCall z;
    z.op = B_ZERO;
    z.x = p;
    blas_launch(latl, lp, nr, z);
    z.x = v;
    blas_launch(latl, lp, nr, z);
    z.x = xl;
    blas_launch(latl, lp, nr, z);
    SolverState &S = state_reset(latl, nr, max_iters);
    for (int i = 0; i < nr; i++) {
      S.v[S_RSD][i] = rsd * rsd * bn[i];
      S.v[S_AUX1][i] = delta * delta * rn[i];
      S.v[S_RNORM][i] = rn[i];
      S.v[S_RHO_RE][i] = rn[i];
      S.v[S_RHOP_RE][i] = 1.0;
      S.v[S_ALPHA_RE][i] = 1.0;
      S.v[S_OMEGA_RE][i] = 1.0;
      S.v[S_BETA_RE][i] = rn[i];
      if (conv[i]) {
        S.rhs_done[i] = 1;
        S.v[S_BETA_RE][i] = S.v[S_ALPHA_RE][i] = S.v[S_OMEGA_RE][i] = 0.0;
      }
    }
    state_upload(latl);
    SolverState *ds = latl->state;
    auto step = [&] {
      BlasCall pu;
      pu.op = B_BICG_P;
      pu.x = r;
      pu.y = p;
      pu.z = v;
      pu.a = cslot(ds, S_BETA_RE, S_BETA_IM);
      pu.b = cslot(ds, S_OMEGA_RE, S_OMEGA_IM);
      pu.state = ds;
      blas_launch(latl, lp, nr, pu);
      ApplyOpts o1;
      o1.red_mask = RED_DOT_W_OUT;
      o1.fin = FIN_BICG_ALPHA;
      o1.state = ds;
      o1.w = r0;
      eo_apply(opl, v, p, isign, cb, o1);
      BlasCall su;
      su.op = B_BICG_S;
      su.x = r;
      su.y = v;
      su.a = cslot(ds, S_ALPHA_RE, S_ALPHA_IM);
      su.state = ds;
      blas_launch(latl, lp, nr, su);
      ApplyOpts o2;
      o2.red_mask = RED_NORM_OUT | RED_DOT_OUT_CHI;
      o2.fin = FIN_BICG_OMEGA;
      o2.state = ds;
      eo_apply(opl, t, r, isign, cb, o2);
      BlasCall rx;
      rx.op = B_BICG_RX;
      rx.x = xl;
      rx.y = r;
      rx.z = t;
      rx.v = p;
      rx.w = r0;
      rx.a = cslot(ds, S_OMEGA_RE, S_OMEGA_IM);
      rx.b = cslot(ds, S_ALPHA_RE, S_ALPHA_IM);
      rx.slots = 0x7;
      rx.fin = FIN_BICG_RU;
      rx.state = ds;
      blas_launch(latl, lp, nr, rx);
    };
    op_tmp(opl, nr, latl);  // the operator's temporary must exist before graph capture
    {
      ApplyOpts t1, t2;
      t1.red_mask = RED_DOT_W_OUT;
      t1.w = r0;
      t2.red_mask = RED_NORM_OUT | RED_DOT_OUT_CHI;
      pretune_op(opl, latl, nr, isign, cb, {t1, t2});
    }
    std::string key = "bicg-ru/" + std::to_string(opl->serial) + "/" + fkey(xl) + fkey(r0) + fkey(r) + fkey(p) +
                      fkey(v) + fkey(t) + "/" + std::to_string(isign) + std::to_string(cb);
    while (true) {
      run_iterations(latl, step, max_iters, key);
      SolverState &H = *latl->h_state;
      low_iters = H.iter;
      // reliable update for every active rhs: x += xl, xl = 0, rh = b - M x
      convert_field(x, xl, cval(1.0), nullptr, 1);
      BlasCall zx;
      zx.op = B_ZERO;
      zx.x = xl;
      blas_launch(latl, lp, nr, zx);
      rn = true_r();
      mv_hi++;
      updates++;
      all = true;
      for (int i = 0; i < nr; i++) {
        if (!conv[i] && rn[i] < rsd * rsd * bn[i]) conv[i] = 1;
        all = all && conv[i];
      }
      bool out_of_iters = H.iter >= max_iters || H.status == 2;
      if (all || out_of_iters) break;
      // r = convert(rh); rho = <r0, r>; beta from it; restart the graph
      convert_field(r, rh, cval(1.0), nullptr);
      BlasCall dt;
      dt.op = B_DOT;
      dt.x = r0;
      dt.y = r;
      dt.slots = 0x3;
      blas_launch(latl, lp, nr, dt);
      const double *rho = fetch_result(latl, nr, 2);
      for (int i = 0; i < nr; i++) {
        if (conv[i]) {
          if (!H.rhs_done[i]) {
            H.rhs_done[i] = 1;
            H.rhs_iter[i] = H.iter;
          }
          H.v[S_BETA_RE][i] = H.v[S_BETA_IM][i] = 0.0;
          H.v[S_ALPHA_RE][i] = H.v[S_ALPHA_IM][i] = 0.0;
          H.v[S_OMEGA_RE][i] = H.v[S_OMEGA_IM][i] = 0.0;
          continue;
        }
        double rr = rho[2 * i], ri = rho[2 * i + 1];
        H.v[S_RHO_RE][i] = rr;
        H.v[S_RHO_IM][i] = ri;
        double t1r, t1i, t2r, t2i, d1 = H.v[S_RHOP_RE][i] * H.v[S_RHOP_RE][i] + H.v[S_RHOP_IM][i] * H.v[S_RHOP_IM][i];
        t1r = (rr * H.v[S_RHOP_RE][i] + ri * H.v[S_RHOP_IM][i]) / d1;
        t1i = (ri * H.v[S_RHOP_RE][i] - rr * H.v[S_RHOP_IM][i]) / d1;
        double d2 = H.v[S_OMEGA_RE][i] * H.v[S_OMEGA_RE][i] + H.v[S_OMEGA_IM][i] * H.v[S_OMEGA_IM][i];
        t2r = (H.v[S_ALPHA_RE][i] * H.v[S_OMEGA_RE][i] + H.v[S_ALPHA_IM][i] * H.v[S_OMEGA_IM][i]) / d2;
        t2i = (H.v[S_ALPHA_IM][i] * H.v[S_OMEGA_RE][i] - H.v[S_ALPHA_RE][i] * H.v[S_OMEGA_IM][i]) / d2;
        H.v[S_BETA_RE][i] = t1r * t2r - t1i * t2i;
        H.v[S_BETA_IM][i] = t1r * t2i + t1i * t2r;
        H.v[S_AUX1][i] = delta * delta * rn[i];
      }
      H.done = 0;
      H.status = 0;
      state_upload(latl);
    }
  }
  std::vector<double> abs2(rn), rel(nr);
  for (int i = 0; i < nr; i++) rel[i] = bn[i] > 0 ? std::sqrt(rn[i] / bn[i]) : 0.0;
  const SolverState &H = *latl->h_state;
  double secs = timer.stop();
  for (int i = 0; i < nr; i++) {
    info[i].n_iters = low_iters;
    info[i].rsd_sq_final = abs2[i];
    info[i].mv_apps = mv_hi + 2ul * (unsigned long)low_iters;
    info[i].site_flops = updates;  // number of reliable updates
    info[i].status = conv[i] ? 0 : (H.status == 2 ? 2 : 1);
    info[i].true_rel_resid = rel[i];
    info[i].seconds = secs;
  }
}

}  // namespace

static int solve_status(const qphix_gpu_solve_info *info, int n)
{
  for (int i = 0; i < n; i++)
    if (info[i].status == 2) return QPHIX_GPU_EBREAKDOWN;
  for (int i = 0; i < n; i++)
    if (info[i].status == 1) return QPHIX_GPU_ENOTCONV;
  return QPHIX_GPU_OK;
}

#define QPX_SOLVE_ENTRY(body)                                               \
  int rc = guard([&] { body; });                                            \
  if (rc) return rc;                                                        \
  int st_ = solve_status(info, x->nrhs);                                    \
  if (st_) g_last_error = st_ == QPHIX_GPU_ENOTCONV ? "solver did not converge" : "solver breakdown"; \
  return st_;

extern "C" int qphix_gpu_solve_cg(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target,
                                  int max_iters, int isign, int cb, qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x, "null argument");
    std::vector<double> rs(x->nrhs, rsd_target);
    solve_cg(op, x, rhs, rs.data(), max_iters, isign, cb, info);
  })
}

extern "C" int qphix_gpu_solve_bicgstab(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs,
                                        double rsd_target, int max_iters, int isign, int cb,
                                        qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x, "null argument");
    std::vector<double> rs(x->nrhs, rsd_target);
    solve_bicgstab(op, x, rhs, rs.data(), max_iters, isign, cb, info);
  })
}

extern "C" int qphix_gpu_solve_mr(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target,
                                  int max_iters, double omega, int isign, int cb, qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x, "null argument");
    std::vector<double> rs(x->nrhs, rsd_target);
    solve_mr(op, x, rhs, rs.data(), max_iters, omega, isign, cb, info);
  })
}

extern "C" int qphix_gpu_solve_mr_smoother(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs,
                                           int n_iters, double omega, int isign, int cb, qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x, "null argument");
    QPX_REQUIRE(n_iters >= 0, "n_iters must be >= 0");
    std::vector<double> rs(x->nrhs, 0.0);
    solve_mr(op, x, rhs, rs.data(), n_iters, omega, isign, cb, info, true, false);
  })
}

extern "C" int qphix_gpu_solve_bicgstab_mixed(qphix_gpu_eo_op op, qphix_gpu_eo_op op_low, qphix_gpu_field x,
                                              qphix_gpu_field rhs, double rsd_target, double delta, int max_iters,
                                              int isign, int cb, qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x, "null argument");
    QPX_REQUIRE(delta > 0.0 && delta < 1.0, "delta must be in (0, 1)");
    solve_bicgstab_mixed(op, op_low, x, rhs, rsd_target, delta, max_iters, isign, cb, info);
  })
}

extern "C" int qphix_gpu_solve_richardson(qphix_gpu_eo_op op_outer, qphix_gpu_eo_op op_inner, int inner_solver,
                                          qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target, double delta,
                                          int max_iters, int inner_max_iters, int isign, int cb,
                                          qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x, "null argument");
    solve_richardson(op_outer, op_inner, inner_solver, x, rhs, rsd_target, delta, max_iters, inner_max_iters,
                     isign, cb, info);
  })
}

// ---------------------------------------------------------------------------
// multishift CG (include/qphix/minvcg.h:77-387): one M^dag M per iteration
// for the base system; the per-shift zeta / beta recurrences run on the device
// (FIN_MCG_*), r += b M^dag M p0 is fused into the second Dslash, and every
// shifted x / p update plus p0 = r + a p0 is one multi-vector kernel.
static void solve_mshift(qphix_gpu_eo_op_s *op, qphix_gpu_field_s **x, qphix_gpu_field_s *rhs, int ns,
                         const double *shifts, const double *rsd, int max_iters, int isign, int cb, int *n_iters,
                         double *rsd_sq_final, unsigned long *mv_apps)
{
  QPX_REQUIRE(op && x && rhs && shifts && rsd && n_iters && rsd_sq_final && mv_apps, "null argument");
  QPX_REQUIRE(ns >= 1 && ns <= QPX_MAX_SHIFTS, "n_shift must be in [1, 32]");
  require_spinor(rhs, "rhs");
  QPX_REQUIRE(rhs->nrhs == 1, "multishift CG takes one right-hand side");
  for (int s = 0; s < ns; s++) {
    require_spinor(x[s], "x");
    require_same(x[s], rhs);
    QPX_REQUIRE(x[s]->nrhs == 1, "multishift CG solutions hold one right-hand side");
  }
  require_same(rhs, op->gauge);
  auto *lat = rhs->lat;
  const int prec = rhs->prec;
  Tmp r(lat, prec, 1), p0(lat, prec, 1), mp(lat, prec, 1), mmp(lat, prec, 1);
  std::vector<Tmp *> ps;
  for (int s = 0; s < ns; s++) ps.push_back(new Tmp(lat, prec, 1));
  struct Free {
    std::vector<Tmp *> &v;
    ~Free()
    {
      for (auto *t : v) delete t;
    }
  } free_ps{ps};
  double cp = norm2_host(rhs)[0];
  // r = p0 = p_s = rhs
  BlasCall cpy;
  cpy.op = B_COPY;
  cpy.x = rhs;
  cpy.y = r;
  blas_launch(lat, prec, 1, cpy);
  cpy.y = p0;
  blas_launch(lat, prec, 1, cpy);
  for (int s = 0; s < ns; s++) {
    cpy.y = *ps[s];
    blas_launch(lat, prec, 1, cpy);
  }
  eo_apply(op, mp, p0, isign, cb, ApplyOpts());
  eo_apply(op, mmp, mp, -isign, cb, ApplyOpts());
  unsigned long mv = 2;
  double d = norm2_host(mp)[0];
  double b = -cp / d;
  // r = r + b mmp, c = |r|^2
  BlasCall ax;
  ax.op = B_CAXPBY_NORM;
  ax.x = mmp;
  ax.y = r;
  ax.a = cval(b);
  ax.b = cval(1.0);
  ax.slots = 0x1;
  blas_launch(lat, prec, 1, ax);
  double c = fetch_result(lat, 1, 1)[0];
  SolverState &S = state_reset(lat, ns, max_iters);
  std::vector<double> beta(ns);
  for (int s = 0; s < ns; s++) {
    double z = 1.0 / (1.0 - shifts[s] * b);
    beta[s] = b / (1.0 - shifts[s] * b);
    S.v[S_AUX1][s] = 1.0;  // zeta_prev
    S.v[S_AUX0][s] = z;
    S.v[S_BETA_RE][s] = beta[s];
    S.v[S_AUX3][s] = shifts[s];
    S.v[S_RSD][s] = rsd[s] * rsd[s] * cp;
    S.v[S_AUX6][s] = 0.0;  // no pending x update before the first iteration
    rsd_sq_final[s] = 0.0;
  }
  // first iteration's coefficients: a = c / cp, as_s = a zeta beta / (zeta_prev b)
  double a = c / cp;
  S.v[S_A][0] = a;
  S.v[S_B][0] = b;
  S.v[S_C][0] = c;
  for (int s = 0; s < ns; s++) S.v[S_AUX2][s] = a * S.v[S_AUX0][s] * S.v[S_BETA_RE][s] / (1.0 * b);
  S.done = (max_iters <= 1) ? 1 : 0;
  // x_s = -beta_s rhs
  for (int s = 0; s < ns; s++) {
    BlasCall xb;
    xb.op = B_CAXPBY;
    xb.x = rhs;
    xb.y = x[s];
    xb.a = cval(-beta[s]);
    xb.b = cval(0.0);
    blas_launch(lat, prec, 1, xb);
  }
  state_upload(lat);
  SolverState *ds = lat->state;
  MShiftArgs ma;
  memset(&ma, 0, sizeof(ma));
  ma.vh = (int)lat->vh;
  ma.nshift = ns;
  ma.r = static_cast<qphix_gpu_field_s *>(r)->sarg();
  ma.p0 = static_cast<qphix_gpu_field_s *>(p0)->sarg();
  for (int s = 0; s < ns; s++) {
    ma.x[s] = x[s]->sarg();
    ma.p[s] = static_cast<qphix_gpu_field_s *>(*ps[s])->sarg();
  }
  ma.state = ds;
  if (!S.done) {
    auto step = [&] {
      MShiftArgs m = ma;
      m.x_only = 0;
      launch_mshift(prec, m, dim3(nblocks_for(lat->vh)), lat->stream);
      check_launch();
      ApplyOpts o1;
      o1.red_mask = RED_NORM_OUT;
      o1.fin = FIN_MCG_D;
      o1.state = ds;
      eo_apply(op, mp, p0, isign, cb, o1);
      ApplyOpts o2;
      o2.post = POST_RAXPY;
      o2.red_mask = RED_NORM_R;
      o2.fin = FIN_MCG_R;
      o2.state = ds;
      o2.r = r;
      eo_apply(op, mmp, mp, -isign, cb, o2);
    };
    std::string key = "mcg/" + std::to_string(op->serial) + "/" + fkey(r) + fkey(p0) + fkey(mp) + fkey(mmp) + "/";
    for (int s = 0; s < ns; s++) key += fkey(x[s]) + "," + fkey(*ps[s]) + ";";
    key += "/" + std::to_string(isign) + std::to_string(cb);
    run_iterations(lat, step, max_iters, key);
    mv += 2ul * lat->h_state->iter;
    // the x update of the last iteration is still pending
    MShiftArgs m = ma;
    m.x_only = 1;
    launch_mshift(prec, m, dim3(nblocks_for(lat->vh)), lat->stream);
    check_launch();
    QPX_CUDA(cudaStreamSynchronize(lat->stream));
  }
  const SolverState &H = *lat->h_state;
  *n_iters = H.iter;
  for (int s = 0; s < ns; s++) rsd_sq_final[s] = H.rhs_done[s] ? H.v[S_RNORM][s] : 0.0;
  *mv_apps = mv;
  bool all = true;
  for (int s = 0; s < ns; s++) all = all && H.rhs_done[s];
  if (!all && !S.done) throw Error(QPHIX_GPU_ENOTCONV, "multishift CG did not converge");
}

extern "C" int qphix_gpu_solve_mshift_cg(qphix_gpu_eo_op op, qphix_gpu_field *x, qphix_gpu_field rhs, int n_shift,
                                         const double *shifts, const double *rsd_target, int max_iters, int isign,
                                         int cb, int *n_iters, double *rsd_sq_final, unsigned long *mv_apps)
{
  return guard([&] {
    solve_mshift(op, x, rhs, n_shift, shifts, rsd_target, max_iters, isign, cb, n_iters, rsd_sq_final, mv_apps);
  });
}

// ---------------------------------------------------------------------------
// CG on the shifted normal equations (M^+M + s_i) x_i = b_i, one shift per
// right-hand side (no reference counterpart: the batched form of the
// per-shift refinement that follows a multishift solve).
extern "C" int qphix_gpu_solve_cg_shifted(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs,
                                          const double *shifts, const double *rsd_target, int max_iters, int isign,
                                          int cb, qphix_gpu_solve_info *info)
{
  QPX_SOLVE_ENTRY({
    QPX_REQUIRE(info && x && shifts && rsd_target, "null argument");
    solve_cg(op, x, rhs, rsd_target, max_iters, isign, cb, info, true, shifts);
  })
}

// one right-hand side of a multi-rhs spinor field as a one-rhs field argument
static SpinorArg slice_arg(const qphix_gpu_field_s *f, int s)
{
  SpinorArg a = f->sarg();
  a.data = static_cast<char *>(a.data) + (size_t)s * a.rhs_stride_chunks * 16;  // 16-byte spinor chunks
  if (a.norm) a.norm += (size_t)s * a.stride;
  return a;
}

static void convert_slice(int pdst, const SpinorArg &dst, int psrc, const SpinorArg &src, qphix_gpu_lattice_s *lat)
{
  launch_convert(pdst, psrc, (int)lat->vh, src, dst, Coef{1.0, 0, nullptr, nullptr}, nullptr,
                 dim3(nblocks_for(lat->vh), 1), lat->stream, 0);
  check_launch();
}

// Multishift CG with low-precision iterations (no reference counterpart;
// the shifted systems of include/qphix/minvcg.h:77-387): one multishift CG
// on op_low (FP32 or 16-bit storage) to rsd_low, then every shift's solution
// in op's precision is refined side by side, a shift per right-hand side:
// R = b - (M^+M + s) X in op's precision, the low-precision shifted CG on
// R / |R| (qphix_gpu_solve_cg_shifted's iteration) to the fraction of
// |R| that is still missing (with a margin), X += |R| D, until every shift
// meets rsd_target by its true residual.
static void solve_mshift_mixed(qphix_gpu_eo_op_s *op, qphix_gpu_eo_op_s *opl, qphix_gpu_field_s **x,
                               qphix_gpu_field_s *rhs, int ns, const double *shifts, const double *rsd,
                               const double *rsd_low, int max_iters, int isign, int cb, int *n_iters,
                               int *refine_iters, int *corrections, double *rel_sq_final, unsigned long *mv_apps)
{
  QPX_REQUIRE(op && opl && x && rhs && shifts && rsd && n_iters && refine_iters && corrections && rel_sq_final &&
                  mv_apps,
              "null argument");
  QPX_REQUIRE(ns >= 1 && ns <= QPX_MAX_RHS, "n_shift must be in [1, 32]");
  require_spinor(rhs, "rhs");
  QPX_REQUIRE(rhs->nrhs == 1, "multishift CG takes one right-hand side");
  for (int s = 0; s < ns; s++) {
    require_spinor(x[s], "x");
    require_same(x[s], rhs);
    QPX_REQUIRE(x[s]->nrhs == 1, "multishift CG solutions hold one right-hand side");
    QPX_REQUIRE(shifts[s] >= 0.0, "shifts must be non-negative");
  }
  require_same(rhs, op->gauge);
  QPX_REQUIRE(!two_flavour_kind(op->p.kind) && !two_flavour_kind(opl->p.kind),
              "multishift CG takes single-flavour operators");
  auto *lat = rhs->lat;
  QPX_REQUIRE(same_shape(opl->gauge->lat, lat), "the two operators' lattices differ");
  sync_op_fields(op, lat);
  sync_op_fields(opl, lat);
  const int prec = rhs->prec, lp = opl->gauge->prec;
  const double bn = norm2_host(rhs)[0];
  if (bn == 0.0) {  // every solution is zero
    for (int s = 0; s < ns; s++) {
      BlasCall z;
      z.op = B_ZERO;
      z.x = x[s];
      blas_launch(lat, prec, 1, z);
      rel_sq_final[s] = 0.0;
    }
    QPX_CUDA(cudaStreamSynchronize(lat->stream));
    *n_iters = *refine_iters = *corrections = 0;
    *mv_apps = 0;
    return;
  }

  // 1. the multishift CG in the low precision
  Tmp bl(lat, lp, 1);
  convert_field(bl, rhs, cval(1.0), nullptr);
  std::vector<Tmp *> xl;
  struct Free {
    std::vector<Tmp *> &v;
    ~Free()
    {
      for (auto *t : v) delete t;
    }
  } free_xl{xl};
  std::vector<qphix_gpu_field_s *> xlp;
  for (int s = 0; s < ns; s++) {
    xl.push_back(new Tmp(lat, lp, 1));
    xlp.push_back(*xl.back());
  }
  std::vector<double> lsq(ns);
  unsigned long mv = 0;
  solve_mshift(opl, xlp.data(), bl, ns, shifts, rsd_low ? rsd_low : rsd, max_iters, isign, cb, n_iters, lsq.data(),
               &mv);

  // 2. every shift as a right-hand side in op's precision
  Tmp X(lat, prec, ns), B(lat, prec, ns), T1(lat, prec, ns), T2(lat, prec, ns), R(lat, prec, ns);
  Tmp Rl(lat, lp, ns), Dl(lat, lp, ns);
  for (int s = 0; s < ns; s++) {
    convert_slice(prec, slice_arg(X, s), lp, static_cast<qphix_gpu_field_s *>(*xl[s])->sarg(), lat);
    convert_slice(prec, slice_arg(B, s), prec, rhs->sarg(), lat);
  }
  std::vector<double> nsig(ns), t2(ns), rn(ns);
  for (int s = 0; s < ns; s++) {
    nsig[s] = -shifts[s];
    t2[s] = rsd[s] * rsd[s] * bn;
  }
  auto residual = [&] {  // R = B - (M^+M + s) X, |R_s|^2
    eo_apply(op, T1, X, isign, cb, ApplyOpts());
    eo_apply(op, T2, T1, -isign, cb, ApplyOpts());
    mv += 2;
    BlasCall c;
    c.op = B_XMY_NORM;
    c.x = B;
    c.y = T2;
    c.z = R;
    c.slots = 0x1;
    blas_launch(lat, prec, ns, c);
    QPX_CUDA(cudaMemcpyAsync(shift_coefs(lat), nsig.data(), sizeof(double) * ns, cudaMemcpyHostToDevice,
                             lat->stream));
    rn = sub_shift_norm(lat, prec, ns, X, R);
  };

  // 3. refinement rounds
  double *d_scales = lat->partials + lat->partials_len - 2 * QPX_MAX_RHS;
  std::vector<qphix_gpu_solve_info> ii(ns);
  std::vector<int> done(ns, 0);
  int corr = 0, rit = 0;
  const int max_rounds = 10;
  for (int round = 0;; round++) {
    residual();
    bool all = true;
    for (int s = 0; s < ns; s++) {
      done[s] = rn[s] <= t2[s] || bn == 0.0;
      all = all && done[s];
    }
    if (all || round == max_rounds) break;
    std::vector<double> sc(2 * QPX_MAX_RHS, 0.0), inner(ns, 1.0);
    for (int s = 0; s < ns; s++) {
      if (done[s]) continue;  // a zero right-hand side: the inner CG leaves it at zero
      const double rnorm = std::sqrt(rn[s]);
      sc[s] = 1.0 / rnorm;
      sc[QPX_MAX_RHS + s] = rnorm;
      // the reduction still missing, with a margin, within what the low
      // precision reaches on its own
      inner[s] = std::min(0.5, std::max(1e-5, 0.3 * std::sqrt(t2[s] / rn[s])));
    }
    QPX_CUDA(cudaMemcpyAsync(d_scales, sc.data(), sizeof(double) * 2 * QPX_MAX_RHS, cudaMemcpyHostToDevice,
                             lat->stream));
    convert_field(Rl, R, Coef{0, 0, d_scales, nullptr}, nullptr);
    BlasCall z;
    z.op = B_ZERO;
    z.x = Dl;
    blas_launch(lat, lp, ns, z);
    solve_cg(opl, Dl, Rl, inner.data(), max_iters, isign, cb, ii.data(), false, shifts);
    mv += ii[0].mv_apps;
    int its = 0;
    for (int s = 0; s < ns; s++) its = std::max(its, ii[s].n_iters);
    rit += its;
    convert_field(X, Dl, Coef{0, 0, d_scales + QPX_MAX_RHS, nullptr}, nullptr, 1);
    corr++;
  }
  for (int s = 0; s < ns; s++) convert_slice(prec, x[s]->sarg(), prec, slice_arg(X, s), lat);
  QPX_CUDA(cudaStreamSynchronize(lat->stream));
  *refine_iters = rit;
  *corrections = corr;
  *mv_apps = mv;
  bool all = true;
  for (int s = 0; s < ns; s++) {
    rel_sq_final[s] = bn > 0 ? rn[s] / bn : 0.0;
    all = all && done[s];
  }
  if (!all) throw Error(QPHIX_GPU_ENOTCONV, "mixed-precision multishift CG did not converge");
}

extern "C" int qphix_gpu_solve_mshift_cg_mixed(qphix_gpu_eo_op op, qphix_gpu_eo_op op_low, qphix_gpu_field *x,
                                               qphix_gpu_field rhs, int n_shift, const double *shifts,
                                               const double *rsd_target, const double *rsd_low, int max_iters,
                                               int isign, int cb, int *n_iters, int *refine_iters,
                                               int *corrections, double *rel_sq_final, unsigned long *mv_apps)
{
  return guard([&] {
    solve_mshift_mixed(op, op_low, x, rhs, n_shift, shifts, rsd_target, rsd_low, max_iters, isign, cb, n_iters,
                       refine_iters, corrections, rel_sq_final, mv_apps);
  });
}
