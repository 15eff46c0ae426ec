// Serving layer: a request loop over the solver library.
//
// A server keeps gauge ensembles resident on the device (FP64 links for the
// outer operator and the clover construction, low-precision links for the
// inner iterations) and runs up to `slots` solve requests at a time, each on
// a worker thread with its own lattice objects, CUDA stream and device
// memory, so that the kernels of different requests (different lattice
// sizes and operators) overlap on the GPU.  Request memory comes from one
// stream-ordered memory pool (allocation and release never synchronise the
// device) and is admitted against an HBM budget: waiting requests are taken
// in arrival order as soon as a slot and the budget allow; a request that
// does not fit may be passed by later, smaller ones at most `max_bypass`
// times before it blocks admission until it fits.
//
// Each request builds its operator on the device: the clover term from the
// resident FP64 links (clover leaf, then a 6x6 inverse per block), low-
// precision copies of it, and solves M x = b on the odd checkerboard with
// BiCGStab in the low precision with FP64 reliable updates (FP64 true
// residual and solution).  A request's arithmetic does not depend on what
// else runs: every reduction has a fixed order, so its result is the same
// alone and in a mix.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "qpx_finalize.cuh"
#include "qpx_host.h"

using namespace qpx;

namespace {

using clk = std::chrono::steady_clock;

double secs(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct Ensemble {
  int dims[4];
  qphix_gpu_lattice lat = nullptr;
  qphix_gpu_field g64 = nullptr, glow = nullptr;
  size_t bytes = 0;
};

struct Req {
  long long ticket = 0;
  qphix_gpu_request r;
  size_t bytes = 0;
  clk::time_point t_submit, t_start, t_end;
  bool done = false;
  qphix_gpu_request_result res;
  std::string error;
};

}  // namespace

struct qphix_gpu_server_s {
  qphix_gpu_server_config cfg;
  int device = 0;
  cudaMemPool_t pool = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> queue;
  std::map<long long, Req *> reqs;
  std::vector<std::unique_ptr<Ensemble>> ens;
  size_t resident = 0, reserved = 0, reserved_peak = 0;
  long long next_ticket = 1;
  int head_bypassed = 0;
  long long bypasses = 0, completed = 0, failed = 0;
  int running = 0, running_peak = 0;
  bool stop = false;
  std::vector<std::thread> workers;
};

namespace {

size_t spinor_bytes(int prec, long long stride, int nrhs)
{
  ChunkSpec c = spinor_spec(prec);
  size_t b = (size_t)c.nchunk * c.chunk_bytes * stride;
  if (prec == PREC_F16 || prec == PREC_BF16 || prec == PREC_Q16 || prec == PREC_Q16F32) b += sizeof(float) * stride;
  return b * nrhs;
}

size_t clover_bytes(int prec, long long stride, int nreal)
{
  ChunkSpec c = clover_spec(prec, nreal);
  return (size_t)c.nchunk * c.chunk_bytes * stride;
}

// every device allocation a request makes (an upper bound: transients are
// counted as if they were all live at once)
size_t request_bytes(const qphix_gpu_server_s *S, const Ensemble &e, const qphix_gpu_request &r)
{
  const long long vh = (long long)e.dims[0] / 2 * e.dims[1] * e.dims[2] * e.dims[3];
  const long long stride = (vh + 63) / 64 * 64;
  const int lp = S->cfg.low_prec, nr = r.nrhs;
  // reliable updates: x, b, two solver temporaries, the operator temporary
  // (FP64); six solver temporaries and the operator temporary (low precision).
  // Richardson: x, b, three outer temporaries, the operator temporary (FP64);
  // two correction fields, five BiCGStab temporaries and the operator
  // temporary (low precision)
  const bool rich = S->cfg.solver == QPHIX_GPU_SERVE_RICHARDSON;
  size_t b = (rich ? 6 : 5) * spinor_bytes(PREC_F64, stride, nr) + (rich ? 8 : 7) * spinor_bytes(lp, stride, nr);
  b += (size_t)nr * vh * 24 * sizeof(double);  // host-layout staging
  if (r.op_kind == QPHIX_GPU_CLOVER_OP)
    b += 3 * clover_bytes(PREC_F64, stride, 72) + 2 * clover_bytes(lp, stride, 72);
  else if (r.op_kind == QPHIX_GPU_TMCLOVER)
    b += 2 * clover_bytes(PREC_F64, stride, 72) + 2 * clover_bytes(PREC_F64, stride, 144) +
         clover_bytes(lp, stride, 72) + 2 * clover_bytes(lp, stride, 144);
  return b;
}

void ok(int rc)
{
  if (rc != QPHIX_GPU_OK) throw Error(rc, qphix_gpu_last_error());
}

// field and operator handles released at scope exit
struct Fields {
  std::vector<qphix_gpu_field> f;
  std::vector<qphix_gpu_eo_op> ops;
  qphix_gpu_field make(qphix_gpu_lattice L, int kind, int prec, int recon, int nrhs)
  {
    qphix_gpu_field h = nullptr;
    ok(qphix_gpu_field_create(L, kind, prec, recon, nrhs, &h));
    f.push_back(h);
    return h;
  }
  ~Fields()
  {
    for (auto o : ops) qphix_gpu_eo_op_destroy(o);
    for (auto h : f) qphix_gpu_field_destroy(h);
  }
};

qphix_gpu_host_layout canonical()
{
  qphix_gpu_host_layout h;
  memset(&h, 0, sizeof(h));
  h.kind = QPHIX_GPU_HOST_CANONICAL;
  h.ft = QPHIX_GPU_HOST_F64;
  return h;
}

struct Worker {
  qphix_gpu_server_s *S;
  std::map<std::string, qphix_gpu_lattice> lats;  // by lattice shape

  qphix_gpu_lattice lattice_for(const int d[4])
  {
    std::string k = std::to_string(d[0]) + "x" + std::to_string(d[1]) + "x" + std::to_string(d[2]) + "x" +
                    std::to_string(d[3]);
    auto it = lats.find(k);
    if (it != lats.end()) return it->second;
    qphix_gpu_lattice L = nullptr;
    ok(lattice_create_pooled(d, S->pool, &L));
    lats[k] = L;
    return L;
  }

  void run(Req *q)
  {
    const qphix_gpu_request &r = q->r;
    const Ensemble &e = *S->ens[r.ensemble];
    qphix_gpu_lattice L = lattice_for(e.dims);
    const int lp = S->cfg.low_prec, nr = r.nrhs;
    std::vector<qphix_gpu_solve_info> info(nr);
    try {
      Fields F;
      qphix_gpu_field x = F.make(L, QPHIX_GPU_SPINOR, PREC_F64, 0, nr);
      qphix_gpu_field b = F.make(L, QPHIX_GPU_SPINOR, PREC_F64, 0, nr);
      qphix_gpu_host_layout hl = canonical();
      ok(qphix_gpu_field_upload(b, r.rhs, &hl, 1, -1));

      qphix_gpu_op_params p;
      memset(&p, 0, sizeof(p));
      p.kind = r.op_kind;
      p.t_boundary = r.t_boundary;
      p.aniso_s = 1.0;
      p.aniso_t = 1.0;
      p.mass = r.mass;
      p.twisted_mass = r.twisted_mass;
      p.prec_mass_rho = (r.op_kind == QPHIX_GPU_TMCLOVER) ? r.twisted_mass : 0.0;
      qphix_gpu_field c64 = nullptr, i64 = nullptr, f064 = nullptr, f164 = nullptr;
      qphix_gpu_field cl = nullptr, il = nullptr, f0l = nullptr, f1l = nullptr;
      const double diag = 4.0 + r.mass;
      if (r.op_kind == QPHIX_GPU_CLOVER_OP || r.op_kind == QPHIX_GPU_TMCLOVER) {
        // A on the odd checkerboard (the operator's diagonal) and the inverse
        // of A (or of A +- i mu g5) on the even one
        c64 = F.make(L, QPHIX_GPU_CLOVER, PREC_F64, 0, 1);
        qphix_gpu_field ce = F.make(L, QPHIX_GPU_CLOVER, PREC_F64, 0, 1);
        ok(qphix_gpu_clover_build(c64, e.g64, 1, diag, r.csw, r.csw));
        ok(qphix_gpu_clover_build(ce, e.g64, 0, diag, r.csw, r.csw));
        cl = F.make(L, QPHIX_GPU_CLOVER, lp, 0, 1);
        ok(qphix_gpu_clover_convert(cl, c64));
        if (r.op_kind == QPHIX_GPU_CLOVER_OP) {
          i64 = F.make(L, QPHIX_GPU_CLOVER, PREC_F64, 0, 1);
          ok(qphix_gpu_clover_invert(i64, ce));
          il = F.make(L, QPHIX_GPU_CLOVER, lp, 0, 1);
          ok(qphix_gpu_clover_convert(il, i64));
        } else {
          f064 = F.make(L, QPHIX_GPU_FULLCLOVER, PREC_F64, 0, 1);
          f164 = F.make(L, QPHIX_GPU_FULLCLOVER, PREC_F64, 0, 1);
          ok(qphix_gpu_clover_invert_twisted(f064, f164, ce, r.twisted_mass));
          f0l = F.make(L, QPHIX_GPU_FULLCLOVER, lp, 0, 1);
          f1l = F.make(L, QPHIX_GPU_FULLCLOVER, lp, 0, 1);
          ok(qphix_gpu_clover_convert(f0l, f064));
          ok(qphix_gpu_clover_convert(f1l, f164));
        }
      }
      qphix_gpu_eo_op op64 = nullptr, opl = nullptr;
      ok(qphix_gpu_eo_op_create(&p, e.g64, c64, i64, f064, f164, &op64));
      F.ops.push_back(op64);
      ok(qphix_gpu_eo_op_create(&p, e.glow, cl, il, f0l, f1l, &opl));
      F.ops.push_back(opl);
      if (S->cfg.solver == QPHIX_GPU_SERVE_RICHARDSON)
        ok(qphix_gpu_solve_richardson(op64, opl, QPHIX_GPU_SOLVER_BICGSTAB, x, b, r.rsd_target, S->cfg.delta, 100,
                                      r.max_iters, 1, 1, info.data()));
      else
        ok(qphix_gpu_solve_bicgstab_mixed(op64, opl, x, b, r.rsd_target, S->cfg.delta, r.max_iters, 1, 1,
                                          info.data()));
      ok(qphix_gpu_field_download(x, r.x, &hl, -1));
    } catch (...) {
      lattice_trim(L);
      throw;
    }
    lattice_trim(L);
    qphix_gpu_request_result &res = q->res;
    res.status = QPHIX_GPU_OK;
    res.n_iters = 0;
    res.mv_apps = 0;
    res.true_rel_resid = 0.0;
    for (int i = 0; i < nr; i++) {
      if (info[i].n_iters > res.n_iters) res.n_iters = info[i].n_iters;
      if (info[i].mv_apps > res.mv_apps) res.mv_apps = info[i].mv_apps;
      if (info[i].true_rel_resid > res.true_rel_resid) res.true_rel_resid = info[i].true_rel_resid;
      if (info[i].status != 0 && res.status == QPHIX_GPU_OK) res.status = QPHIX_GPU_ENOTCONV;
    }
  }

  // next admissible request (caller holds S->mu), or nullptr
  Req *admit()
  {
    const size_t avail = S->cfg.hbm_budget_bytes > S->resident ? S->cfg.hbm_budget_bytes - S->resident : 0;
    for (size_t i = 0; i < S->queue.size(); i++) {
      Req *q = S->queue[i];
      if (S->reserved + q->bytes <= avail) {
        if (i == 0) {
          S->head_bypassed = 0;
        } else {
          S->head_bypassed++;
          S->bypasses++;
        }
        S->queue.erase(S->queue.begin() + i);
        S->reserved += q->bytes;
        if (S->reserved > S->reserved_peak) S->reserved_peak = S->reserved;
        return q;
      }
      if (i == 0 && S->head_bypassed >= S->cfg.max_bypass) return nullptr;
    }
    return nullptr;
  }

  void loop()
  {
    cudaSetDevice(S->device);
    for (;;) {
      Req *q = nullptr;
      {
        std::unique_lock<std::mutex> lk(S->mu);
        for (;;) {
          if (S->stop) return;
          q = admit();
          if (q) break;
          S->cv_work.wait(lk);
        }
        S->running++;
        if (S->running > S->running_peak) S->running_peak = S->running;
      }
      q->t_start = clk::now();
      std::string err;
      int rc = QPHIX_GPU_OK;
      try {
        run(q);
      } catch (const Error &e) {
        rc = e.code;
        err = e.what();
      } catch (const std::exception &e) {
        rc = QPHIX_GPU_ECUDA;
        err = e.what();
      }
      q->t_end = clk::now();
      {
        std::lock_guard<std::mutex> lk(S->mu);
        if (rc != QPHIX_GPU_OK) {
          q->res.status = rc;
          q->error = err;
        }
        q->res.queue_s = secs(q->t_submit, q->t_start);
        q->res.solve_s = secs(q->t_start, q->t_end);
        q->res.latency_s = secs(q->t_submit, q->t_end);
        q->res.bytes = q->bytes;
        q->done = true;
        S->reserved -= q->bytes;
        S->running--;
        S->completed++;
        if (q->res.status != QPHIX_GPU_OK) S->failed++;
      }
      S->cv_done.notify_all();
      S->cv_work.notify_all();
    }
  }

  ~Worker()
  {
    for (auto &kv : lats) qphix_gpu_lattice_destroy(kv.second);
  }
};

void check_request(qphix_gpu_server S, const qphix_gpu_request *r)
{
  if (!S || !r) throw Error(QPHIX_GPU_EINVAL, "null argument");
  if (r->ensemble < 0 || r->ensemble >= (int)S->ens.size()) throw Error(QPHIX_GPU_EINVAL, "unknown ensemble");
  if (r->op_kind < QPHIX_GPU_WILSON || r->op_kind > QPHIX_GPU_TMCLOVER)
    throw Error(QPHIX_GPU_EINVAL, "bad operator kind");
  if (r->nrhs < 1 || r->nrhs > QPX_MAX_RHS) throw Error(QPHIX_GPU_EINVAL, "nrhs must be in [1, 32]");
  if (!r->rhs || !r->x) throw Error(QPHIX_GPU_EINVAL, "null rhs or x");
  if (!(r->rsd_target > 0.0)) throw Error(QPHIX_GPU_EINVAL, "rsd_target must be positive");
  if (r->max_iters < 1) throw Error(QPHIX_GPU_EINVAL, "max_iters must be positive");
}

}  // namespace

extern "C" int qphix_gpu_server_create(const qphix_gpu_server_config *cfg, qphix_gpu_server *out)
{
  int rc = 0;
  qphix_gpu_server_s *S = nullptr;
  try {
    if (!cfg || !out) throw Error(QPHIX_GPU_EINVAL, "null argument");
    if (cfg->slots < 1 || cfg->slots > 64) throw Error(QPHIX_GPU_EINVAL, "slots must be in [1, 64]");
    if (cfg->low_prec != PREC_F32 && cfg->low_prec != PREC_F16 && cfg->low_prec != PREC_BF16 &&
        cfg->low_prec != PREC_Q16 && cfg->low_prec != PREC_Q16F32)
      throw Error(QPHIX_GPU_EINVAL, "low_prec must be F32, F16, BF16, Q16 or Q16F32");
    if (!(cfg->delta > 0.0 && cfg->delta < 1.0)) throw Error(QPHIX_GPU_EINVAL, "delta must be in (0, 1)");
    if (cfg->solver != QPHIX_GPU_SERVE_RELIABLE_UPDATE && cfg->solver != QPHIX_GPU_SERVE_RICHARDSON)
      throw Error(QPHIX_GPU_EINVAL, "solver must be QPHIX_GPU_SERVE_RELIABLE_UPDATE or _RICHARDSON");
    S = new qphix_gpu_server_s();
    S->cfg = *cfg;
    if (S->cfg.max_bypass < 0) S->cfg.max_bypass = 0;
    QPX_CUDA(cudaGetDevice(&S->device));
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = S->device;
    QPX_CUDA(cudaMemPoolCreate(&S->pool, &props));
    // keep released request memory reserved for the next request
    unsigned long long keep = cfg->hbm_budget_bytes;
    QPX_CUDA(cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    for (int i = 0; i < cfg->slots; i++)
      S->workers.emplace_back([S] {
        Worker w{S, {}};
        w.loop();
      });
    *out = S;
  } catch (const Error &e) {
    rc = qpx_set_last_error(e.what(), e.code);
    if (S) {
      if (S->pool) cudaMemPoolDestroy(S->pool);
      delete S;
    }
  }
  return rc;
}

extern "C" int qphix_gpu_server_add_ensemble(qphix_gpu_server S, const int dims[4], const double *gauge_canonical,
                                             int *ensemble_id)
{
  int rc = 0;
  auto e = std::make_unique<Ensemble>();
  try {
    if (!S || !dims || !gauge_canonical || !ensemble_id) throw Error(QPHIX_GPU_EINVAL, "null argument");
    for (int i = 0; i < 4; i++) e->dims[i] = dims[i];
    ok(qphix_gpu_lattice_create(dims, &e->lat));
    ok(qphix_gpu_field_create(e->lat, QPHIX_GPU_GAUGE, PREC_F64, 12, 1, &e->g64));
    ok(qphix_gpu_field_create(e->lat, QPHIX_GPU_GAUGE, S->cfg.low_prec, 12, 1, &e->glow));
    qphix_gpu_host_layout hl = canonical();
    ok(qphix_gpu_field_upload(e->g64, gauge_canonical, &hl, -1, -1));
    ok(qphix_gpu_field_upload(e->glow, gauge_canonical, &hl, -1, -1));
    ok(qphix_gpu_lattice_sync(e->lat));
    size_t b1 = 0, b2 = 0;
    ok(qphix_gpu_field_bytes(e->g64, &b1));
    ok(qphix_gpu_field_bytes(e->glow, &b2));
    e->bytes = b1 + b2;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->resident + e->bytes > S->cfg.hbm_budget_bytes)
      throw Error(QPHIX_GPU_ENOMEM, "ensemble does not fit in the server's HBM budget");
    S->resident += e->bytes;
    *ensemble_id = (int)S->ens.size();
    S->ens.push_back(std::move(e));
  } catch (const Error &err) {
    rc = qpx_set_last_error(err.what(), err.code);
    if (e) {
      qphix_gpu_field_destroy(e->g64);
      qphix_gpu_field_destroy(e->glow);
      qphix_gpu_lattice_destroy(e->lat);
    }
  }
  return rc;
}

extern "C" int qphix_gpu_server_request_bytes(qphix_gpu_server S, const qphix_gpu_request *r, size_t *bytes)
{
  try {
    if (!bytes || !S) throw Error(QPHIX_GPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    check_request(S, r);
    *bytes = request_bytes(S, *S->ens[r->ensemble], *r);
  } catch (const Error &e) {
    return qpx_set_last_error(e.what(), e.code);
  }
  return 0;
}

extern "C" int qphix_gpu_server_submit(qphix_gpu_server S, const qphix_gpu_request *r, long long *ticket)
{
  try {
    if (!ticket || !S) throw Error(QPHIX_GPU_EINVAL, "null argument");
    auto q = std::make_unique<Req>();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      check_request(S, r);
      q->r = *r;
      q->bytes = request_bytes(S, *S->ens[r->ensemble], *r);
      if (q->bytes + S->resident > S->cfg.hbm_budget_bytes)
        throw Error(QPHIX_GPU_ENOMEM, "request does not fit in the server's HBM budget");
      memset(&q->res, 0, sizeof(q->res));
      q->t_submit = clk::now();
      q->ticket = S->next_ticket++;
      *ticket = q->ticket;
      S->reqs[q->ticket] = q.get();
      S->queue.push_back(q.release());
    }
    S->cv_work.notify_one();
  } catch (const Error &e) {
    return qpx_set_last_error(e.what(), e.code);
  }
  return 0;
}

extern "C" int qphix_gpu_server_poll(qphix_gpu_server S, long long ticket, int *done)
{
  try {
    if (!S || !done) throw Error(QPHIX_GPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) throw Error(QPHIX_GPU_EINVAL, "unknown ticket");
    *done = it->second->done ? 1 : 0;
  } catch (const Error &e) {
    return qpx_set_last_error(e.what(), e.code);
  }
  return 0;
}

// Blocks until the request is done; fills `res` and forgets the ticket.  The
// return value is the request's own status (its error text in last_error).
extern "C" int qphix_gpu_server_wait(qphix_gpu_server S, long long ticket, qphix_gpu_request_result *res)
{
  Req *q = nullptr;
  try {
    if (!S || !res) throw Error(QPHIX_GPU_EINVAL, "null argument");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) throw Error(QPHIX_GPU_EINVAL, "unknown ticket");
    q = it->second;
    S->cv_done.wait(lk, [&] { return q->done; });
    S->reqs.erase(ticket);
  } catch (const Error &e) {
    return qpx_set_last_error(e.what(), e.code);
  }
  *res = q->res;
  int rc = q->res.status;
  if (rc != QPHIX_GPU_OK) qpx_set_last_error(q->error.empty() ? "solve did not converge" : q->error.c_str(), rc);
  delete q;
  return rc;
}

extern "C" int qphix_gpu_server_get_stats(qphix_gpu_server S, qphix_gpu_server_stats *st)
{
  try {
    if (!S || !st) throw Error(QPHIX_GPU_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    st->completed = S->completed;
    st->failed = S->failed;
    st->waiting = (long long)S->queue.size();
    st->bypasses = S->bypasses;
    st->running = S->running;
    st->running_peak = S->running_peak;
    st->resident_bytes = S->resident;
    st->reserved_bytes = S->reserved;
    st->reserved_peak_bytes = S->reserved_peak;
    unsigned long long used_hi = 0;
    QPX_CUDA(cudaMemPoolGetAttribute(S->pool, cudaMemPoolAttrUsedMemHigh, &used_hi));
    st->pool_used_peak_bytes = (size_t)used_hi;
  } catch (const Error &e) {
    return qpx_set_last_error(e.what(), e.code);
  }
  return 0;
}

// Finishes the requests already admitted, drops the waiting ones (their
// tickets become unknown) and frees everything.
extern "C" int qphix_gpu_server_destroy(qphix_gpu_server S)
{
  if (!S) return 0;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto &t : S->workers) t.join();
  for (auto *q : S->queue) {
    S->reqs.erase(q->ticket);
    delete q;
  }
  for (auto &kv : S->reqs) delete kv.second;
  for (auto &e : S->ens) {
    qphix_gpu_field_destroy(e->g64);
    qphix_gpu_field_destroy(e->glow);
    qphix_gpu_lattice_destroy(e->lat);
  }
  if (S->pool) cudaMemPoolDestroy(S->pool);
  delete S;
  return 0;
}
