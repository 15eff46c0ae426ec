// Drives QPhiX's own code-generated Dslash family, even-odd operators and
// Krylov solvers on host arrays in QPhiX's blocked layout -- TEST
// INFRASTRUCTURE AND CPU BASELINE ONLY.
//
// Compiled by oracle/ref/codegen.mk against the unmodified reference headers
// and the kernels its code generator emits (codegen/dslash_common.cc,
// driven by include/qphix/dslash_body.h, clover_dslash_body.h,
// tm_dslash_body.h, tm_clov_dslash_body.h):
//   Dslash::dslash / dslashAChiMinusBDPsi / dslashDir   dslash_def.h:36-58
//   ClovDslash::dslash / dslashAChiMinusBDPsi / clovMult clover_dslash_def.h:33-53
//   TMDslash::dslash / dslashAChiMinusBDPsi             tm_dslash_def.h:33-49
//   TMClovDslash::dslash / dslashAChiMinusBDPsi         tm_clov_dslash_def.h:44-66
//   EvenOdd{Wilson,Clover,TMWilson,TMClover}Operator    wilson.h:49, clover.h:162,
//                                                       twisted_mass.h:62,
//                                                       twisted_mass_clover.h:92
//   InvCG, InvBiCGStab, InvRichardsonMultiPrec          invcg.h:88, invbicgstab.h:80,
//                                                       inv_richardson_multiprec.h:42
//
// Every array crosses this boundary exactly as Geometry<FT,V,S,c12> allocates
// it (no padding): a spinor is spinor_bytes including its leading pad block,
// a gauge checkerboard gauge_bytes, a clover term clover_bytes, a full clover
// block full_clover_bytes (geometry.h:171-175).  The caller builds them (the
// test suite with qphix_b200.fields.QPhiXLayout), so the reference's kernels
// also check that packer.
#include <fcntl.h>
#include <omp.h>
#include <unistd.h>

#include <cstring>
#include <memory>

#include "qphix/clover.h"
#include "qphix/clover_dslash_def.h"
#include "qphix/dslash_def.h"
#include "qphix/geometry.h"
#include "qphix/inv_richardson_multiprec.h"
#include "qphix/invbicgstab.h"
#include "qphix/invcg.h"
#include "qphix/tm_clov_dslash_def.h"
#include "qphix/tm_dslash_def.h"
#include "qphix/twisted_mass_clover.h"
#include "qphix/wilson.h"

using namespace QPhiX;

namespace {

enum { K_WILSON = 0, K_CLOVER = 1, K_TM = 2, K_TMCLOVER = 3 };
enum { OP_DSLASH = 0, OP_ACHIMBDPSI = 1, OP_CLOVMULT = 2, OP_EO = 3, OP_DIR = 4 };
enum { S_CG = 0, S_BICGSTAB = 1, S_RICHARDSON = 2 };
// parameter vector: t_boundary, aniso_s, aniso_t, mass, twisted_mass, rho,
// alpha, beta, musign, dir
enum { P_TBC = 0, P_AS, P_AT, P_MASS, P_MU, P_RHO, P_ALPHA, P_BETA, P_MUSIGN, P_DIR };

// The reference prints progress from its solvers and constructors; the
// callers of this library read stdout for their own results.
struct QuietStdout {
  int saved;
  QuietStdout()
  {
    fflush(stdout);
    saved = dup(1);
    int nul = open("/dev/null", O_WRONLY);
    dup2(nul, 1);
    close(nul);
  }
  ~QuietStdout()
  {
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

int pick_block(int n, int ngy)
{
  // By (and Bz with ngy = 1) must divide n and be a multiple of ngy
  // (dslash_body.h:74-85); 4 as in the reference's timing programs.
  for (int b : {4, 2, 1})
    if (b % ngy == 0 && n % b == 0) return b;
  return ngy;
}

template <typename FT, int V, int S, bool C12>
struct Fields {
  typedef Geometry<FT, V, S, C12> Geom;
  typedef typename Geom::FourSpinorBlock Spinor;
  typedef typename Geom::SU3MatrixBlock Gauge;
  typedef typename Geom::CloverBlock Clover;
  typedef typename Geom::FullCloverBlock FullClover;

  std::unique_ptr<Geom> g;
  std::vector<Spinor *> sp;
  std::vector<Gauge *> ga;
  std::vector<Clover *> cl;
  std::vector<FullClover *> fc;

  // Geometry's allocation sizes (geometry.h:171-175), which it keeps private
  long n_blocks() const { return (long)g->getPxyz() * g->Nt(); }
  size_t spinor_bytes() const { return (n_blocks() + 1) * sizeof(Spinor); }
  size_t gauge_bytes() const { return (n_blocks() * S / V) * sizeof(Gauge); }
  size_t clover_bytes() const { return (n_blocks() * S / V) * sizeof(Clover); }
  size_t full_clover_bytes() const { return (n_blocks() * S / V) * sizeof(FullClover); }

  Fields(const int dims[4], int nthreads)
  {
    int latt[4] = {dims[0], dims[1], dims[2], dims[3]};
    const int ngy = V / S;
    g.reset(new Geom(latt, pick_block(dims[1], ngy), pick_block(dims[2], 1), nthreads, 1, 1, 0, 0, 1, false));
  }
  ~Fields()
  {
    for (auto *p : sp) g->free(p);
    for (auto *p : ga) g->free(p);
    for (auto *p : cl) g->free(p);
    for (auto *p : fc) g->free(p);
  }
  Spinor *spinor(const void *src = nullptr)
  {
    Spinor *p = g->allocCBFourSpinor();
    if (src) std::memcpy((void *)(p - 1), src, spinor_bytes());
    sp.push_back(p);
    return p;
  }
  void spinor_out(const Spinor *p, void *dst) const { std::memcpy(dst, (const void *)(p - 1), spinor_bytes()); }
  Gauge *gauge(const void *src)
  {
    if (!src) return nullptr;
    Gauge *p = g->allocCBGauge();
    std::memcpy((void *)p, src, gauge_bytes());
    ga.push_back(p);
    return p;
  }
  Clover *clover(const void *src)
  {
    if (!src) return nullptr;
    Clover *p = g->allocCBClov();
    std::memcpy((void *)p, src, clover_bytes());
    cl.push_back(p);
    return p;
  }
  FullClover *full_clover(const void *src)
  {
    if (!src) return nullptr;
    FullClover *p = g->allocCBFullClov();
    std::memcpy((void *)p, src, full_clover_bytes());
    fc.push_back(p);
    return p;
  }
};

// EvenOddTMWilsonOperator (twisted_mass.h:22-77) does not compile: its
// M_diag_inv is marked override with a signature the base class lacks
// (twisted_mass.h:89 lacks the cb argument of linearOp.h:33-35).  This class makes the same two TMDslash
// calls as its operator() (twisted_mass.h:62-77) with the same alpha = 4 + m
// and beta = 0.25 (twisted_mass.h:31-32).
template <typename FT, int V, int S, bool C12>
class TMWilsonEO : public EvenOddLinearOperator<FT, V, S, C12>
{
 public:
  typedef typename Geometry<FT, V, S, C12>::FourSpinorBlock Spinor;
  typedef typename Geometry<FT, V, S, C12>::SU3MatrixBlock Gauge;
  TMWilsonEO(double mass, double mu, Gauge *u_[2], Geometry<FT, V, S, C12> *geom, double tbc, double as, double at)
      : D(geom, tbc, as, at, mass, mu), alpha(4.0 + mass), beta(0.25)
  {
    u[0] = u_[0];
    u[1] = u_[1];
    tmp = geom->allocCBFourSpinor();
  }
  ~TMWilsonEO() { D.getGeometry().free(tmp); }
  void operator()(Spinor *res, const Spinor *in, int isign, int target_cb = 1) const override
  {
    int source_cb = 1 - target_cb;
    D.dslash(tmp, in, u[source_cb], isign, source_cb);
    D.dslashAChiMinusBDPsi(res, tmp, in, u[target_cb], alpha, beta, isign, target_cb);
  }
  void M_offdiag(Spinor *, const Spinor *, int, int) const override {}
  void M_diag_inv(Spinor *, const Spinor *, int, int) const override {}
  Geometry<FT, V, S, C12> &getGeometry() override { return D.getGeometry(); }

 private:
  mutable TMDslash<FT, V, S, C12> D;
  Gauge *u[2];
  Spinor *tmp;
  double alpha, beta;
};

// the even-odd operator of `kind` over fields already in F
template <typename FT, int V, int S, bool C12>
std::unique_ptr<EvenOddLinearOperator<FT, V, S, C12>> make_eo_op(Fields<FT, V, S, C12> &F, int kind,
                                                                 const double *p, const void *u0,
                                                                 const void *u1, const void *c0,
                                                                 const void *c1, const void *c2)
{
  typedef typename Fields<FT, V, S, C12>::Gauge Gauge;
  typedef typename Fields<FT, V, S, C12>::FullClover FullClover;
  Gauge *u[2] = {F.gauge(u0), F.gauge(u1)};
  auto *geom = F.g.get();
  switch (kind) {
  case K_WILSON:
    return std::unique_ptr<EvenOddLinearOperator<FT, V, S, C12>>(
        new EvenOddWilsonOperator<FT, V, S, C12>(p[P_MASS], u, geom, p[P_TBC], p[P_AS], p[P_AT]));
  case K_CLOVER:
    // clov = A on the odd (target) checkerboard, invclov = A^-1 on the even one
    return std::unique_ptr<EvenOddLinearOperator<FT, V, S, C12>>(new EvenOddCloverOperator<FT, V, S, C12>(
        u, F.clover(c0), F.clover(c1), geom, p[P_TBC], p[P_AS], p[P_AT], nullptr, nullptr, p[P_RHO]));
  case K_TM:
    return std::unique_ptr<EvenOddLinearOperator<FT, V, S, C12>>(
        new TMWilsonEO<FT, V, S, C12>(p[P_MASS], p[P_MU], u, geom, p[P_TBC], p[P_AS], p[P_AT]));
  case K_TMCLOVER: {
    FullClover *inv[2] = {F.full_clover(c1), F.full_clover(c2)};
    return std::unique_ptr<EvenOddLinearOperator<FT, V, S, C12>>(new EvenOddTMCloverOperator<FT, V, S, C12>(
        u, F.clover(c0), inv, geom, p[P_TBC], p[P_AS], p[P_AT], nullptr, nullptr, p[P_RHO]));
  }
  }
  return nullptr;
}

template <typename FT, int V, int S, bool C12>
int apply(const int dims[4], int nthreads, int kind, int op, const double *p, void *res, const void *psi,
          const void *chi, const void *u0, const void *u1, const void *c0, const void *c1, const void *c2,
          int isign, int cb)
{
  QuietStdout quiet;
  omp_set_num_threads(nthreads);
  Fields<FT, V, S, C12> F(dims, nthreads);
  auto *geom = F.g.get();
  auto *out = F.spinor();
  auto *in = F.spinor(psi);
  auto *x = chi ? F.spinor(chi) : nullptr;
  const void *ucb = cb == 0 ? u0 : u1;
  if (op == OP_EO) {
    auto M = make_eo_op<FT, V, S, C12>(F, kind, p, u0, u1, c0, c1, c2);
    if (!M) return -1;
    (*M)(out, in, isign, cb);
  } else if (kind == K_WILSON) {
    Dslash<FT, V, S, C12> D(geom, p[P_TBC], p[P_AS], p[P_AT]);
    if (op == OP_DSLASH)
      D.dslash(out, in, F.gauge(ucb), isign, cb);
    else if (op == OP_ACHIMBDPSI)
      D.dslashAChiMinusBDPsi(out, in, x, F.gauge(ucb), p[P_ALPHA], p[P_BETA], isign, cb);
    else if (op == OP_DIR)
      D.dslashDir(out, in, F.gauge(ucb), cb, (int)p[P_DIR]);
    else
      return -1;
  } else if (kind == K_CLOVER) {
    ClovDslash<FT, V, S, C12> D(geom, p[P_TBC], p[P_AS], p[P_AT], nullptr, nullptr, p[P_RHO]);
    if (op == OP_DSLASH)
      D.dslash(out, in, F.gauge(ucb), F.clover(c0), isign, cb);
    else if (op == OP_ACHIMBDPSI)
      D.dslashAChiMinusBDPsi(out, in, x, F.gauge(ucb), F.clover(c0), p[P_BETA], isign, cb);
    else if (op == OP_CLOVMULT)
      D.clovMult(out, in, F.clover(c0));
    else
      return -1;
  } else if (kind == K_TM) {
    TMDslash<FT, V, S, C12> D(geom, p[P_TBC], p[P_AS], p[P_AT], p[P_MASS], p[P_MU]);
    if (op == OP_DSLASH)
      D.dslash(out, in, F.gauge(ucb), isign, cb);
    else if (op == OP_ACHIMBDPSI)
      D.dslashAChiMinusBDPsi(out, in, x, F.gauge(ucb), p[P_ALPHA], p[P_BETA], isign, cb, p[P_MUSIGN]);
    else
      return -1;
  } else if (kind == K_TMCLOVER) {
    TMClovDslash<FT, V, S, C12> D(geom, p[P_TBC], p[P_AS], p[P_AT], nullptr, nullptr, p[P_RHO]);
    if (op == OP_DSLASH) {
      typename Fields<FT, V, S, C12>::FullClover *inv[2] = {F.full_clover(c0), F.full_clover(c1)};
      D.dslash(out, in, F.gauge(ucb), inv, isign, cb);
    } else if (op == OP_ACHIMBDPSI) {
      D.dslashAChiMinusBDPsi(out, in, x, F.gauge(ucb), F.clover(c0), p[P_BETA], isign, cb);
    } else {
      return -1;
    }
  } else {
    return -1;
  }
  F.spinor_out(out, res);
  return 0;
}

template <typename FT, int V, int S, bool C12>
int solve(const int dims[4], int nthreads, int kind, int solver, const double *p, const void *u0, const void *u1,
          const void *c0, const void *c1, const void *c2, void *x, const void *rhs, double rsd, int max_iters,
          int isign, int cb, int *n_iters, double *rsd_sq_final, unsigned long *mv_apps, double *seconds)
{
  QuietStdout quiet;
  omp_set_num_threads(nthreads);
  Fields<FT, V, S, C12> F(dims, nthreads);
  auto M = make_eo_op<FT, V, S, C12>(F, kind, p, u0, u1, c0, c1, c2);
  if (!M) return -1;
  auto *bx = F.spinor(x);
  auto *bb = F.spinor(rhs);
  unsigned long site_flops = 0;
  *rsd_sq_final = -1;
  double t0 = omp_get_wtime();
  if (solver == S_CG) {
    InvCG<FT, V, S, C12> s(*M, max_iters);
    s(bx, bb, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  } else if (solver == S_BICGSTAB) {
    InvBiCGStab<FT, V, S, C12> s(*M, max_iters);
    s(bx, bb, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  } else {
    return -1;
  }
  *seconds = omp_get_wtime() - t0;
  F.spinor_out(bx, x);
  return 0;
}

// InvRichardsonMultiPrec: FT outer (operator on the outer fields) around an
// FTI BiCGStab on the inner-precision copies of the same fields
// (inv_richardson_multiprec.h:42-239).
template <typename FT, int V, int S, bool C12, typename FTI, int VI, int SI>
int solve_richardson(const int dims[4], int nthreads, int kind, const double *p, const void *const *outer,
                     const void *const *inner, void *x, const void *rhs, double rsd, double delta, int max_iters,
                     int inner_max, int isign, int cb, int *n_iters, double *rsd_sq_final,
                     unsigned long *mv_apps, double *seconds)
{
  QuietStdout quiet;
  omp_set_num_threads(nthreads);
  Fields<FT, V, S, C12> F(dims, nthreads);
  Fields<FTI, VI, SI, C12> FI(dims, nthreads);
  auto M = make_eo_op<FT, V, S, C12>(F, kind, p, outer[0], outer[1], outer[2], outer[3], outer[4]);
  auto MI = make_eo_op<FTI, VI, SI, C12>(FI, kind, p, inner[0], inner[1], inner[2], inner[3], inner[4]);
  if (!M || !MI) return -1;
  auto *bx = F.spinor(x);
  auto *bb = F.spinor(rhs);
  InvBiCGStab<FTI, VI, SI, C12> in_solver(*MI, inner_max);
  InvRichardsonMultiPrec<FT, V, S, C12, FTI, VI, SI, C12> s(*M, in_solver, delta, max_iters);
  typename Fields<FT, V, S, C12>::Spinor *xa[1] = {bx};
  const typename Fields<FT, V, S, C12>::Spinor *ba[1] = {bb};
  unsigned long site_flops = 0;
  double t0 = omp_get_wtime();
  s(xa, ba, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  *seconds = omp_get_wtime() - t0;
  F.spinor_out(bx, x);
  return 0;
}

template <typename FT, int V, int S, bool C12>
void sizes(const int dims[4], long out[4])
{
  Fields<FT, V, S, C12> F(dims, 1);
  out[0] = F.spinor_bytes();
  out[1] = F.gauge_bytes();
  out[2] = F.clover_bytes();
  out[3] = F.full_clover_bytes();
}

// (precision, V, S) triples built into this library: prec 0 = double, 1 = float
#if defined(QPHIX_REF_ISA_AVX512)
#define REFK_VARIANTS(X) X(0, double, 8, 4) X(0, double, 8, 8) X(1, float, 16, 8)
#else
#define REFK_VARIANTS(X) X(0, double, 1, 1) X(1, float, 1, 1)
#endif

}  // namespace

extern "C" {

// The (precision, veclen, soalen) variants compiled in, as triples; returns
// how many there are.
int refk_variants(int *out, int max)
{
  int n = 0;
#define X(P, T, V, S)      \
  if (n < max) {           \
    out[3 * n + 0] = P;    \
    out[3 * n + 1] = V;    \
    out[3 * n + 2] = S;    \
  }                        \
  n++;
  REFK_VARIANTS(X)
#undef X
  return n;
}

// Geometry's allocation sizes in bytes: spinor (with its pad block), gauge
// checkerboard, clover term, full clover block.
int refk_sizes(int prec, int V, int S, int c12, const int dims[4], long out[4])
{
#define X(P, T, VV, SS)                                   \
  if (prec == P && V == VV && S == SS) {                  \
    if (c12)                                              \
      sizes<T, VV, SS, true>(dims, out);                  \
    else                                                  \
      sizes<T, VV, SS, false>(dims, out);                 \
    return 0;                                             \
  }
  REFK_VARIANTS(X)
#undef X
  return -1;
}

// One operator application.  kind: 0 Wilson, 1 clover, 2 twisted mass,
// 3 twisted-mass clover.  op: 0 dslash, 1 dslashAChiMinusBDPsi, 2 clovMult,
// 3 even-odd operator (target checkerboard cb), 4 dslashDir (p[9] = dir).
// Clover inputs: clover dslash c0 = A^-1; clover / TM-clover achimbdpsi and
// clovMult c0 = A; TM-clover dslash c0, c1 = the two full inverses; even-odd
// clover c0 = A (odd), c1 = A^-1 (even); even-odd TM clover c0 = A (odd),
// c1, c2 = the two full inverses (even).  u0 / u1 are the two checkerboards.
int refk_apply(int prec, int V, int S, int c12, const int dims[4], int nthreads, int kind, int op,
               const double *p, void *res, const void *psi, const void *chi, const void *u0, const void *u1,
               const void *c0, const void *c1, const void *c2, int isign, int cb)
{
#define X(P, T, VV, SS)                                                                                    \
  if (prec == P && V == VV && S == SS) {                                                                   \
    if (c12)                                                                                               \
      return apply<T, VV, SS, true>(dims, nthreads, kind, op, p, res, psi, chi, u0, u1, c0, c1, c2, isign, cb); \
    return apply<T, VV, SS, false>(dims, nthreads, kind, op, p, res, psi, chi, u0, u1, c0, c1, c2, isign, cb);  \
  }
  REFK_VARIANTS(X)
#undef X
  return -2;
}

// A full even-odd solve with the reference's InvCG (on M^dagger M) or
// InvBiCGStab (on M); x is the initial guess on entry and the solution on
// exit.  seconds = wall time of the solver call alone.
int refk_solve(int prec, int V, int S, int c12, const int dims[4], int nthreads, int kind, int solver,
               const double *p, const void *u0, const void *u1, const void *c0, const void *c1, const void *c2,
               void *x, const void *rhs, double rsd, int max_iters, int isign, int cb, int *n_iters,
               double *rsd_sq_final, unsigned long *mv_apps, double *seconds)
{
#define X(P, T, VV, SS)                                                                                       \
  if (prec == P && V == VV && S == SS) {                                                                      \
    if (c12)                                                                                                  \
      return solve<T, VV, SS, true>(dims, nthreads, kind, solver, p, u0, u1, c0, c1, c2, x, rhs, rsd, max_iters, \
                                    isign, cb, n_iters, rsd_sq_final, mv_apps, seconds);                     \
    return solve<T, VV, SS, false>(dims, nthreads, kind, solver, p, u0, u1, c0, c1, c2, x, rhs, rsd, max_iters,  \
                                   isign, cb, n_iters, rsd_sq_final, mv_apps, seconds);                      \
  }
  REFK_VARIANTS(X)
#undef X
  return -2;
}

// InvRichardsonMultiPrec with a double outer operator on the (V, S) layout
// and a float inner BiCGStab on the float variant of this build; outer[] and
// inner[] hold u0, u1, c0, c1, c2 of the two precisions.
int refk_solve_richardson(int V, int S, int c12, const int dims[4], int nthreads, int kind, const double *p,
                          const void *const *outer, const void *const *inner, void *x, const void *rhs, double rsd,
                          double delta, int max_iters, int inner_max, int isign, int cb, int *n_iters,
                          double *rsd_sq_final, unsigned long *mv_apps, double *seconds)
{
#if defined(QPHIX_REF_ISA_AVX512)
  if (V == 8 && S == 8) {
    if (c12)
      return solve_richardson<double, 8, 8, true, float, 16, 8>(dims, nthreads, kind, p, outer, inner, x, rhs, rsd,
                                                                delta, max_iters, inner_max, isign, cb, n_iters,
                                                                rsd_sq_final, mv_apps, seconds);
    return solve_richardson<double, 8, 8, false, float, 16, 8>(dims, nthreads, kind, p, outer, inner, x, rhs, rsd,
                                                               delta, max_iters, inner_max, isign, cb, n_iters,
                                                               rsd_sq_final, mv_apps, seconds);
  }
#else
  if (V == 1 && S == 1) {
    if (c12)
      return solve_richardson<double, 1, 1, true, float, 1, 1>(dims, nthreads, kind, p, outer, inner, x, rhs, rsd,
                                                               delta, max_iters, inner_max, isign, cb, n_iters,
                                                               rsd_sq_final, mv_apps, seconds);
    return solve_richardson<double, 1, 1, false, float, 1, 1>(dims, nthreads, kind, p, outer, inner, x, rhs, rsd,
                                                              delta, max_iters, inner_max, isign, cb, n_iters,
                                                              rsd_sq_final, mv_apps, seconds);
  }
#endif
  return -2;
}

}  // extern "C"
