// Drives the reference's own header-only code on canonical arrays, to pin the
// CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// Compiled (by oracle/ref/Makefile) against the unmodified QPhiX headers:
//   clover product   include/qphix/clover_product.h:47-346
//   BLAS             include/qphix/blas_new_c.h (+ site_loops.h, functors)
//   solvers          include/qphix/invcg.h, invbicgstab.h, invmr.h,
//                    minvcg.h, inv_richardson_multiprec.h
// with Geometry<double, 1, 1, false> (veclen = soalen = 1, no padding), for
// which the blocked host layout is site-major: spinor block s = cb-site s,
// element [colour][spin][re/im]; clover block s = the 72 canonical reals.
//
// The solvers are run on an operator supplied as a C callback working on
// canonical spinors (the oracle's even-odd operator): the solver recurrences
// are then the reference's, the operator the oracle's.
#include <omp.h>

#include <cstring>
#include <vector>

#include "qphix/blas_new_c.h"
#include "qphix/clover_product.h"
#include "qphix/geometry.h"
#include "qphix/inv_richardson_multiprec.h"
#include "qphix/invbicgstab.h"
#include "qphix/invcg.h"
#include "qphix/invmr.h"
#include "qphix/linearOp.h"
#include "qphix/minvcg.h"

using namespace QPhiX;

typedef Geometry<double, 1, 1, false> Geom;
typedef Geom::FourSpinorBlock Spinor;
typedef void (*apply_fn)(void *ctx, double *out, const double *in, int isign, int target_cb);

namespace {

Geom *make_geom(const int dims[4])
{
  int latt[4] = {dims[0], dims[1], dims[2], dims[3]};
  return new Geom(latt, 1, 1, 1, 1, 1, 0, 0, 1, false);
}

long vh(const Geom &g) { return (long)g.Nxh() * g.Ny() * g.Nz() * g.Nt(); }

// canonical [Vh][4][3][2] <-> blocked [Vh][3][4][2][1]
void to_blocked(const double *c, Spinor *b, long n)
{
  for (long s = 0; s < n; s++)
    for (int sp = 0; sp < 4; sp++)
      for (int col = 0; col < 3; col++)
        for (int ri = 0; ri < 2; ri++) b[s][col][sp][ri][0] = c[s * 24 + (sp * 3 + col) * 2 + ri];
}

void from_blocked(const Spinor *b, double *c, long n)
{
  for (long s = 0; s < n; s++)
    for (int sp = 0; sp < 4; sp++)
      for (int col = 0; col < 3; col++)
        for (int ri = 0; ri < 2; ri++) c[s * 24 + (sp * 3 + col) * 2 + ri] = b[s][col][sp][ri][0];
}

// EvenOddLinearOperator whose operator() is the oracle's (a C callback)
class CallbackOp : public EvenOddLinearOperator<double, 1, 1, false>
{
 public:
  CallbackOp(Geom &g, apply_fn f, void *ctx) : g_(g), f_(f), ctx_(ctx), n_(vh(g)), a_(24 * n_), b_(24 * n_) {}
  void operator()(Spinor *res, const Spinor *in, int isign, int target_cb = 1) const override
  {
    from_blocked(in, a_.data(), n_);
    f_(ctx_, b_.data(), a_.data(), isign, target_cb);
    to_blocked(b_.data(), res, n_);
    applications++;
  }
  void M_offdiag(Spinor *, const Spinor *, int, int) const override {}
  void M_diag_inv(Spinor *, const Spinor *, int, int) const override {}
  Geom &getGeometry() override { return g_; }
  mutable long applications = 0;

 private:
  Geom &g_;
  apply_fn f_;
  void *ctx_;
  long n_;
  mutable std::vector<double> a_, b_;
};

struct Fields {
  Geom *g;
  std::vector<Spinor *> sp;
  explicit Fields(const int dims[4]) : g(make_geom(dims)) {}
  Spinor *alloc()
  {
    sp.push_back(g->allocCBFourSpinor());
    return sp.back();
  }
  ~Fields()
  {
    for (auto *p : sp) g->free(p);
    delete g;
  }
};

}  // namespace

extern "C" {

// ---- clover product (include/qphix/clover_product.h:250-346) -------------
void ref_clover_apply(const int dims[4], double *out, const double *in, const double *clov, int full)
{
  omp_set_num_threads(1);
  Fields F(dims);
  long n = vh(*F.g);
  Spinor *x = F.alloc(), *y = F.alloc();
  to_blocked(in, x, n);
  if (full) {
    Geom::FullCloverBlock *c = (Geom::FullCloverBlock *)F.g->allocCBFullClov();
    std::memcpy(c, clov, sizeof(double) * 144 * n);
    clover_product(y, x, c, *F.g);
    F.g->free(c);
  } else {
    Geom::CloverBlock *c = (Geom::CloverBlock *)F.g->allocCBClov();
    std::memcpy(c, clov, sizeof(double) * 72 * n);
    clover_product(y, x, c, *F.g);
    F.g->free(c);
  }
  from_blocked(y, out, n);
}

// ---- BLAS ----------------------------------------------------------------
// op 0: norm2(x); 1: innerProduct(x, y); 2: axpy(a, x, y); 3: caxpy(a, x, y);
// 4: xmyNorm2(res = x - y); 5: axpby(a, x, b, y); 6: aypx(a, x, y)
void ref_blas(const int dims[4], int op, const double *a, const double *b, const double *x, double *y,
              double *res_out, double *scalar_out)
{
  omp_set_num_threads(1);
  Fields F(dims);
  long n = vh(*F.g);
  Spinor *bx = F.alloc(), *by = F.alloc(), *br = F.alloc();
  to_blocked(x, bx, n);
  to_blocked(y, by, n);
  int nt = F.g->getNSIMT();
  switch (op) {
  case 0: norm2Spinor<double, 1, 1, false>(scalar_out[0], bx, *F.g, nt); break;
  case 1: innerProduct<double, 1, 1, false>(scalar_out, bx, by, *F.g, nt); break;
  case 2: axpy<double, 1, 1, false>(a[0], bx, by, *F.g, nt); break;
  case 3: {
    double ac[2] = {a[0], a[1]};
    caxpySpinor<double, 1, 1, false>(ac, bx, by, *F.g, nt);
    break;
  }
  case 4: xmyNorm2Spinor<double, 1, 1, false>(br, bx, by, scalar_out[0], *F.g, nt); break;
  case 5: axpby<double, 1, 1, false>(a[0], bx, b[0], by, *F.g, nt); break;
  case 6: aypx<double, 1, 1, false>(a[0], bx, by, *F.g, nt); break;
  }
  from_blocked(op == 4 ? br : by, res_out, n);
}

// ---- solvers -------------------------------------------------------------
// kind 0 CG, 1 BiCGStab, 2 MR (omega); returns n_iters, rsd_sq_final, mv_apps
void ref_solve(const int dims[4], int kind, apply_fn f, void *ctx, double *x, const double *rhs, double rsd,
               int max_iters, double omega, int isign, int cb, int *n_iters, double *rsd_sq_final,
               unsigned long *mv_apps)
{
  omp_set_num_threads(1);
  Fields F(dims);
  long n = vh(*F.g);
  CallbackOp M(*F.g, f, ctx);
  Spinor *bx = F.alloc(), *bb = F.alloc();
  to_blocked(x, bx, n);
  to_blocked(rhs, bb, n);
  unsigned long site_flops = 0;
  *rsd_sq_final = -1;
  if (kind == 0) {
    InvCG<double, 1, 1, false> s(M, max_iters);
    s(bx, bb, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  } else if (kind == 1) {
    InvBiCGStab<double, 1, 1, false> s(M, max_iters);
    s(bx, bb, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  } else {
    InvMR<double, 1, 1, false> s(M, max_iters, omega);
    s(bx, bb, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  }
  from_blocked(bx, x, n);
}

// Richardson (FP64 outer, BiCGStab inner on the same operator in FP64)
void ref_richardson(const int dims[4], apply_fn f, void *ctx, double *x, const double *rhs, double rsd,
                    double delta, int max_iters, int inner_max, int isign, int cb, int *n_iters,
                    double *rsd_sq_final, unsigned long *mv_apps)
{
  omp_set_num_threads(1);
  Fields F(dims);
  long n = vh(*F.g);
  CallbackOp M(*F.g, f, ctx);
  Spinor *bx = F.alloc(), *bb = F.alloc();
  to_blocked(x, bx, n);
  to_blocked(rhs, bb, n);
  InvBiCGStab<double, 1, 1, false> inner(M, inner_max);
  InvRichardsonMultiPrec<double, 1, 1, false, double, 1, 1, false> s(M, inner, delta, max_iters);
  Spinor *xa[1] = {bx};
  const Spinor *ba[1] = {bb};
  unsigned long site_flops = 0;
  s(xa, ba, rsd, *n_iters, *rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  from_blocked(bx, x, n);
}

// multishift CG (include/qphix/minvcg.h:77-387)
void ref_minvcg(const int dims[4], apply_fn f, void *ctx, double **x, const double *rhs, int n_shift,
                const double *shifts, const double *rsd, int max_iters, int isign, int cb, int *n_iters,
                double *rsd_sq_final, unsigned long *mv_apps)
{
  omp_set_num_threads(1);
  Fields F(dims);
  long n = vh(*F.g);
  CallbackOp M(*F.g, f, ctx);
  std::vector<Spinor *> xs(n_shift);
  for (int i = 0; i < n_shift; i++) xs[i] = F.alloc();
  Spinor *bb = F.alloc();
  to_blocked(rhs, bb, n);
  MInvCG<double, 1, 1, false> s(M, max_iters, n_shift);
  unsigned long site_flops = 0;
  s(xs.data(), bb, n_shift, shifts, rsd, *n_iters, rsd_sq_final, site_flops, *mv_apps, isign, false, cb);
  for (int i = 0; i < n_shift; i++) from_blocked(xs[i], x[i], n);
}

}  // extern "C"
