// Drop-in solver interfaces (reference: include/qphix/abs_solver.h:13-267):
// ResiduumType, AbstractSolver and AbstractMultiSolver with the same
// operator() signatures.  The concrete solvers run on the device operator of
// the EvenOddLinearOperator they are given.
#pragma once

#include <cmath>

#include "qphix/full_spinor.h"
#include "qphix/linearOp.h"

namespace QPhiX
{

enum ResiduumType { ABSOLUTE, RELATIVE, INVALID };

template <typename FT, int V, int S, bool compress12, int num_flav = 1>
class AbstractSolver
{
 public:
  virtual ~AbstractSolver() {}
  typedef typename Geometry<FT, V, S, compress12>::FourSpinorBlock Spinor;

  virtual void operator()(Spinor *const x[num_flav], const Spinor *const rhs[num_flav], const double RsdTarget,
                          int &niters, double &rsd_sq_final, unsigned long &site_flops, unsigned long &mv_apps,
                          int isign, bool verboseP, int cb = 1, ResiduumType residType = RELATIVE) const = 0;

  void operator()(Spinor *x, const Spinor *rhs, const double RsdTarget, int &niters, double &rsd_sq_final,
                  unsigned long &site_flops, unsigned long &mv_apps, int isign, bool verboseP, int cb = 1,
                  ResiduumType residType = RELATIVE) const
  {
    Spinor *xa[1] = {x};
    const Spinor *ra[1] = {rhs};
    (*this)(xa, ra, RsdTarget, niters, rsd_sq_final, site_flops, mv_apps, isign, verboseP, cb, residType);
  }

  virtual Geometry<FT, V, S, compress12> &getGeometry() = 0;

  // device description of this solver, used by InvRichardsonMultiPrec for
  // its inner solve (not part of QPhiX's interface)
  virtual int gpu_solver_kind() const = 0;
  virtual qphix_gpu_eo_op gpu_solver_op() const = 0;
  virtual int gpu_max_iters() const = 0;
};

template <typename FT, int V, int S, bool compress12, int num_flav = 1>
class AbstractMultiSolver
{
 public:
  virtual ~AbstractMultiSolver() {}
  typedef typename Geometry<FT, V, S, compress12>::FourSpinorBlock Spinor;

  virtual void operator()(Spinor **x, const Spinor *rhs, const int n_shift, const double *shifts,
                          const double *RsdTarget, int &niters, double *rsd_sq_final, unsigned long &site_flops,
                          unsigned long &mv_apps, int isign, bool verboseP, int cb = 1) const = 0;
  virtual Geometry<FT, V, S, compress12> &getGeometry() = 0;
};

// reference: include/qphix/abs_solver.h:271-438 (AbstractUnprecSolver): solves the
// unpreconditioned system M x = b on both checkerboards with an even-odd
// solver: prepare the source, solve on solve_cb, reconstruct the other
// checkerboard
template <typename FT, int V, int S, bool compress12, int num_flav = 1>
class AbstractUnprecSolver
{
 public:
  using Spinor = FullSpinor<FT, V, S, compress12>;
  using CBSpinor = typename Spinor::CBSpinor;

  virtual ~AbstractUnprecSolver() {}
  virtual AbstractSolver<FT, V, S, compress12> &getEOSolver() const = 0;
  virtual void SourcePrepare(CBSpinor *const out[num_flav], CBSpinor const *const in_cb[num_flav],
                             CBSpinor const *const in_other_cb[num_flav], int isign, int solve_cb) const = 0;
  virtual void SolutionReconstruct(CBSpinor *const out_other_cb[num_flav], CBSpinor const *const in_other_cb[num_flav],
                                   CBSpinor const *const out_cb[num_flav], int isign, int solve_cb) const = 0;

  virtual void operator()(Spinor *x, const Spinor *rhs, const double RsdTarget, int &niters, double &rsd_sq_final,
                          unsigned long &site_flops, unsigned long &mv_apps, int isign, bool verboseP,
                          int solve_cb = 1, ResiduumType residType = RELATIVE) const
  {
    Spinor *xa[1] = {x};
    const Spinor *ra[1] = {rhs};
    (*this)(xa, ra, RsdTarget, niters, rsd_sq_final, site_flops, mv_apps, isign, verboseP, solve_cb, residType);
  }

  virtual void operator()(Spinor *const x[num_flav], const Spinor *const rhs[num_flav], const double RsdTarget,
                          int &niters, double &rsd_sq_final, unsigned long &site_flops, unsigned long &mv_apps,
                          int isign, bool verboseP, int solve_cb = 1, ResiduumType residType = RELATIVE) const
  {
    CBSpinor *in_cb[num_flav], *in_other_cb[num_flav], *out_cb[num_flav], *out_other_cb[num_flav];
    for (int f = 0; f < num_flav; ++f) {
      in_cb[f] = rhs[f]->getCBData(solve_cb);
      in_other_cb[f] = rhs[f]->getCBData(1 - solve_cb);
      out_cb[f] = x[f]->getCBData(solve_cb);
      out_other_cb[f] = x[f]->getCBData(1 - solve_cb);
    }
    // the prepared source is kept in the solution's other checkerboard
    SourcePrepare(out_other_cb, in_cb, in_other_cb, isign, solve_cb);
    getEOSolver()(out_cb, out_other_cb, RsdTarget, niters, rsd_sq_final, site_flops, mv_apps, isign, verboseP,
                  solve_cb, residType);
    SolutionReconstruct(out_other_cb, in_other_cb, out_cb, isign, solve_cb);
  }
};

namespace gpu
{
// relative target for a possibly absolute request
// the library's targets are relative; an absolute target is divided by the
// norm of the whole right-hand side (both flavours of a two-flavour field)
inline double relative_target(qphix_gpu_field rhs, double rsd, ResiduumType t)
{
  if (t == RELATIVE) return rsd;
  double n2[32] = {0};
  check(qphix_gpu_blas_norm2(rhs, n2), "norm2");
  double s = 0;
  for (int i = 0; i < 32; i++) s += n2[i];
  return s > 0 ? rsd / std::sqrt(s) : rsd;
}
}  // namespace gpu

}  // namespace QPhiX
