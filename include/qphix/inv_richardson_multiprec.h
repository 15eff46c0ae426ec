// Drop-in InvRichardsonMultiPrec (reference: include/qphix/
// inv_richardson_multiprec.h:22-320): defect correction with the outer
// operator in FT and the inner solver (CG / BiCGStab / MR on its own
// operator, typically in float or half) in FTInner.  Runs on the device;
// MdagM = true (outer residual of M^dag M) is not supported.
#pragma once

#include "qphix/abs_solver.h"

namespace QPhiX
{

template <typename FT, int V, int S, bool Compress, typename FTInner, int VInner, int SInner, bool CompressInner,
          bool MdagM = false, typename EvenOddLinearOperatorBase = EvenOddLinearOperator<FT, V, S, Compress>>
class InvRichardsonMultiPrec : public AbstractSolver<FT, V, S, Compress, 1>
{
 public:
  typedef typename Geometry<FT, V, S, Compress>::FourSpinorBlock Spinor;
  using AbstractSolver<FT, V, S, Compress, 1>::operator();

  InvRichardsonMultiPrec(EvenOddLinearOperatorBase &m_outer_,
                         AbstractSolver<FTInner, VInner, SInner, CompressInner, 1> &solver_inner_, const double delta_,
                         const int max_iters_)
      : m_outer(m_outer_), solver_inner(solver_inner_), delta(delta_), max_iters(max_iters_)
  {
    static_assert(!MdagM, "InvRichardsonMultiPrec with MdagM = true is not supported on the device");
  }

  void operator()(Spinor *const x[1], const Spinor *const rhs[1], const double RsdTarget, int &n_iters,
                  double &rsd_sq_final, unsigned long &site_flops, unsigned long &mv_apps, int isign, bool verbose,
                  int cb = 1, ResiduumType residType = RELATIVE) const override
  {
    (void)verbose;
    auto &g = m_outer.getGeometry();
    auto dx = g.upload_spinor(x[0]);
    auto db = g.upload_spinor(rhs[0]);
    double rsd = gpu::relative_target(db.get(), RsdTarget, residType);
    qphix_gpu_solve_info info;
    gpu::check(qphix_gpu_solve_richardson(m_outer.gpu_op(), solver_inner.gpu_solver_op(),
                                          solver_inner.gpu_solver_kind(), dx.get(), db.get(), rsd, delta, max_iters,
                                          solver_inner.gpu_max_iters(), isign, cb, &info),
               "InvRichardsonMultiPrec");
    g.download_spinor(dx, x[0]);
    n_iters = info.n_iters;
    rsd_sq_final = info.rsd_sq_final;
    site_flops = info.site_flops;
    mv_apps = info.mv_apps;
  }

  Geometry<FT, V, S, Compress> &getGeometry() override { return m_outer.getGeometry(); }
  int gpu_solver_kind() const override { return -1; }
  qphix_gpu_eo_op gpu_solver_op() const override { return m_outer.gpu_op(); }
  int gpu_max_iters() const override { return max_iters; }
  void tune() {}

 private:
  EvenOddLinearOperatorBase &m_outer;
  AbstractSolver<FTInner, VInner, SInner, CompressInner, 1> &solver_inner;
  const double delta;
  const int max_iters;
};

}  // namespace QPhiX
