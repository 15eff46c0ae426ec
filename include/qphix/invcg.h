// Drop-in Krylov solvers InvCG (reference: include/qphix/invcg.h:31-456),
// InvBiCGStab (invbicgstab.h:24-263) and InvMR / InvMRSmoother (invmr.h:
// 24-354): same constructors and operator(); the iteration runs on the
// device with the reference's recurrences and reports the same outputs.
#pragma once

#include "qphix/abs_solver.h"

namespace QPhiX
{

namespace gpu
{
// solver kind of InvMRSmoother (a fixed number of MR iterations), beside the
// QPHIX_GPU_SOLVER_* kinds of the C ABI
constexpr int MR_SMOOTHER = 100;

// Op::num_flav = 2 (two-flavour operators): x and rhs are (up, down) pairs,
// solved as one system on a device field of two right-hand sides
template <typename FT, int V, int S, bool C, typename Op>
class DeviceSolver : public AbstractSolver<FT, V, S, C, Op::num_flav>
{
 public:
  static constexpr int NF = Op::num_flav;
  typedef typename Geometry<FT, V, S, C>::FourSpinorBlock Spinor;
  DeviceSolver(Op &M_, int MaxIters_, int kind_, double omega_ = 1.0)
      : M(M_), MaxIters(MaxIters_), kind(kind_), omega(omega_)
  {
  }
  using AbstractSolver<FT, V, S, C, NF>::operator();

  void operator()(Spinor *const x[NF], const Spinor *const rhs[NF], const double RsdTarget, int &n_iters,
                  double &rsd_sq_final, unsigned long &site_flops, unsigned long &mv_apps, int isign, bool verbose,
                  int cb = 1, ResiduumType residType = RELATIVE) const override
  {
    (void)verbose;
    auto &g = M.getGeometry();
    auto dx = NF == 1 ? g.upload_spinor(x[0]) : g.upload_flavours(x);
    auto db = NF == 1 ? g.upload_spinor(rhs[0]) : g.upload_flavours(rhs);
    double rsd = relative_target(db.get(), RsdTarget, residType);
    qphix_gpu_solve_info infos[NF];  // one per right-hand side (the flavours of a pair agree)
    const qphix_gpu_solve_info &info = infos[0];
    int rc;
    if (kind == QPHIX_GPU_SOLVER_CG)
      rc = qphix_gpu_solve_cg(M.gpu_op(), dx.get(), db.get(), rsd, MaxIters, isign, cb, infos);
    else if (kind == QPHIX_GPU_SOLVER_BICGSTAB)
      rc = qphix_gpu_solve_bicgstab(M.gpu_op(), dx.get(), db.get(), rsd, MaxIters, isign, cb, infos);
    else if (kind == MR_SMOOTHER)  // RsdTarget is not a stopping test here (invmr.h:330-335)
      rc = qphix_gpu_solve_mr_smoother(M.gpu_op(), dx.get(), db.get(), MaxIters, omega, isign, cb, infos);
    else
      rc = qphix_gpu_solve_mr(M.gpu_op(), dx.get(), db.get(), rsd, MaxIters, omega, isign, cb, infos);
    check(rc, "solver");
    if (NF == 1)
      g.download_spinor(dx, x[0]);
    else
      g.download_flavours(dx, x);
    n_iters = info.n_iters;
    rsd_sq_final = info.rsd_sq_final;
    site_flops = info.site_flops;
    mv_apps = info.mv_apps;
  }

  Geometry<FT, V, S, C> &getGeometry() override { return M.getGeometry(); }
  // the smoother is not offered as the inner solver of InvRichardsonMultiPrec
  int gpu_solver_kind() const override { return kind == MR_SMOOTHER ? -1 : kind; }
  qphix_gpu_eo_op gpu_solver_op() const override { return M.gpu_op(); }
  int gpu_max_iters() const override { return MaxIters; }

 protected:
  Op &M;
  int MaxIters;
  int kind;
  double omega;
};
}  // namespace gpu

template <typename FT, int veclen, int soalen, bool compress12,
          typename EvenOddLinearOperatorBase = EvenOddLinearOperator<FT, veclen, soalen, compress12>>
class InvCG : public gpu::DeviceSolver<FT, veclen, soalen, compress12, EvenOddLinearOperatorBase>
{
 public:
  InvCG(EvenOddLinearOperatorBase &M_, int MaxIters_)
      : gpu::DeviceSolver<FT, veclen, soalen, compress12, EvenOddLinearOperatorBase>(M_, MaxIters_,
                                                                                      QPHIX_GPU_SOLVER_CG)
  {
  }
  void tune() {}
};

template <typename FT, int V, int S, bool compress12,
          typename EvenOddLinearOperatorBase = EvenOddLinearOperator<FT, V, S, compress12>>
class InvBiCGStab : public gpu::DeviceSolver<FT, V, S, compress12, EvenOddLinearOperatorBase>
{
 public:
  InvBiCGStab(EvenOddLinearOperatorBase &M_, int MaxIters_)
      : gpu::DeviceSolver<FT, V, S, compress12, EvenOddLinearOperatorBase>(M_, MaxIters_,
                                                                            QPHIX_GPU_SOLVER_BICGSTAB)
  {
  }
  void tune() {}
};

template <typename FT, int V, int S, bool compress12,
          typename EvenOddLinearOperatorBase = EvenOddLinearOperator<FT, V, S, compress12>>
class InvMR : public gpu::DeviceSolver<FT, V, S, compress12, EvenOddLinearOperatorBase>
{
 public:
  InvMR(EvenOddLinearOperatorBase &M_, int MaxIters_, double Omega)
      : gpu::DeviceSolver<FT, V, S, compress12, EvenOddLinearOperatorBase>(M_, MaxIters_, QPHIX_GPU_SOLVER_MR,
                                                                            Omega)
  {
  }
};

// InvMRSmoother (reference invmr.h:294-354): exactly MaxIters MR iterations
// with over-relaxation Omega and no residual test; n_iters = MaxIters and
// rsd_sq_final = -1, as the reference's InvMRBase reports with
// terminateOnResiduum = false.
template <typename FT, int V, int S, bool compress12,
          typename EvenOddLinearOperatorBase = EvenOddLinearOperator<FT, V, S, compress12>>
class InvMRSmoother : public gpu::DeviceSolver<FT, V, S, compress12, EvenOddLinearOperatorBase>
{
 public:
  InvMRSmoother(EvenOddLinearOperatorBase &M_, int MaxIters_, double Omega)
      : gpu::DeviceSolver<FT, V, S, compress12, EvenOddLinearOperatorBase>(M_, MaxIters_, gpu::MR_SMOOTHER, Omega)
  {
  }
};

}  // namespace QPhiX
