// Drop-in MInvCG (reference: include/qphix/minvcg.h:23-452): multishift CG
// for (M^dag M + shifts[i]) x_i = rhs, same constructor and operator().
#pragma once

#include <vector>

#include "qphix/abs_solver.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12,
          typename EvenOddLinearOperatorBase = EvenOddLinearOperator<FT, veclen, soalen, compress12>>
class MInvCG : public AbstractMultiSolver<FT, veclen, soalen, compress12, 1>
{
 public:
  typedef typename Geometry<FT, veclen, soalen, compress12>::FourSpinorBlock Spinor;
  MInvCG(EvenOddLinearOperatorBase &M_, int MaxIters_, int MaxShifts_)
      : M(M_), MaxIters(MaxIters_), MaxShifts(MaxShifts_)
  {
  }

  void operator()(Spinor **x, const Spinor *rhs, const int n_shift, const double *shifts, const double *RsdTarget,
                  int &n_iters, double *rsd_sq_final, unsigned long &site_flops, unsigned long &mv_apps, int isign,
                  bool verboseP, int cb = 1) const override
  {
    (void)verboseP;
    if (n_shift > MaxShifts) throw std::invalid_argument("MInvCG: too many shifts requested");
    auto &g = M.getGeometry();
    auto db = g.upload_spinor(rhs);
    std::vector<gpu::Field> xs;
    std::vector<qphix_gpu_field> xh;
    for (int s = 0; s < n_shift; s++) {
      xs.emplace_back(g.lattice(), QPHIX_GPU_SPINOR, g.device_prec(), 0, 1);
      xh.push_back(xs.back().get());
    }
    gpu::check(qphix_gpu_solve_mshift_cg(M.gpu_op(), xh.data(), db.get(), n_shift, shifts, RsdTarget, MaxIters, isign,
                                         cb, &n_iters, rsd_sq_final, &mv_apps),
               "MInvCG");
    site_flops = 0;
    for (int s = 0; s < n_shift; s++) g.download_spinor(xs[s], x[s]);
  }

  Geometry<FT, veclen, soalen, compress12> &getGeometry() override { return M.getGeometry(); }

 private:
  EvenOddLinearOperatorBase &M;
  int MaxIters;
  int MaxShifts;
};

}  // namespace QPhiX
