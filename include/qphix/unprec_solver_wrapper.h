// Drop-in UnprecSolverWrapper (reference: include/qphix/unprec_solver_wrapper.h):
// the unpreconditioned solve of an even-odd operator with M_offdiag and
// M_diag_inv (the clover and Wilson operators provide them):
//   source   b' = b_cb - M_offdiag(M_diag_inv(b_other), solve_cb)
//   solve    M_eo x_cb = b'
//   other cb x_other = M_diag_inv(b_other - M_offdiag(x_cb, 1 - solve_cb))
// M_diag_inv is called with its default checkerboard, as in the reference
// (unprec_solver_wrapper.h:54,84): the inverse diagonal block the operator
// was built with, which is the block of the checkerboard not solved for.
// The copies and differences run on the device.
#pragma once

#include "qphix/abs_solver.h"

namespace QPhiX
{

template <typename FT, int V, int S, bool compress12, typename LinearOpType, int num_flav = 1>
class UnprecSolverWrapper : public AbstractUnprecSolver<FT, V, S, compress12, num_flav>
{
 public:
  using Spinor = FullSpinor<FT, V, S, compress12>;
  using CBSpinor = typename Spinor::CBSpinor;
  typedef Geometry<FT, V, S, compress12> Geom;

  UnprecSolverWrapper(AbstractSolver<FT, V, S, compress12> &theEOSolver_, LinearOpType &M_)
      : theEOSolver(theEOSolver_), M(M_), geom(M_.getGeometry())
  {
    static_assert(num_flav == 1, "two-flavour unpreconditioned solves are not provided");
    tmp1 = geom.allocCBFourSpinor();
    tmp2 = geom.allocCBFourSpinor();
  }
  ~UnprecSolverWrapper()
  {
    geom.free(tmp1);
    geom.free(tmp2);
  }

  void SourcePrepare(CBSpinor *const out[num_flav], CBSpinor const *const in_cb[num_flav],
                     CBSpinor const *const in_other_cb[num_flav], int isign, int solve_cb) const override
  {
    M.M_diag_inv(tmp1, in_other_cb[0], isign);
    M.M_offdiag(tmp2, tmp1, isign, solve_cb);
    difference(out[0], in_cb[0], tmp2);
  }

  void SolutionReconstruct(CBSpinor *const out_other_cb[num_flav], CBSpinor const *const in_other_cb[num_flav],
                           CBSpinor const *const out_cb[num_flav], int isign, int solve_cb) const override
  {
    M.M_offdiag(tmp1, out_cb[0], isign, 1 - solve_cb);
    difference(tmp2, in_other_cb[0], tmp1);
    M.M_diag_inv(out_other_cb[0], tmp2, isign);
  }

  AbstractSolver<FT, V, S, compress12> &getEOSolver() const override { return theEOSolver; }

 private:
  // out = a - b (host arrays in Geometry's layout; computed on the device)
  void difference(CBSpinor *out, const CBSpinor *a, const CBSpinor *b) const
  {
    auto da = geom.upload_spinor(a);
    auto db = geom.upload_spinor(b);
    double one[2] = {1.0, 0.0}, mone[2] = {-1.0, 0.0};
    gpu::check(qphix_gpu_blas_caxpby(mone, db.get(), one, da.get()), "unprec difference");
    geom.download_spinor(da, out);
  }

  AbstractSolver<FT, V, S, compress12> &theEOSolver;
  LinearOpType &M;
  Geom &geom;
  CBSpinor *tmp1, *tmp2;
};

}  // namespace QPhiX
