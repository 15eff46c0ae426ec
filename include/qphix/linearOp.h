// Drop-in EvenOddLinearOperator (reference: include/qphix/linearOp.h:9-92):
// operator()(res, in, isign, target_cb = 1), M_offdiag, M_diag_inv,
// getGeometry.  The GPU operators below also expose the device operator they
// run (gpu_op), which the drop-in solvers use.
#pragma once

#include "qphix/dslash_def.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress>
class EvenOddLinearOperator
{
 public:
  virtual ~EvenOddLinearOperator() {}
  typedef typename Geometry<FT, veclen, soalen, compress>::FourSpinorBlock FourSpinorBlock;
  static constexpr int num_flav = 1;

  virtual void operator()(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int target_cb = 1) const = 0;
  virtual void M_offdiag(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int target_cb) const = 0;
  virtual void M_diag_inv(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int cb = 0) const = 0;
  virtual void operator()(FourSpinorBlock *const res[1], FourSpinorBlock const *const in[1], int isign,
                          int target_cb = 1) const
  {
    (*this)(res[0], in[0], isign, target_cb);
  }
  virtual Geometry<FT, veclen, soalen, compress> &getGeometry() = 0;

  // the device operator (not part of QPhiX's interface)
  virtual qphix_gpu_eo_op gpu_op() const = 0;
};

// reference: include/qphix/linearOp.h (TwoFlavEvenOddLinearOperator): the
// operator on two-flavour spinors res[2], in[2] (up, down)
template <typename FT, int veclen, int soalen, bool compress>
class TwoFlavEvenOddLinearOperator
{
 public:
  virtual ~TwoFlavEvenOddLinearOperator() {}
  typedef typename Geometry<FT, veclen, soalen, compress>::FourSpinorBlock FourSpinorBlock;
  static constexpr int num_flav = 2;

  virtual void operator()(FourSpinorBlock *const res[2], FourSpinorBlock const *const in[2], int isign,
                          int target_cb = 1) = 0;
  virtual Geometry<FT, veclen, soalen, compress> &getGeometry() = 0;

  // the device operator (not part of QPhiX's interface)
  virtual qphix_gpu_eo_op gpu_op() const = 0;
};

namespace gpu
{
// shared body of the four even-odd operators
template <typename FT, int V, int S, bool C>
class EoOperatorBase : public EvenOddLinearOperator<FT, V, S, C>
{
 public:
  typedef Geometry<FT, V, S, C> Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;

  explicit EoOperatorBase(Geom *g) : geom(g) {}

  void operator()(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int target_cb = 1) const override
  {
    auto x = geom->upload_spinor(in);
    Field out(geom->lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    check(qphix_gpu_eo_op_apply(op.get(), out.get(), x.get(), isign, target_cb), "even-odd operator");
    geom->download_spinor(out, res);
  }
  using EvenOddLinearOperator<FT, V, S, C>::operator();

  Geom &getGeometry() override { return *geom; }
  qphix_gpu_eo_op gpu_op() const override { return op.get(); }

 protected:
  Geom *geom;
  Field u, clov, invclov, invclov_odd, f0, f1;
  EoOp op;
  qphix_gpu_op_params p;
};
}  // namespace gpu

}  // namespace QPhiX
