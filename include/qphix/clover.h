// Drop-in EvenOddCloverOperator (reference: include/qphix/clover.h:15-268):
// M_oo = A_oo + i rho g5 - 0.25 D_oe A_ee^-1 D_eo, all constructors and
// setFields.  Fields are copied to the device at construction / setFields.
#pragma once

#include "qphix/linearOp.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12>
class EvenOddCloverOperator : public gpu::EoOperatorBase<FT, veclen, soalen, compress12>
{
 public:
  typedef gpu::EoOperatorBase<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::CloverBlock CloverBlock;

  EvenOddCloverOperator(SU3MatrixBlock *u_[2], CloverBlock *clov_, CloverBlock *invclov_even, Geom *geom_,
                        double t_boundary, double aniso_coeff_s, double aniso_coeff_t, bool use_tbc_[4] = nullptr,
                        double tbc_phases_[4][2] = nullptr, double const prec_mass_rho = 0.0,
                        CloverBlock *invclov_odd = nullptr)
      : Base(geom_)
  {
    init(t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_, prec_mass_rho);
    setFields(u_, clov_, invclov_even);
    if (invclov_odd) this->invclov_odd = geom_->upload_clover(invclov_odd);
  }

  EvenOddCloverOperator(SU3MatrixBlock *u_[2], CloverBlock *clov_[2], CloverBlock *invclov_even, Geom *geom_,
                        double t_boundary, double aniso_coeff_s, double aniso_coeff_t, bool use_tbc_[4] = nullptr,
                        double tbc_phases_[4][2] = nullptr, double const prec_mass_rho = 0.0,
                        CloverBlock *invclov_odd = nullptr)
      : Base(geom_)
  {
    init(t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_, prec_mass_rho);
    setFields(u_, clov_[1], invclov_even);
    if (invclov_odd) this->invclov_odd = geom_->upload_clover(invclov_odd);
  }

  EvenOddCloverOperator(Geom *geom_, double t_boundary, double aniso_coeff_s, double aniso_coeff_t,
                        bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr,
                        double const prec_mass_rho = 0.0)
      : Base(geom_)
  {
    init(t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_, prec_mass_rho);
  }

  void setFields(SU3MatrixBlock *u_[2], CloverBlock *clov_, CloverBlock *invclov_)
  {
    Geom &g = *this->geom;
    this->u = g.upload_gauge(u_[0], u_[1]);
    this->clov = g.upload_clover(clov_);
    this->invclov = g.upload_clover(invclov_);
    this->op.create(this->p, this->u.get(), this->clov.get(), this->invclov.get(), nullptr, nullptr);
  }
  void setFields(SU3MatrixBlock *u_[2], CloverBlock *clov_[2], CloverBlock *invclov_) { setFields(u_, clov_[1], invclov_); }

  // -0.5 D (clover.h:175-184)
  void M_offdiag(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int target_cb) const override
  {
    Geom &g = *this->geom;
    auto x = g.upload_spinor(in);
    gpu::Field out(g.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    qphix_gpu_op_params w = this->p;
    w.kind = QPHIX_GPU_WILSON;
    gpu::check(qphix_gpu_dslash(&w, out.get(), x.get(), this->u.get(), nullptr, nullptr, isign, target_cb),
               "M_offdiag");
    double a[2] = {-0.5, 0.0}, b[2] = {0.0, 0.0};
    gpu::check(qphix_gpu_blas_caxpby(a, out.get(), b, out.get()), "M_offdiag scale");
    g.download_spinor(out, res);
  }

  // A^-1 of checkerboard cb (clover.h:186-192)
  void M_diag_inv(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int cb = 0) const override
  {
    (void)isign;
    const gpu::Field &ai = (cb == 0) ? this->invclov : this->invclov_odd;
    if (!ai) throw std::invalid_argument("M_diag_inv: no inverse clover term for this checkerboard");
    Geom &g = *this->geom;
    auto x = g.upload_spinor(in);
    gpu::Field out(g.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_clover_apply(out.get(), x.get(), ai.get()), "M_diag_inv");
    g.download_spinor(out, res);
  }

 private:
  void init(double tb, double as, double at, bool *use_tbc, double (*tbc)[2], double rho)
  {
    this->p = gpu::make_params(QPHIX_GPU_CLOVER_OP, tb, as, at, use_tbc, tbc, 0.0, 0.0, rho);
  }
};

}  // namespace QPhiX
