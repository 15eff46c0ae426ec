// Drop-in EvenOddWilsonOperator (reference: include/qphix/wilson.h:11-101):
// M_oo = (4 + m) - 0.25/(4 + m) D_oe D_eo.  The gauge arrays are copied to
// the device when the operator is constructed.
#pragma once

#include "qphix/linearOp.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12>
class EvenOddWilsonOperator : public gpu::EoOperatorBase<FT, veclen, soalen, compress12>
{
 public:
  typedef gpu::EoOperatorBase<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;

  EvenOddWilsonOperator(const double Mass_, SU3MatrixBlock *u_[2], Geom *geom_, double t_boundary_,
                        double aniso_fac_s_, double aniso_fac_t_, bool use_tbc_[4] = nullptr,
                        double tbc_phases_[4][2] = nullptr)
      : Base(geom_), Mass(Mass_)
  {
    this->p = gpu::make_params(QPHIX_GPU_WILSON, t_boundary_, aniso_fac_s_, aniso_fac_t_, use_tbc_, tbc_phases_,
                               Mass_);
    this->u = geom_->upload_gauge(u_[0], u_[1]);
    this->op.create(this->p, this->u.get(), nullptr, nullptr, nullptr, nullptr);
  }

  // -0.5 D (wilson.h:68-76)
  void M_offdiag(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int target_cb) const override
  {
    Geom &g = *this->geom;
    auto x = g.upload_spinor(in);
    gpu::Field out(g.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash(&this->p, out.get(), x.get(), this->u.get(), nullptr, nullptr, isign, target_cb),
               "M_offdiag");
    double a[2] = {-0.5, 0.0}, b[2] = {0.0, 0.0};
    gpu::check(qphix_gpu_blas_caxpby(a, out.get(), b, out.get()), "M_offdiag scale");
    g.download_spinor(out, res);
  }

  // (1 / (4 + m)) in (wilson.h:79-86)
  void M_diag_inv(FourSpinorBlock *res, FourSpinorBlock const *in, int isign, int cb = 0) const override
  {
    (void)isign;
    (void)cb;
    Geom &g = *this->geom;
    auto x = g.upload_spinor(in);
    double a[2] = {1.0 / (4.0 + Mass), 0.0}, b[2] = {0.0, 0.0};
    gpu::check(qphix_gpu_blas_caxpby(a, x.get(), b, x.get()), "M_diag_inv");
    g.download_spinor(x, res);
  }

 private:
  double Mass;
};

}  // namespace QPhiX
