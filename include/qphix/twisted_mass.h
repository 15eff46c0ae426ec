// Drop-in EvenOddTMWilsonOperator (reference: include/qphix/twisted_mass.h:
// 12-111): M_oo = (alpha + i mu g5) - 0.25 D [(alpha + i mu g5)^-1] D.
#pragma once

#include "qphix/linearOp.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12>
class EvenOddTMWilsonOperator : public gpu::EoOperatorBase<FT, veclen, soalen, compress12>
{
 public:
  typedef gpu::EoOperatorBase<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;

  EvenOddTMWilsonOperator(const double Mass_, const double TwistedMass_, SU3MatrixBlock *u_[2], Geom *geom_,
                          double t_boundary_, double aniso_fac_s_, double aniso_fac_t_, bool use_tbc_[4] = nullptr,
                          double tbc_phases_[4][2] = nullptr)
      : Base(geom_)
  {
    this->p = gpu::make_params(QPHIX_GPU_TM, t_boundary_, aniso_fac_s_, aniso_fac_t_, use_tbc_, tbc_phases_, Mass_,
                               TwistedMass_);
    this->u = geom_->upload_gauge(u_[0], u_[1]);
    this->op.create(this->p, this->u.get(), nullptr, nullptr, nullptr, nullptr);
  }

  // not provided by the reference either (twisted_mass.h:79-95 abort)
  void M_offdiag(FourSpinorBlock *, FourSpinorBlock const *, int, int) const override
  {
    throw std::logic_error("M_offdiag not implemented for EvenOddTMWilsonOperator");
  }
  void M_diag_inv(FourSpinorBlock *, FourSpinorBlock const *, int, int = 0) const override
  {
    throw std::logic_error("M_diag_inv not implemented for EvenOddTMWilsonOperator");
  }
};

}  // namespace QPhiX
