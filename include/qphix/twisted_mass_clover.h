// Drop-in EvenOddTMCloverOperator (reference: include/qphix/
// twisted_mass_clover.h:13-137): M_oo = (A + i rho g5) - 0.25 D
// [(A_ee +/- i mu g5)^-1] D with the two full inverses supplied by the caller.
#pragma once

#include "qphix/linearOp.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12>
class EvenOddTMCloverOperator : public gpu::EoOperatorBase<FT, veclen, soalen, compress12>
{
 public:
  typedef gpu::EoOperatorBase<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::CloverBlock CloverBlock;
  typedef typename Geom::FullCloverBlock FullCloverBlock;

  EvenOddTMCloverOperator(SU3MatrixBlock *const u_[2], CloverBlock *clov_, FullCloverBlock *const invclov_[2],
                          Geom *geom_, double t_boundary, double aniso_coeff_s, double aniso_coeff_t,
                          bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr,
                          double const prec_mass_rho = 0.0)
      : Base(geom_)
  {
    this->p = gpu::make_params(QPHIX_GPU_TMCLOVER, t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_,
                               0.0, 0.0, prec_mass_rho);
    setFields(const_cast<SU3MatrixBlock **>(u_), clov_, const_cast<FullCloverBlock **>(invclov_));
  }

  EvenOddTMCloverOperator(Geom *const geom_, double const t_boundary, double const aniso_coeff_s,
                          double const aniso_coeff_t, bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr,
                          double const prec_mass_rho = 0.0)
      : Base(geom_)
  {
    this->p = gpu::make_params(QPHIX_GPU_TMCLOVER, t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_,
                               0.0, 0.0, prec_mass_rho);
  }

  void setFields(SU3MatrixBlock *u_[2], CloverBlock *clov_, FullCloverBlock *invclov_[2])
  {
    Geom &g = *this->geom;
    this->u = g.upload_gauge(u_[0], u_[1]);
    this->clov = g.upload_clover(clov_);
    this->f0 = g.upload_full_clover(invclov_[0]);
    this->f1 = g.upload_full_clover(invclov_[1]);
    this->op.create(this->p, this->u.get(), this->clov.get(), nullptr, this->f0.get(), this->f1.get());
  }

  void M_offdiag(FourSpinorBlock *, FourSpinorBlock const *, int, int) const override
  {
    throw std::logic_error("M_offdiag not implemented for EvenOddTMCloverOperator");
  }
  void M_diag_inv(FourSpinorBlock *, FourSpinorBlock const *, int, int = 0) const override
  {
    throw std::logic_error("M_diag_inv not implemented for EvenOddTMCloverOperator");
  }
};

}  // namespace QPhiX
