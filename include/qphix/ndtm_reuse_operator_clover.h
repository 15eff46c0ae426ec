// Drop-in EvenOddNDTMCloverReuseOperator (reference: include/qphix/
// ndtm_reuse_operator_clover.h:23-165): the two-flavour twisted-mass clover
// operator on (up, down) spinor pairs,
//   M_oo^f = A chi^f + i s_f mu g5 chi^f - eps chi^{1-f}
//            - 1/4 D_oe [B_ee^-1 (D_eo chi)]^f,   s_up = +1, s_dn = -1,
// with B_ee^-1 given by the caller as the flavour-diagonal full inverses
// invclov[2] and the flavour-off-diagonal packed inverse invclov_odiag
// (qphix_gpu_clover_invert_ndtm builds them on the device).  It runs as one
// device operator whose fields hold the two flavours as right-hand sides 0
// and 1; InvCG solves the pair as one system.  As in the reference,
// M_offdiag / M_diag_inv are not provided.
#pragma once

#include <stdexcept>

#include "qphix/linearOp.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12>
class EvenOddNDTMCloverReuseOperator : public TwoFlavEvenOddLinearOperator<FT, veclen, soalen, compress12>
{
 public:
  typedef Geometry<FT, veclen, soalen, compress12> Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::CloverBlock CloverBlock;
  typedef typename Geom::FullCloverBlock FullCloverBlock;

  EvenOddNDTMCloverReuseOperator(double TwistedMass_, double Epsilon_, SU3MatrixBlock *u_[2], CloverBlock *clov_,
                                 CloverBlock *invclov_odiag_, FullCloverBlock *invclov_[2], Geom *geom_,
                                 double t_boundary, double aniso_coeff_s, double aniso_coeff_t,
                                 bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr)
      : EvenOddNDTMCloverReuseOperator(TwistedMass_, Epsilon_, geom_, t_boundary, aniso_coeff_s, aniso_coeff_t,
                                       use_tbc_, tbc_phases_)
  {
    setFields(u_, clov_, invclov_odiag_, invclov_);
  }

  EvenOddNDTMCloverReuseOperator(double TwistedMass_, double Epsilon_, Geom *geom_, double t_boundary,
                                 double aniso_coeff_s, double aniso_coeff_t, bool use_tbc_[4] = nullptr,
                                 double tbc_phases_[4][2] = nullptr)
      : geom(geom_)
  {
    p = gpu::make_params(QPHIX_GPU_NDTMCLOVER, t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_, 0.0,
                         TwistedMass_);
    p.epsilon = Epsilon_;
  }

  void setFields(SU3MatrixBlock *u_[2], CloverBlock *clov_, CloverBlock *invclov_odiag_,
                 FullCloverBlock *invclov_[2])
  {
    uf = geom->upload_gauge(u_[0], u_[1]);
    clov = geom->upload_clover(clov_);
    odiag = geom->upload_clover(invclov_odiag_);
    f0 = geom->upload_full_clover(invclov_[0]);
    f1 = geom->upload_full_clover(invclov_[1]);
    op.create(p, uf.get(), clov.get(), odiag.get(), f0.get(), f1.get());
  }

  void operator()(FourSpinorBlock *const res[2], FourSpinorBlock const *const in[2], int isign,
                  int target_cb = 1) override
  {
    if (!op.get()) throw std::logic_error("EvenOddNDTMCloverReuseOperator: setFields was not called");
    auto x = geom->upload_flavours(in);
    gpu::Field out(geom->lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0, 2);
    gpu::check(qphix_gpu_eo_op_apply(op.get(), out.get(), x.get(), isign, target_cb),
               "two-flavour clover operator");
    geom->download_flavours(out, res);
  }

  Geom &getGeometry() override { return *geom; }
  qphix_gpu_eo_op gpu_op() const override { return op.get(); }

 private:
  Geom *geom;
  gpu::Field uf, clov, odiag, f0, f1;
  gpu::EoOp op;
  qphix_gpu_op_params p;
};

}  // namespace QPhiX
