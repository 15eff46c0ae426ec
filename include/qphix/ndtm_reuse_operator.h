// Drop-in EvenOddNDTMWilsonReuseOperator (reference: include/qphix/
// ndtm_reuse_operator.h:16-150): the two-flavour twisted-mass Wilson operator
//   M_oo^f = (alpha + i mu g5 tau3) chi^f - eps (tau1 chi)^f
//            - 1/4 D_oe mu_inv [(alpha - i mu g5 tau3) + eps tau1] D_eo chi,
// mu_inv = 1 / (alpha^2 + mu^2 - eps^2), on (up, down) spinor pairs.  It runs
// as one device operator whose fields hold the two flavours as right-hand
// sides 0 and 1; InvCG solves the pair as one system.
#pragma once

#include "qphix/linearOp.h"

namespace QPhiX
{

template <typename FT, int veclen, int soalen, bool compress12>
class EvenOddNDTMWilsonReuseOperator : public TwoFlavEvenOddLinearOperator<FT, veclen, soalen, compress12>
{
 public:
  typedef Geometry<FT, veclen, soalen, compress12> Geom;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;

  EvenOddNDTMWilsonReuseOperator(const double mass, const double mu, const double epsilon, SU3MatrixBlock *u[2],
                                 Geom *geom_, double t_boundary, double aniso_coeff_s, double aniso_coeff_t,
                                 bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr)
      : geom(geom_)
  {
    p = gpu::make_params(QPHIX_GPU_NDTM, t_boundary, aniso_coeff_s, aniso_coeff_t, use_tbc_, tbc_phases_, mass, mu);
    p.epsilon = epsilon;
    uf = geom_->upload_gauge(u[0], u[1]);
    op.create(p, uf.get(), nullptr, nullptr, nullptr, nullptr);
  }

  void operator()(FourSpinorBlock *const res[2], FourSpinorBlock const *const in[2], int isign,
                  int target_cb = 1) override
  {
    auto x = geom->upload_flavours(in);
    gpu::Field out(geom->lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0, 2);
    gpu::check(qphix_gpu_eo_op_apply(op.get(), out.get(), x.get(), isign, target_cb), "two-flavour operator");
    geom->download_flavours(out, res);
  }

  Geom &getGeometry() override { return *geom; }
  qphix_gpu_eo_op gpu_op() const override { return op.get(); }

 private:
  Geom *geom;
  gpu::Field uf;
  gpu::EoOp op;
  qphix_gpu_op_params p;
};

}  // namespace QPhiX
