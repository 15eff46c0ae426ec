// Drop-in Dslash family: Dslash (reference: include/qphix/dslash_def.h:27-58),
// ClovDslash (clover_dslash_def.h:24-53), TMDslash (tm_dslash_def.h:23-49)
// and TMClovDslash (tm_clov_dslash_def.h:30-66), same constructors and
// member functions.  Each call moves its spinor arrays (QPhiX layout) to the
// device, runs one sm_100a kernel and moves the result back; the gauge and
// clover arrays are uploaded on first use and kept on the device for later
// calls with the same arrays (invalidateFieldCache()).  `u` is the gauge
// array of the target checkerboard, as in QPhiX (its eight links per site
// carry both hop directions).
#pragma once

#include "qphix/geometry.h"

namespace QPhiX
{

namespace gpu
{
// device gauge field from one QPhiX checkerboard array (forward + back links)
template <typename G>
Field upload_gauge_cb(const G &geom, const typename G::SU3MatrixBlock *u, int cb)
{
  Field f(geom.lattice(), QPHIX_GPU_GAUGE, G::device_prec(), G::compress12 ? 12 : 18);
  auto l = geom.host_layout();
  check(qphix_gpu_field_upload(f.get(), u, &l, 2 + cb, -1), "gauge upload");
  return f;
}
}  // namespace gpu

template <typename FT, int veclen, int soalen, bool compress12>
class Dslash
{
 public:
  typedef Geometry<FT, veclen, soalen, compress12> Geom;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::TwoSpinorBlock TwoSpinorBlock;

  Dslash(Geom *geom_, double t_boundary_, double aniso_coeff_S_, double aniso_coeff_T_, bool use_tbc_[4] = nullptr,
         double tbc_phases_[4][2] = nullptr)
      : s(geom_), p(gpu::make_params(QPHIX_GPU_WILSON, t_boundary_, aniso_coeff_S_, aniso_coeff_T_, use_tbc_,
                                     tbc_phases_))
  {
  }

  void dslash(FourSpinorBlock *res, const FourSpinorBlock *psi, const SU3MatrixBlock *u, int isign, int cb)
  {
    qphix_gpu_field g = gauge_dev(u, cb);
    auto in = s->upload_spinor(psi);
    gpu::Field out(s->lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash(&p, out.get(), in.get(), g, nullptr, nullptr, isign, cb), "dslash");
    s->download_spinor(out, res);
  }

  void dslashAChiMinusBDPsi(FourSpinorBlock *res, const FourSpinorBlock *psi, const FourSpinorBlock *chi,
                            const SU3MatrixBlock *u, double alpha, double beta, int isign, int cb)
  {
    qphix_gpu_field g = gauge_dev(u, cb);
    auto in = s->upload_spinor(psi);
    auto x = s->upload_spinor(chi);
    gpu::Field out(s->lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash_achimbdpsi(&p, out.get(), in.get(), x.get(), g, nullptr, alpha, beta, isign,
                                           cb, 1.0),
               "dslashAChiMinusBDPsi");
    s->download_spinor(out, res);
  }

  void dslashDir(FourSpinorBlock *res, const FourSpinorBlock *psi, const SU3MatrixBlock *u, int cb, int dir)
  {
    qphix_gpu_field g = gauge_dev(u, cb);
    auto in = s->upload_spinor(psi);
    gpu::Field out(s->lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash_dir(&p, out.get(), in.get(), g, cb, dir), "dslashDir");
    s->download_spinor(out, res);
  }

  void free(void *) {}
  Geom &getGeometry() { return *s; }

  // Device copies of the gauge and clover arrays passed to this object are
  // kept between calls (keyed by the host array's address; an array released
  // through Geometry::free is never matched again).  A caller that rewrites
  // one of those arrays in place and calls again must call this first.  Not
  // part of QPhiX's interface (its kernels read the host arrays directly).
  void invalidateFieldCache() { cache_.clear(); }

 protected:
  typedef typename Geom::CloverBlock CloverBlock_;
  typedef typename Geom::FullCloverBlock FullCloverBlock_;
  qphix_gpu_field gauge_dev(const SU3MatrixBlock *u, int cb)
  {
    return cache_.get(u, cb, [&] { return gpu::upload_gauge_cb(*s, u, cb); });
  }
  qphix_gpu_field clover_dev(const CloverBlock_ *c)
  {
    return cache_.get(c, 2, [&] { return s->upload_clover(c); });
  }
  qphix_gpu_field full_clover_dev(const FullCloverBlock_ *c)
  {
    return cache_.get(c, 3, [&] { return s->upload_full_clover(c); });
  }

  Geom *s;
  qphix_gpu_op_params p;
  gpu::FieldCache cache_;
};

template <typename FT, int veclen, int soalen, bool compress12>
class ClovDslash : public Dslash<FT, veclen, soalen, compress12>
{
 public:
  typedef Dslash<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::CloverBlock CloverBlock;

  ClovDslash(Geom *geom_, double t_boundary_, double dslash_aniso_s_, double dslash_aniso_t_,
             bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr, double const prec_mass_rho = 0.0)
      : Base(geom_, t_boundary_, dslash_aniso_s_, dslash_aniso_t_, use_tbc_, tbc_phases_)
  {
    this->p.kind = QPHIX_GPU_CLOVER_OP;
    this->p.prec_mass_rho = prec_mass_rho;
  }

  // res = A^-1 D psi
  void dslash(FourSpinorBlock *res, const FourSpinorBlock *psi, const SU3MatrixBlock *u, const CloverBlock *invclov,
              int isign, int cb)
  {
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    qphix_gpu_field c = this->clover_dev(invclov);
    auto in = s.upload_spinor(psi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash(&this->p, out.get(), in.get(), g, c, nullptr, isign, cb), "clover dslash");
    s.download_spinor(out, res);
  }

  // res = A chi + i rho isign g5 chi - beta D psi
  void dslashAChiMinusBDPsi(FourSpinorBlock *res, const FourSpinorBlock *psi, const FourSpinorBlock *chi,
                            const SU3MatrixBlock *u, const CloverBlock *clov, const double beta, int isign, int cb)
  {
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    qphix_gpu_field c = this->clover_dev(clov);
    auto in = s.upload_spinor(psi);
    auto x = s.upload_spinor(chi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash_achimbdpsi(&this->p, out.get(), in.get(), x.get(), g, c, 0.0, beta, isign,
                                           cb, 1.0),
               "clover dslashAChiMinusBDPsi");
    s.download_spinor(out, res);
  }

  void clovMult(FourSpinorBlock *res, const FourSpinorBlock *chi, const CloverBlock *clov)
  {
    Geom &s = *this->s;
    qphix_gpu_field c = this->clover_dev(clov);
    auto x = s.upload_spinor(chi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_clover_apply(out.get(), x.get(), c), "clovMult");
    s.download_spinor(out, res);
  }
};

template <typename FT, int veclen, int soalen, bool compress12>
class TMDslash : public Dslash<FT, veclen, soalen, compress12>
{
 public:
  typedef Dslash<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;

  TMDslash(Geom *geom_, double t_boundary_, double aniso_coeff_S_, double aniso_coeff_T_, double Mass_,
           double TwistedMass_, bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr)
      : Base(geom_, t_boundary_, aniso_coeff_S_, aniso_coeff_T_, use_tbc_, tbc_phases_)
  {
    this->p.kind = QPHIX_GPU_TM;
    this->p.mass = Mass_;
    this->p.twisted_mass = TwistedMass_;
  }

  // res = (alpha - i mu isign g5)/(alpha^2 + mu^2) D psi
  void dslash(FourSpinorBlock *res, const FourSpinorBlock *psi, const SU3MatrixBlock *u, int isign, int cb)
  {
    Base::dslash(res, psi, u, isign, cb);
  }

  // res = alpha (1 + i isign musign mu/(4+m) g5) chi - beta D psi
  void dslashAChiMinusBDPsi(FourSpinorBlock *res, const FourSpinorBlock *psi, const FourSpinorBlock *chi,
                            const SU3MatrixBlock *u, double alpha, double beta, int isign, int cb,
                            const double musign = 1.0)
  {
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    auto in = s.upload_spinor(psi);
    auto x = s.upload_spinor(chi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash_achimbdpsi(&this->p, out.get(), in.get(), x.get(), g, nullptr, alpha, beta,
                                           isign, cb, musign),
               "tm dslashAChiMinusBDPsi");
    s.download_spinor(out, res);
  }

  // res_f = alpha (1 + i s_f isign mu/(4+m) g5) chi_f - beta D psi_f - epsilon chi_{1-f},
  // s_up = +1, s_dn = -1 (tm_dslash_body.h:1174-1207)
  void two_flav_AChiMinusBDPsi(FourSpinorBlock *const res[2], const FourSpinorBlock *const psi[2],
                               const FourSpinorBlock *const chi[2], const SU3MatrixBlock *u, double alpha,
                               double beta, double epsilon, int isign, int cb)
  {
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    auto in = s.upload_flavours(psi);
    auto x = s.upload_flavours(chi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0, 2);
    qphix_gpu_op_params q = this->p;
    q.kind = QPHIX_GPU_NDTM;
    q.epsilon = epsilon;
    gpu::check(qphix_gpu_dslash_achimbdpsi(&q, out.get(), in.get(), x.get(), g, nullptr, alpha, beta, isign,
                                           cb, 1.0),
               "tm two_flav_AChiMinusBDPsi");
    s.download_flavours(out, res);
  }
};

template <typename FT, int veclen, int soalen, bool compress12>
class TMClovDslash : public Dslash<FT, veclen, soalen, compress12>
{
 public:
  typedef Dslash<FT, veclen, soalen, compress12> Base;
  typedef typename Base::Geom Geom;
  typedef typename Geom::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Geom::FourSpinorBlock FourSpinorBlock;
  typedef typename Geom::CloverBlock CloverBlock;
  typedef typename Geom::FullCloverBlock FullCloverBlock;

  TMClovDslash(Geom *geom_, double t_boundary_, double dslash_aniso_s_, double dslash_aniso_t_,
               bool use_tbc_[4] = nullptr, double tbc_phases_[4][2] = nullptr, double const prec_mass_rho = 0.0)
      : Base(geom_, t_boundary_, dslash_aniso_s_, dslash_aniso_t_, use_tbc_, tbc_phases_)
  {
    this->p.kind = QPHIX_GPU_TMCLOVER;
    this->p.prec_mass_rho = prec_mass_rho;
  }

  // res = invclov[k] D psi, k = 0 for (isign = +1, up) and (isign = -1, down),
  // else 1 (tm_clov_dslash_body.h:348-353)
  void dslash(FourSpinorBlock *res, const FourSpinorBlock *psi, const SU3MatrixBlock *u,
              const FullCloverBlock *const invclov[2], int isign, int cb, int fl = 0)
  {
    if (fl != 0 && fl != 1) throw std::invalid_argument("TMClovDslash: flavour must be 0 (up) or 1 (down)");
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    qphix_gpu_field f0 = this->full_clover_dev(invclov[fl]);
    qphix_gpu_field f1 = this->full_clover_dev(invclov[1 - fl]);
    auto in = s.upload_spinor(psi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    gpu::check(qphix_gpu_dslash(&this->p, out.get(), in.get(), g, f0, f1, isign, cb),
               "tm clover dslash");
    s.download_spinor(out, res);
  }

  // res = (A + i rho_f g5) chi - beta D psi, rho_up = prec_mass_rho, rho_dn = -prec_mass_rho
  // (tm_clov_dslash_body.h:983)
  void dslashAChiMinusBDPsi(FourSpinorBlock *res, const FourSpinorBlock *psi, const FourSpinorBlock *chi,
                            const SU3MatrixBlock *u, const CloverBlock *clov, const double beta, int isign, int cb,
                            int fl = 0)
  {
    if (fl != 0 && fl != 1) throw std::invalid_argument("TMClovDslash: flavour must be 0 (up) or 1 (down)");
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    qphix_gpu_field c = this->clover_dev(clov);
    auto in = s.upload_spinor(psi);
    auto x = s.upload_spinor(chi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0);
    qphix_gpu_op_params q = this->p;
    if (fl == 1) q.prec_mass_rho = -q.prec_mass_rho;
    gpu::check(qphix_gpu_dslash_achimbdpsi(&q, out.get(), in.get(), x.get(), g, c, 0.0, beta, isign, cb,
                                           1.0),
               "tm clover dslashAChiMinusBDPsi");
    s.download_spinor(out, res);
  }

  // the two-flavour inverse clover term alone: res_up = fcl_a psi_up + C psi_dn,
  // res_dn = fcl_b psi_dn + C psi_up, (fcl_a, fcl_b) = (fcl[0], fcl[1]) for
  // isign = +1, swapped for -1 (tm_clov_dslash_body.h:1184-1343)
  void two_flav_inverse_clover_term(FourSpinorBlock *const res[2], const FourSpinorBlock *const psi[2],
                                    const FullCloverBlock *const fcl[2], const CloverBlock *const clOffDiag,
                                    int isign)
  {
    Geom &s = *this->s;
    auto in = s.upload_flavours(psi);
    qphix_gpu_field f0 = this->full_clover_dev(fcl[0]);
    qphix_gpu_field f1 = this->full_clover_dev(fcl[1]);
    qphix_gpu_field c = this->clover_dev(clOffDiag);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0, 2);
    gpu::check(qphix_gpu_two_flav_clover_apply(out.get(), in.get(), f0, f1, c, isign),
               "two_flav_inverse_clover_term");
    s.download_flavours(out, res);
  }

  // res_f = (A + i rho_f g5) chi_f - beta D psi_f - epsilon chi_{1-f}
  // (tm_clov_dslash_body.h:1345-1365)
  void two_flav_AChiMinusBDPsi(FourSpinorBlock *const res[2], const FourSpinorBlock *const psi[2],
                               const FourSpinorBlock *const chi[2], const SU3MatrixBlock *u, const CloverBlock *clov,
                               const double beta, const double epsilon, const int isign, const int cb)
  {
    Geom &s = *this->s;
    qphix_gpu_field g = this->gauge_dev(u, cb);
    qphix_gpu_field c = this->clover_dev(clov);
    auto in = s.upload_flavours(psi);
    auto x = s.upload_flavours(chi);
    gpu::Field out(s.lattice(), QPHIX_GPU_SPINOR, Geom::device_prec(), 0, 2);
    qphix_gpu_op_params q = this->p;
    q.kind = QPHIX_GPU_NDTMCLOVER;
    q.twisted_mass = this->p.prec_mass_rho;
    q.epsilon = epsilon;
    gpu::check(qphix_gpu_dslash_achimbdpsi(&q, out.get(), in.get(), x.get(), g, c, 0.0, beta, isign, cb,
                                           1.0),
               "tm clover two_flav_AChiMinusBDPsi");
    s.download_flavours(out, res);
  }
};

}  // namespace QPhiX
