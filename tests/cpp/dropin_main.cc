// Drives the QPhiX drop-in headers (include/qphix/) the way a QPhiX caller
// does: Geometry-allocated host arrays in QPhiX's blocked layout, Dslash /
// operator / solver objects, results back in the host arrays.  Inputs and
// outputs are raw binary files in a directory given on the command line;
// tests/test_dropin_gpu.py writes the inputs (packed from seeded canonical
// fields) and checks the outputs against the CPU oracle.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "qphix/blas_new_c.h"
#include "qphix/clover.h"
#include "qphix/geometry.h"
#include "qphix/inv_richardson_multiprec.h"
#include "qphix/invbicgstab.h"
#include "qphix/invcg.h"
#include "qphix/minvcg.h"
#include "qphix/ndtm_reuse_operator.h"
#include "qphix/invmr.h"
#include "qphix/ndtm_reuse_operator_clover.h"
#include "qphix/twisted_mass.h"
#include "qphix/twisted_mass_clover.h"
#include "qphix/unprec_solver_wrapper.h"
#include "qphix/wilson.h"

using namespace QPhiX;

static std::string dir;

template <typename T>
void read_into(const std::string &name, T *p, size_t bytes)
{
  std::ifstream f(dir + "/" + name, std::ios::binary);
  if (!f) throw std::runtime_error("missing input " + name);
  f.read(reinterpret_cast<char *>(p), bytes);
  if (!f) throw std::runtime_error("short input " + name);
}

template <typename T>
void write_from(const std::string &name, const T *p, size_t bytes)
{
  std::ofstream f(dir + "/" + name, std::ios::binary);
  f.write(reinterpret_cast<const char *>(p), bytes);
}

template <typename FT, int V, int S>
struct Fields {
  typedef Geometry<FT, V, S, true> G;
  G &g;
  typename G::SU3MatrixBlock *u[2];
  typename G::CloverBlock *A_odd, *Ainv_even;
  size_t gbytes, cbytes;
  Fields(G &geom, const std::string &tag) : g(geom)
  {
    gbytes = (size_t)(g.getPxyz() * g.Nt() * S / V) * sizeof(typename G::SU3MatrixBlock);
    cbytes = (size_t)(g.getPxyz() * g.Nt() * S / V) * sizeof(typename G::CloverBlock);
    for (int cb = 0; cb < 2; cb++) {
      u[cb] = g.allocCBGauge();
      read_into(tag + "u" + std::to_string(cb), u[cb], gbytes);
    }
    A_odd = g.allocCBClov();
    Ainv_even = g.allocCBClov();
    read_into(tag + "A_odd", A_odd, cbytes);
    read_into(tag + "Ainv_even", Ainv_even, cbytes);
  }
  ~Fields()
  {
    g.free(u[0]);
    g.free(u[1]);
    g.free(A_odd);
    g.free(Ainv_even);
  }
};

int main(int argc, char **argv)
{
  if (argc < 2) {
    fprintf(stderr, "usage: %s <dir>\n", argv[0]);
    return 2;
  }
  dir = argv[1];
  int latt[4];
  read_into("dims", latt, sizeof(latt));
  double mass;
  read_into("mass", &mass, sizeof(double));
  try {
    qphix_gpu_init(0);
    // double, veclen 4, soalen 2, 12-real links, padding on
    Geometry<double, 4, 2, true> geom(latt, 2, 2, 1, 1, 1, 1, 1, 1);
    Geometry<float, 8, 2, true> geomf(latt, 4, 2, 1, 1, 1, 1, 1, 1);
    Fields<double, 4, 2> F(geom, "d_");
    Fields<float, 8, 2> Ff(geomf, "f_");
    size_t sbytes = (size_t)(geom.getPxyz() * geom.Nt()) * sizeof(Geometry<double, 4, 2, true>::FourSpinorBlock);
    auto *psi = geom.allocCBFourSpinor();
    auto *res = geom.allocCBFourSpinor();
    auto *x = geom.allocCBFourSpinor();
    read_into("d_psi", psi, sbytes);

    // 1. Dslash::dslash onto cb 0 with u[0] (isign +1, antiperiodic t)
    Dslash<double, 4, 2, true> D(&geom, -1.0, 1.0, 1.0);
    D.dslash(res, psi, F.u[0], 1, 0);
    write_from("out_dslash", res, sbytes);

    // 2. EvenOddCloverOperator applied on the odd checkerboard
    EvenOddCloverOperator<double, 4, 2, true> M(F.u, F.A_odd, F.Ainv_even, &geom, -1.0, 1.0, 1.0);
    M(res, psi, 1, 1);
    write_from("out_clover_op", res, sbytes);

    // 3. InvBiCGStab on it
    int n_iters;
    double rsd_sq;
    unsigned long flops, mv;
    InvBiCGStab<double, 4, 2, true> bicg(M, 2000);
    bicg(x, psi, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
    write_from("out_bicgstab_x", x, sbytes);
    double info[3] = {(double)n_iters, rsd_sq, (double)mv};
    write_from("out_bicgstab_info", info, sizeof(info));

    // 4. InvCG on the Wilson operator
    EvenOddWilsonOperator<double, 4, 2, true> W(mass, F.u, &geom, -1.0, 1.0, 1.0);
    auto *y = geom.allocCBFourSpinor();
    InvCG<double, 4, 2, true> cg(W, 2000);
    cg(y, psi, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
    write_from("out_cg_x", y, sbytes);
    double cinfo[3] = {(double)n_iters, rsd_sq, (double)mv};
    write_from("out_cg_info", cinfo, sizeof(cinfo));

    // 5. InvRichardsonMultiPrec: double outer, float BiCGStab inner
    EvenOddCloverOperator<float, 8, 2, true> Mf(Ff.u, Ff.A_odd, Ff.Ainv_even, &geomf, -1.0, 1.0, 1.0);
    InvBiCGStab<float, 8, 2, true> inner(Mf, 2000);
    InvRichardsonMultiPrec<double, 4, 2, true, float, 8, 2, true> rich(M, inner, 0.1, 100);
    auto *z = geom.allocCBFourSpinor();
    rich(z, psi, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
    write_from("out_rich_x", z, sbytes);

    // 6. MInvCG on the clover operator
    const int ns = 3;
    double shifts[ns] = {0.01, 0.1, 0.5}, rsd[ns] = {1e-9, 1e-9, 1e-9}, fin[ns];
    Geometry<double, 4, 2, true>::FourSpinorBlock *xs[ns];
    for (int s = 0; s < ns; s++) xs[s] = geom.allocCBFourSpinor();
    MInvCG<double, 4, 2, true> mcg(M, 2000, ns);
    mcg(xs, psi, ns, shifts, rsd, n_iters, fin, flops, mv, 1, false, 1);
    for (int s = 0; s < ns; s++) write_from("out_minv_x" + std::to_string(s), xs[s], sbytes);

    // 7. two-flavour twisted mass: the operator on (psi, chi) and InvCG on the pair
    auto *chi = geom.allocCBFourSpinor();
    read_into("d_chi", chi, sbytes);
    double nd[3];
    read_into("ndtm", nd, sizeof(nd));
    EvenOddNDTMWilsonReuseOperator<double, 4, 2, true> N(nd[0], nd[1], nd[2], F.u, &geom, -1.0, 1.0, 1.0);
    Geometry<double, 4, 2, true>::FourSpinorBlock *nres[2] = {geom.allocCBFourSpinor(), geom.allocCBFourSpinor()};
    const Geometry<double, 4, 2, true>::FourSpinorBlock *nin[2] = {psi, chi};
    N(nres, nin, 1, 1);
    write_from("out_nd_up", nres[0], sbytes);
    write_from("out_nd_dn", nres[1], sbytes);
    InvCG<double, 4, 2, true, EvenOddNDTMWilsonReuseOperator<double, 4, 2, true>> ncg(N, 2000);
    ncg(nres, nin, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
    write_from("out_ndcg_up", nres[0], sbytes);
    write_from("out_ndcg_dn", nres[1], sbytes);

    // 7b. two-flavour twisted-mass clover: clov = A_odd, the caller's
    // two-flavour inverses of the even block, operator and InvCG on the pair
    {
      size_t cbytes = F.cbytes;
      size_t fbytes = (size_t)(geom.getPxyz() * geom.Nt() * 2 / 4) * sizeof(Geometry<double, 4, 2, true>::FullCloverBlock);
      auto *odiag = geom.allocCBClov();
      Geometry<double, 4, 2, true>::FullCloverBlock *finv[2] = {geom.allocCBFullClov(), geom.allocCBFullClov()};
      read_into("d_ndc_odiag", odiag, cbytes);
      read_into("d_ndc_fup", finv[0], fbytes);
      read_into("d_ndc_fdn", finv[1], fbytes);
      EvenOddNDTMCloverReuseOperator<double, 4, 2, true> NC(nd[1], nd[2], F.u, F.A_odd, odiag, finv, &geom, -1.0,
                                                            1.0, 1.0);
      NC(nres, nin, 1, 1);
      write_from("out_ndc_up", nres[0], sbytes);
      write_from("out_ndc_dn", nres[1], sbytes);
      InvCG<double, 4, 2, true, EvenOddNDTMCloverReuseOperator<double, 4, 2, true>> nccg(NC, 2000);
      nccg(nres, nin, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
      write_from("out_ndccg_up", nres[0], sbytes);
      write_from("out_ndccg_dn", nres[1], sbytes);
      // 7c. the Dslash-level two-flavour members on (psi, chi)
      const Geometry<double, 4, 2, true>::FourSpinorBlock *swp[2] = {chi, psi};
      TMClovDslash<double, 4, 2, true> TC(&geom, -1.0, 1.0, 1.0, nullptr, nullptr, nd[1]);
      TC.two_flav_inverse_clover_term(nres, nin, finv, odiag, 1);
      write_from("out_2f_inv_up", nres[0], sbytes);
      write_from("out_2f_inv_dn", nres[1], sbytes);
      TC.two_flav_AChiMinusBDPsi(nres, nin, swp, F.u[1], F.A_odd, 0.25, nd[2], 1, 1);
      write_from("out_2f_clachi_up", nres[0], sbytes);
      write_from("out_2f_clachi_dn", nres[1], sbytes);
      TMDslash<double, 4, 2, true> TD(&geom, -1.0, 1.0, 1.0, nd[0], nd[1]);
      TD.two_flav_AChiMinusBDPsi(nres, nin, swp, F.u[1], 4.0 + nd[0], 0.25, nd[2], -1, 1);
      write_from("out_2f_tmachi_up", nres[0], sbytes);
      write_from("out_2f_tmachi_dn", nres[1], sbytes);
      geom.free(odiag);
      geom.free(finv[0]);
      geom.free(finv[1]);
    }
    geom.free(nres[0]);
    geom.free(nres[1]);
    geom.free(chi);

    // 8. unpreconditioned clover solve: b = (chi on even, psi on odd) through
    // UnprecSolverWrapper around InvBiCGStab on cb 1
    {
      FullSpinor<double, 4, 2, true> fb(geom), fx(geom);
      read_into("d_chi", fb.getCBData(0), sbytes);
      read_into("d_psi", fb.getCBData(1), sbytes);
      UnprecSolverWrapper<double, 4, 2, true, EvenOddCloverOperator<double, 4, 2, true>> unprec(bicg, M);
      unprec(&fx, &fb, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
      write_from("out_unprec_e", fx.getCBData(0), sbytes);
      write_from("out_unprec_o", fx.getCBData(1), sbytes);
    }

    // 9. BLAS (blas_new_c.h) on host arrays: psi, chi as read
    {
      auto *a = geom.allocCBFourSpinor();
      auto *b = geom.allocCBFourSpinor();
      auto *c = geom.allocCBFourSpinor();
      auto *ch = geom.allocCBFourSpinor();
      read_into("d_chi", ch, sbytes);
      double out[16];
      norm2Spinor(out[0], psi, geom, 1);
      innerProduct(out + 1, psi, ch, geom, 1);
      innerProductNorm(out + 3, psi, ch, geom, 1);
      copySpinor(a, psi, geom, 1);
      axpy(0.5, ch, a, geom, 1);                    // a = psi + 0.5 chi
      write_from("out_blas_axpy", a, sbytes);
      copySpinor(b, ch, geom, 1);
      axpby(2.0, psi, -1.5, b, geom, 1);            // b = 2 psi - 1.5 chi
      write_from("out_blas_axpby", b, sbytes);
      xmyNorm2Spinor(c, psi, ch, out[6], geom, 1);  // c = psi - chi
      write_from("out_blas_xmy", c, sbytes);
      copySpinor(c, ch, geom, 1);
      aypx(-0.25, psi, c, geom, 1);                 // c = psi - 0.25 chi
      write_from("out_blas_aypx", c, sbytes);
      double ca[2] = {0.3, -0.7};
      copySpinor(c, ch, geom, 1);
      caxpySpinor(ca, psi, c, geom, 1);             // c = (0.3 - 0.7i) psi + chi
      write_from("out_blas_caxpy", c, sbytes);
      axpyNorm2(1.0, psi, c, out[7], geom, 1);      // c += psi
      copySpinor(c, psi, geom, 1);
      ymeqx(ch, c, geom, 1);                        // c = psi - chi
      ax(3.0, c, geom, 1);                          // c = 3 (psi - chi)
      write_from("out_blas_ax", c, sbytes);
      zeroSpinor(c, geom, 1);
      norm2Spinor(out[8], c, geom, 1);
      // FP64 -> float Geometry and back
      auto *f = geomf.allocCBFourSpinor();
      convert(f, 1.0, psi, geomf, geom, 1);
      convert(c, 2.0, f, geom, geomf, 1);             // c = 2 psi (through FP32)
      write_from("out_blas_convert", c, sbytes);
      write_from("out_blas_scalars", out, sizeof(double) * 9);
      geomf.free(f);
      geom.free(a);
      geom.free(b);
      geom.free(c);
      geom.free(ch);
    }

    // 10. ClovDslash members, InvMR / InvMRSmoother with over-relaxation,
    // the twisted-mass Wilson and twisted-mass clover even-odd operators
    {
      auto *chi = geom.allocCBFourSpinor();
      auto *w = geom.allocCBFourSpinor();
      read_into("d_chi", chi, sbytes);
      ClovDslash<double, 4, 2, true> CD(&geom, -1.0, 1.0, 1.0, nullptr, nullptr, 0.05);
      CD.dslash(w, psi, F.u[0], F.Ainv_even, 1, 0);
      write_from("out_clov_dslash", w, sbytes);
      CD.dslashAChiMinusBDPsi(w, psi, chi, F.u[1], F.A_odd, 0.25, -1, 1);
      write_from("out_clov_achi", w, sbytes);
      CD.clovMult(w, psi, F.A_odd);
      write_from("out_clovmult", w, sbytes);

      InvMR<double, 4, 2, true> mr(M, 2000, 1.1);
      zeroSpinor(w, geom, 1);
      mr(w, psi, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
      write_from("out_mr_x", w, sbytes);
      double minfo[3] = {(double)n_iters, rsd_sq, (double)mv};
      write_from("out_mr_info", minfo, sizeof(minfo));
      InvMRSmoother<double, 4, 2, true> sm(M, 5, 1.2);
      zeroSpinor(w, geom, 1);
      sm(w, psi, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
      write_from("out_mrs_x", w, sbytes);
      double sinfo[3] = {(double)n_iters, rsd_sq, (double)mv};
      write_from("out_mrs_info", sinfo, sizeof(sinfo));

      double tm[1];
      read_into("tm_mu", tm, sizeof(tm));
      EvenOddTMWilsonOperator<double, 4, 2, true> TW(mass, tm[0], F.u, &geom, -1.0, 1.0, 1.0);
      TW(w, psi, 1, 1);
      write_from("out_tmw_op", w, sbytes);
      InvBiCGStab<double, 4, 2, true, EvenOddTMWilsonOperator<double, 4, 2, true>> tbicg(TW, 2000);
      zeroSpinor(w, geom, 1);
      tbicg(w, psi, 1e-10, n_iters, rsd_sq, flops, mv, 1, false, 1);
      write_from("out_tmw_bicg_x", w, sbytes);

      size_t fbytes = (size_t)(geom.getPxyz() * geom.Nt() * 2 / 4) * sizeof(Geometry<double, 4, 2, true>::FullCloverBlock);
      Geometry<double, 4, 2, true>::FullCloverBlock *tinv[2] = {geom.allocCBFullClov(), geom.allocCBFullClov()};
      read_into("d_tm_finv0", tinv[0], fbytes);
      read_into("d_tm_finv1", tinv[1], fbytes);
      EvenOddTMCloverOperator<double, 4, 2, true> TMC(F.u, F.A_odd, tinv, &geom, -1.0, 1.0, 1.0, nullptr, nullptr,
                                                      tm[0]);
      TMC(w, psi, -1, 1);
      write_from("out_tmc_op", w, sbytes);
      geom.free(tinv[0]);
      geom.free(tinv[1]);
      geom.free(chi);
      geom.free(w);
    }

    // 11. the device copy of the gauge array is kept between calls: repeated
    // calls, an in-place rewrite announced with invalidateFieldCache(), and an
    // array released and allocated again
    {
      auto *w = geom.allocCBFourSpinor();
      Dslash<double, 4, 2, true> DC(&geom, -1.0, 1.0, 1.0);
      DC.dslash(w, psi, F.u[0], 1, 0);
      DC.dslash(w, psi, F.u[0], 1, 0);
      write_from("out_cache_1", w, sbytes);
      read_into("d_u0b", F.u[0], F.gbytes);  // rewritten in place
      DC.invalidateFieldCache();
      DC.dslash(w, psi, F.u[0], 1, 0);
      write_from("out_cache_2", w, sbytes);
      auto *ua = geom.allocCBGauge();
      read_into("d_u0", ua, F.gbytes);
      DC.dslash(w, psi, ua, 1, 0);
      geom.free(ua);
      auto *ub = geom.allocCBGauge();  // may reuse ua's address
      read_into("d_u0b", ub, F.gbytes);
      DC.dslash(w, psi, ub, 1, 0);
      write_from("out_cache_3", w, sbytes);
      geom.free(ub);
      geom.free(w);
    }

    for (int s = 0; s < ns; s++) geom.free(xs[s]);
    geom.free(psi);
    geom.free(res);
    geom.free(x);
    geom.free(y);
    geom.free(z);
  } catch (const std::exception &e) {
    fprintf(stderr, "drop-in test failed: %s\n", e.what());
    return 1;
  }
  printf("drop-in ok\n");
  return 0;
}
