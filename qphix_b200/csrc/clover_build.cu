// Clover term construction and inversion on the device.
//
// QPhiX takes the clover term and its inverse as inputs (its callers build
// them with Chroma's QDPCloverTerm); these kernels produce the same packed
// arrays on the GPU from a resident gauge field, so that a solve never has to
// leave the device:
//   clover_build   A = diag_mass + sigma.F in the clover-leaf normalisation
//                  of tests/mesfield.cc:25-64 (F = (Q - Q^+)/8, Q the four
//                  plaquette leaves) and the packing of
//                  tests/clover_term_qdp_w.h:114-200,325-442 (coefficients
//                  x 1/2), two 6x6 Hermitian blocks (diag[6], offd[15])
//   clover_invert  packed A^-1 (exact 6x6 inverse per block)
//   clover_invert_twisted  full (A + i mu g5)^-1 and (A - i mu g5)^-1 for
//                  the twisted-mass clover operator (g5 = +1 on block 0)
//   clover_invert_ndtm  the inverse of the two-flavour diagonal block
//                  [[A + i mu g5, -eps], [-eps, A - i mu g5]]: with
//                  Q = (A^2 + mu^2 - eps^2)^-1 (A commutes with g5) it is
//                  [[Q (A - i mu g5), eps Q], [eps Q, Q (A + i mu g5)]]; the
//                  flavour-diagonal blocks as full clover fields, eps Q packed
//                  (the fields include/qphix/ndtm_reuse_operator_clover.h:38-50
//                   takes, tm_clov_dslash_def.h:96-104)
// All arithmetic in FP64; results are stored in the destination field's
// precision.
#include "qpx_finalize.cuh"
#include "qpx_host.h"

namespace qpx {

typedef cx<double> zd;

struct M3 {
  zd m[3][3];
};

__device__ __forceinline__ M3 mm(const M3 &a, const M3 &b)
{
  M3 c;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      zd v = a.m[i][0] * b.m[0][j];
      v = v + a.m[i][1] * b.m[1][j];
      v = v + a.m[i][2] * b.m[2][j];
      c.m[i][j] = v;
    }
  return c;
}

__device__ __forceinline__ M3 dag(const M3 &a)
{
  M3 c;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) c.m[i][j] = conj(a.m[j][i]);
  return c;
}

template <int RECON>
__device__ __forceinline__ M3 link_at(const GaugeArg &g, const Geom &geo, int c0, int c1, int c2, int c3, int mu)
{
  int n[4] = {geo.nx, geo.ny, geo.nz, geo.nt};
  int c[4] = {c0, c1, c2, c3};
#pragma unroll
  for (int d = 0; d < 4; d++) c[d] = (c[d] % n[d] + n[d]) % n[d];
  int cb = (c[0] + c[1] + c[2] + c[3]) & 1;
  int s = ((c[3] * geo.nz + c[2]) * geo.ny + c[1]) * geo.nxh + c[0] / 2;
  M3 u;
  GaugeIO<F64, RECON>::load(g, cb, mu, s, u.m);
  return u;
}

template <int RECON, typename Q>
__global__ void clover_build_kernel(Geom geo, GaugeArg g, void *out, long long stride, int vpc, int cb,
                                    double diag_mass, double coeff_r, double coeff_t)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= geo.vh) return;
  int xh, y, z, t, par;
  site_coords(geo, s, cb, xh, y, z, t, par);
  const int x[4] = {2 * xh + par, y, z, t};
  // F for the planes (0,1),(0,2),(0,3),(1,2),(1,3),(2,3), times their coefficient
  M3 f[6];
  int k = 0;
  for (int mu = 0; mu < 3; mu++) {
    for (int nu = mu + 1; nu < 4; nu++, k++) {
      int e[4] = {0, 0, 0, 0}, d[4] = {0, 0, 0, 0};
      e[mu] = 1;
      d[nu] = 1;
#define AT(a, b, dir) link_at<RECON>(g, geo, x[0] + (a) * e[0] + (b) * d[0], x[1] + (a) * e[1] + (b) * d[1], \
                                     x[2] + (a) * e[2] + (b) * d[2], x[3] + (a) * e[3] + (b) * d[3], dir)
      M3 q;
      // U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
      q = mm(mm(AT(0, 0, mu), AT(1, 0, nu)), mm(dag(AT(0, 1, mu)), dag(AT(0, 0, nu))));
      // U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
      M3 l = mm(mm(AT(0, 0, nu), dag(AT(-1, 1, mu))), mm(dag(AT(-1, 0, nu)), AT(-1, 0, mu)));
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) q.m[i][j] = q.m[i][j] + l.m[i][j];
      // U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
      l = mm(mm(dag(AT(-1, 0, mu)), dag(AT(-1, -1, nu))), mm(AT(-1, -1, mu), AT(0, -1, nu)));
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) q.m[i][j] = q.m[i][j] + l.m[i][j];
      // U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^+
      l = mm(mm(dag(AT(0, -1, nu)), AT(0, -1, mu)), mm(AT(1, -1, nu), dag(AT(0, 0, mu))));
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) q.m[i][j] = q.m[i][j] + l.m[i][j];
#undef AT
      const double cf = 0.125 * ((mu == 3 || nu == 3) ? coeff_t : coeff_r);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          zd a = q.m[i][j], b = conj(q.m[j][i]);
          f[k].m[i][j] = cf * (a - b);
        }
    }
  }
  const M3 &f0 = f[0], &f1 = f[1], &f2 = f[2], &f3 = f[3], &f4 = f[4], &f5 = f[5];
  double diag[2][6];
  zd offd[2][15];
  for (int b = 0; b < 2; b++)
    for (int i = 0; i < 6; i++) diag[b][i] = diag_mass;
  for (int i = 0; i < 3; i++) {
    double r0 = (f5.m[i][i] - f0.m[i][i]).im;
    diag[0][i] += r0;
    diag[0][i + 3] -= r0;
    double r1 = (f5.m[i][i] + f0.m[i][i]).im;
    diag[1][i] -= r1;
    diag[1][i + 3] += r1;
  }
  for (int i = 1; i < 3; i++)
    for (int j = 0; j < i; j++) {
      int eij = i * (i - 1) / 2 + j;
      int etmp = (i + 3) * (i + 2) / 2 + j + 3;
      offd[0][eij] = itimes(f0.m[i][j] - f5.m[i][j]);
      offd[0][etmp] = zd{-offd[0][eij].re, -offd[0][eij].im};
      offd[1][eij] = itimes(f5.m[i][j] + f0.m[i][j]);
      offd[1][etmp] = zd{-offd[1][eij].re, -offd[1][eij].im};
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      int e = (i + 3) * (i + 2) / 2 + j;
      zd em = itimes(f2.m[i][j]) + f4.m[i][j];
      zd bm = itimes(f3.m[i][j]) - f1.m[i][j];
      offd[0][e] = bm - em;
      offd[1][e] = em + bm;
    }
  for (int b = 0; b < 2; b++) {
    for (int i = 0; i < 6; i++) dev_store_real<Q>(out, stride, vpc, s, 36 * b + i, diag[b][i]);
    for (int o = 0; o < 15; o++) {
      dev_store_real<Q>(out, stride, vpc, s, 36 * b + 6 + 2 * o, offd[b][o].re);
      dev_store_real<Q>(out, stride, vpc, s, 36 * b + 7 + 2 * o, offd[b][o].im);
    }
  }
}

// in-place Gauss-Jordan inverse of a 6x6 complex matrix with partial pivoting
__device__ void invert6(zd a[6][6], zd inv[6][6])
{
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) inv[i][j] = zd{i == j ? 1.0 : 0.0, 0.0};
  for (int c = 0; c < 6; c++) {
    int piv = c;
    double best = a[c][c].re * a[c][c].re + a[c][c].im * a[c][c].im;
    for (int r = c + 1; r < 6; r++) {
      double v = a[r][c].re * a[r][c].re + a[r][c].im * a[r][c].im;
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (piv != c) {
      for (int j = 0; j < 6; j++) {
        zd tmp = a[c][j];
        a[c][j] = a[piv][j];
        a[piv][j] = tmp;
        tmp = inv[c][j];
        inv[c][j] = inv[piv][j];
        inv[piv][j] = tmp;
      }
    }
    // 1 / pivot
    double d = a[c][c].re * a[c][c].re + a[c][c].im * a[c][c].im;
    zd p = {a[c][c].re / d, -a[c][c].im / d};
    for (int j = 0; j < 6; j++) {
      a[c][j] = a[c][j] * p;
      inv[c][j] = inv[c][j] * p;
    }
    for (int r = 0; r < 6; r++) {
      if (r == c) continue;
      zd fct = a[r][c];
      for (int j = 0; j < 6; j++) {
        a[r][j] = a[r][j] - fct * a[c][j];
        inv[r][j] = inv[r][j] - fct * inv[c][j];
      }
    }
  }
}

// mode 0: packed Hermitian inverse of A; mode 1: full inverses of A +/- i mu g5;
// mode 2: the two-flavour inverses (full out0 = up, out1 = down, packed out2)
template <typename Pin, typename Q>
__global__ void clover_invert_kernel(Geom geo, const void *in, long long stride, int vpc_in, void *out0, void *out1,
                                     int vpc_out, int mode, double mu, void *out2, int vpc_out2, double eps)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= geo.vh) return;
  for (int b = 0; b < 2; b++) {
    zd a[6][6];
    for (int i = 0; i < 6; i++) a[i][i] = zd{dev_load_real<Pin>(in, stride, vpc_in, s, 36 * b + i), 0.0};
    for (int i = 1; i < 6; i++)
      for (int j = 0; j < i; j++) {
        int od = i * (i - 1) / 2 + j;
        zd v = {dev_load_real<Pin>(in, stride, vpc_in, s, 36 * b + 6 + 2 * od),
                dev_load_real<Pin>(in, stride, vpc_in, s, 36 * b + 7 + 2 * od)};
        a[i][j] = v;
        a[j][i] = conj(v);
      }
    if (mode == 2) {
      const double g5 = (b == 0) ? 1.0 : -1.0;
      zd m[6][6], q[6][6];
      for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) {
          zd v = {0.0, 0.0};
          for (int k = 0; k < 6; k++) v = v + a[i][k] * a[k][j];
          m[i][j] = v;
        }
      for (int i = 0; i < 6; i++) m[i][i].re += mu * mu - eps * eps;
      invert6(m, q);
      for (int f = 0; f < 2; f++) {  // up: Q (A - i mu g5), down: Q (A + i mu g5)
        const double tw = (f == 0 ? -1.0 : 1.0) * mu * g5;
        void *o = f == 0 ? out0 : out1;
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) {
            zd v = {0.0, 0.0};
            for (int k = 0; k < 6; k++) v = v + q[i][k] * a[k][j];
            v.re -= tw * q[i][j].im;  // + i tw Q_ij
            v.im += tw * q[i][j].re;
            dev_store_real<Q>(o, stride, vpc_out, s, 72 * b + (i * 6 + j) * 2, v.re);
            dev_store_real<Q>(o, stride, vpc_out, s, 72 * b + (i * 6 + j) * 2 + 1, v.im);
          }
      }
      for (int i = 0; i < 6; i++) dev_store_real<Q>(out2, stride, vpc_out2, s, 36 * b + i, eps * q[i][i].re);
      for (int i = 1; i < 6; i++)
        for (int j = 0; j < i; j++) {
          int od = i * (i - 1) / 2 + j;
          dev_store_real<Q>(out2, stride, vpc_out2, s, 36 * b + 6 + 2 * od, eps * q[i][j].re);
          dev_store_real<Q>(out2, stride, vpc_out2, s, 36 * b + 7 + 2 * od, eps * q[i][j].im);
        }
    } else if (mode == 0) {
      zd inv[6][6];
      invert6(a, inv);
      for (int i = 0; i < 6; i++) dev_store_real<Q>(out0, stride, vpc_out, s, 36 * b + i, inv[i][i].re);
      for (int i = 1; i < 6; i++)
        for (int j = 0; j < i; j++) {
          int od = i * (i - 1) / 2 + j;
          dev_store_real<Q>(out0, stride, vpc_out, s, 36 * b + 6 + 2 * od, inv[i][j].re);
          dev_store_real<Q>(out0, stride, vpc_out, s, 36 * b + 7 + 2 * od, inv[i][j].im);
        }
    } else {
      for (int sgn = 0; sgn < 2; sgn++) {
        zd m[6][6], inv[6][6];
        double g5 = (b == 0) ? 1.0 : -1.0;
        double tw = (sgn == 0 ? 1.0 : -1.0) * mu * g5;
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) m[i][j] = a[i][j];
        for (int i = 0; i < 6; i++) m[i][i].im += tw;
        invert6(m, inv);
        void *o = sgn == 0 ? out0 : out1;
        for (int i = 0; i < 6; i++)
          for (int j = 0; j < 6; j++) {
            dev_store_real<Q>(o, stride, vpc_out, s, 72 * b + (i * 6 + j) * 2, inv[i][j].re);
            dev_store_real<Q>(o, stride, vpc_out, s, 72 * b + (i * 6 + j) * 2 + 1, inv[i][j].im);
          }
      }
    }
  }
}

// The two-flavour inverse clover term on its own (no hop), one (up, down)
// pair per thread: out_up = Fa psi_up + C psi_dn, out_dn = Fb psi_dn + C psi_up
// (TMClovDslash::two_flav_inverse_clover_term, tm_clov_dslash_body.h:1184-1343;
// per-site form codegen/dslash_common.cc:1198-1341), FP64 arithmetic
template <typename P>
__global__ void two_flav_clover_kernel(int vh, int npairs, SpinorArg out, SpinorArg in, CloverArg fa, CloverArg fb,
                                       CloverArg c)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (s >= vh || k >= npairs) return;
  using T = typename P::real;
  T up[24], dn[24], f[72], cl[36];
  SpinorIO<P>::load(in, 2 * k, s, up);
  SpinorIO<P>::load(in, 2 * k + 1, s, dn);
  double ou[24], od[24];
  for (int b = 0; b < 2; b++) {
    // one 6-vector block: index i = 3 (spin - 2b) + colour
    zd xu[6], xd[6];
    for (int i = 0; i < 6; i++) {
      const int e = ((2 * b + i / 3) * 3 + i % 3) * 2;
      xu[i] = zd{(double)up[e], (double)up[e + 1]};
      xd[i] = zd{(double)dn[e], (double)dn[e + 1]};
    }
    zd yu[6], yd[6];
    CloverIO<P, 144>::load(fa, s, 72 * b, 72, f);
    for (int i = 0; i < 6; i++) {
      zd v = {0.0, 0.0};
      for (int j = 0; j < 6; j++) v = v + zd{(double)f[(i * 6 + j) * 2], (double)f[(i * 6 + j) * 2 + 1]} * xu[j];
      yu[i] = v;
    }
    CloverIO<P, 144>::load(fb, s, 72 * b, 72, f);
    for (int i = 0; i < 6; i++) {
      zd v = {0.0, 0.0};
      for (int j = 0; j < 6; j++) v = v + zd{(double)f[(i * 6 + j) * 2], (double)f[(i * 6 + j) * 2 + 1]} * xd[j];
      yd[i] = v;
    }
    // packed Hermitian C: up += C dn, dn += C up
    CloverIO<P, 72>::load(c, s, 36 * b, 36, cl);
    for (int i = 0; i < 6; i++) {
      yu[i] = yu[i] + zd{(double)cl[i], 0.0} * xd[i];
      yd[i] = yd[i] + zd{(double)cl[i], 0.0} * xu[i];
    }
    for (int i = 1; i < 6; i++)
      for (int j = 0; j < i; j++) {
        const int od = i * (i - 1) / 2 + j;
        const zd a = {(double)cl[6 + 2 * od], (double)cl[7 + 2 * od]};
        yu[i] = yu[i] + a * xd[j];
        yu[j] = yu[j] + conj(a) * xd[i];
        yd[i] = yd[i] + a * xu[j];
        yd[j] = yd[j] + conj(a) * xu[i];
      }
    for (int i = 0; i < 6; i++) {
      const int e = ((2 * b + i / 3) * 3 + i % 3) * 2;
      ou[e] = yu[i].re;
      ou[e + 1] = yu[i].im;
      od[e] = yd[i].re;
      od[e + 1] = yd[i].im;
    }
  }
  for (int e = 0; e < 24; e++) {
    up[e] = (T)ou[e];
    dn[e] = (T)od[e];
  }
  SpinorIO<P>::store(out, 2 * k, s, up);
  SpinorIO<P>::store(out, 2 * k + 1, s, dn);
}

template <typename Pin, typename Q>
__global__ void clover_convert_kernel(Geom geo, const void *in, int vpc_in, void *out, int vpc_out, long long stride,
                                      int nr)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= geo.vh) return;
  for (int k = 0; k < nr; k++)
    dev_store_real<Q>(out, stride, vpc_out, s, k, dev_load_real<Pin>(in, stride, vpc_in, s, k));
}

#define QPX_OUT_SWITCH(prec, CALL)                          \
  switch (prec) {                                           \
  case PREC_F64: { using Q = F64; CALL; } break;            \
  case PREC_F32: { using Q = F32; CALL; } break;            \
  case PREC_F16: { using Q = F16; CALL; } break;            \
  case PREC_BF16: { using Q = BF16; CALL; } break;          \
  case PREC_Q16: { using Q = F16; CALL; } break;            \
  case PREC_Q16F32: { using Q = F32; CALL; } break;         \
  default: throw Error(QPHIX_GPU_EINVAL, "bad precision");  \
  }
#define QPX_IN_SWITCH(prec, CALL)                           \
  switch (prec) {                                           \
  case PREC_F64: { using Pin = F64; CALL; } break;          \
  case PREC_F32: { using Pin = F32; CALL; } break;          \
  case PREC_F16: { using Pin = F16; CALL; } break;          \
  case PREC_BF16: { using Pin = BF16; CALL; } break;        \
  case PREC_Q16: { using Pin = F16; CALL; } break;          \
  case PREC_Q16F32: { using Pin = F32; CALL; } break;       \
  default: throw Error(QPHIX_GPU_EINVAL, "bad precision");  \
  }

void launch_clover_build(int recon, int prec_out, Geom geo, GaugeArg g, void *out, long long stride, int vpc, int cb,
                         double diag_mass, double cr, double ct, dim3 grid, cudaStream_t st)
{
  if (recon == 12) {
    QPX_OUT_SWITCH(prec_out, (clover_build_kernel<12, Q><<<grid, 64, 0, st>>>(geo, g, out, stride, vpc, cb, diag_mass,
                                                                                cr, ct)));
  } else {
    QPX_OUT_SWITCH(prec_out, (clover_build_kernel<18, Q><<<grid, 64, 0, st>>>(geo, g, out, stride, vpc, cb, diag_mass,
                                                                                cr, ct)));
  }
}

void launch_clover_invert(int prec_in, int prec_out, Geom geo, const void *in, long long stride, int vpc_in, void *o0,
                          void *o1, int vpc_out, int mode, double mu, dim3 grid, cudaStream_t st, void *o2,
                          int vpc_out2, double eps)
{
  QPX_IN_SWITCH(prec_in, QPX_OUT_SWITCH(prec_out, (clover_invert_kernel<Pin, Q><<<grid, 64, 0, st>>>(
                                                       geo, in, stride, vpc_in, o0, o1, vpc_out, mode, mu, o2,
                                                       vpc_out2, eps))));
}

void launch_two_flav_clover(int prec, int vh, int npairs, SpinorArg out, SpinorArg in, CloverArg fa, CloverArg fb,
                            CloverArg c, cudaStream_t st)
{
  dim3 grid((unsigned)((vh + 63) / 64), (unsigned)npairs);
  switch (prec) {
  case PREC_F64: two_flav_clover_kernel<F64><<<grid, 64, 0, st>>>(vh, npairs, out, in, fa, fb, c); break;
  case PREC_F32: two_flav_clover_kernel<F32><<<grid, 64, 0, st>>>(vh, npairs, out, in, fa, fb, c); break;
  case PREC_F16: two_flav_clover_kernel<F16><<<grid, 64, 0, st>>>(vh, npairs, out, in, fa, fb, c); break;
  case PREC_BF16: two_flav_clover_kernel<BF16><<<grid, 64, 0, st>>>(vh, npairs, out, in, fa, fb, c); break;
  case PREC_Q16: two_flav_clover_kernel<Q16><<<grid, 64, 0, st>>>(vh, npairs, out, in, fa, fb, c); break;
  case PREC_Q16F32: two_flav_clover_kernel<Q16F32><<<grid, 64, 0, st>>>(vh, npairs, out, in, fa, fb, c); break;
  default: throw Error(QPHIX_GPU_EINVAL, "bad precision");
  }
}

void launch_clover_convert(int prec_in, int prec_out, Geom geo, const void *in, int vpc_in, void *out, int vpc_out,
                           long long stride, int nr, dim3 grid, cudaStream_t st)
{
  QPX_IN_SWITCH(prec_in, QPX_OUT_SWITCH(prec_out, (clover_convert_kernel<Pin, Q><<<grid, QPX_BLOCK, 0, st>>>(
                                                       geo, in, vpc_in, out, vpc_out, stride, nr))));
}

}  // namespace qpx
