/*
 * CPU oracle for the QPhiX hot path -- TEST INFRASTRUCTURE ONLY (see
 * qphix_oracle.h for the layouts and for how this file is pinned to the
 * reference).  Deliberately naive: full 4x4 gamma matrices, explicit 3x3
 * complex products, one site at a time, FP64 throughout.
 */
#include "qphix_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

long or_vh(const or_lattice *L)
{
  return (long)(L->dims[0] / 2) * L->dims[1] * L->dims[2] * L->dims[3];
}

/* DeGrand-Rossi (Chroma) gamma matrices.  The projector tables of the
   reference (codegen/dslash_common.cc:848-866) are (1 -/+ gamma_mu) with these
   matrices; gamma_5 = gamma_0 gamma_1 gamma_2 gamma_3 = diag(1, 1, -1, -1). */
static cplx G[4][4][4];
/* filled once at library load, before any parallel region reads it */
__attribute__((constructor)) static void init_gamma(void)
{
  memset(G, 0, sizeof(G));
  /* gamma_0 (x) */
  G[0][0][3] = I;  G[0][1][2] = I;  G[0][2][1] = -I; G[0][3][0] = -I;
  /* gamma_1 (y) */
  G[1][0][3] = -1; G[1][1][2] = 1;  G[1][2][1] = 1;  G[1][3][0] = -1;
  /* gamma_2 (z) */
  G[2][0][2] = I;  G[2][1][3] = -I; G[2][2][0] = -I; G[2][3][1] = I;
  /* gamma_3 (t) */
  G[3][0][2] = 1;  G[3][1][3] = 1;  G[3][2][0] = 1;  G[3][3][1] = 1;
}

static inline void coords(const or_lattice *L, long s, int cb, int c[4])
{
  int nxh = L->dims[0] / 2;
  long r = s;
  int xh = (int)(r % nxh); r /= nxh;
  c[1] = (int)(r % L->dims[1]); r /= L->dims[1];
  c[2] = (int)(r % L->dims[2]); r /= L->dims[2];
  c[3] = (int)r;
  c[0] = 2 * xh + ((c[1] + c[2] + c[3] + cb) & 1);
}

static inline long cbindex(const or_lattice *L, const int c[4])
{
  int nxh = L->dims[0] / 2;
  return (((long)c[3] * L->dims[2] + c[2]) * L->dims[1] + c[1]) * nxh + c[0] / 2;
}

static inline void load_spinor(const double *f, long s, cplx out[4][3])
{
  const double *p = f + s * 24;
  for (int sp = 0; sp < 4; sp++)
    for (int c = 0; c < 3; c++)
      out[sp][c] = p[(sp * 3 + c) * 2] + I * p[(sp * 3 + c) * 2 + 1];
}

static inline void store_spinor(double *f, long s, cplx in[4][3])
{
  double *p = f + s * 24;
  for (int sp = 0; sp < 4; sp++)
    for (int c = 0; c < 3; c++) {
      p[(sp * 3 + c) * 2] = creal(in[sp][c]);
      p[(sp * 3 + c) * 2 + 1] = cimag(in[sp][c]);
    }
}

static inline void load_link(const or_lattice *L, const double *g, int cb,
                             int mu, long s, cplx u[3][3])
{
  long vh = or_vh(L);
  const double *p = g + ((((long)cb * 4 + mu) * vh + s) * 18);
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      u[r][c] = p[(r * 3 + c) * 2] + I * p[(r * 3 + c) * 2 + 1];
}

/* One hop, as in tests/dslashm_w.cc:64-122 with the link coefficient of
   include/qphix/dslash_body.h:484-512 and the twisted-boundary phase of
   codegen/dslash_common.cc:1739-1772 (forward hop x phase, backward hop x
   conj(phase), on every hop of the dimension).
   fwd=1: U_mu(x) (1 - isign g_mu) psi(x+mu); fwd=0: U_mu(x-mu)^+ (1 + isign g_mu) psi(x-mu) */
static void hop(const or_lattice *L, const double *psi, const double *gauge,
                int cb, const int c[4], int mu, int fwd, int isign,
                cplx acc[4][3])
{
  int n[4] = {c[0], c[1], c[2], c[3]};
  int N = L->dims[mu];
  n[mu] = fwd ? (c[mu] + 1) % N : (c[mu] - 1 + N) % N;
  long ns = cbindex(L, n);
  cplx p[4][3], proj[4][3];
  load_spinor(psi, ns, p);
  double sg = fwd ? -(double)isign : (double)isign;
  for (int i = 0; i < 4; i++)
    for (int col = 0; col < 3; col++) {
      cplx v = p[i][col];
      for (int j = 0; j < 4; j++) v += sg * G[mu][i][j] * p[j][col];
      proj[i][col] = v;
    }
  cplx u[3][3];
  if (fwd)
    load_link(L, gauge, cb, mu, cbindex(L, c), u);
  else
    load_link(L, gauge, 1 - cb, mu, ns, u);
  double coeff = (mu == 3) ? L->aniso_t : L->aniso_s;
  if (mu == 3) {
    if (fwd && c[3] == L->dims[3] - 1) coeff *= L->t_boundary;
    if (!fwd && c[3] == 0) coeff *= L->t_boundary;
  }
  cplx phase = 1.0;
  if (L->use_tbc[mu]) {
    phase = L->tbc[mu][0] + I * L->tbc[mu][1];
    if (!fwd) phase = conj(phase);
  }
  for (int i = 0; i < 4; i++)
    for (int r = 0; r < 3; r++) {
      cplx v = 0;
      for (int k = 0; k < 3; k++)
        v += (fwd ? u[r][k] : conj(u[k][r])) * proj[i][k];
      acc[i][r] += coeff * phase * v;
    }
}

static void dslash_site(const or_lattice *L, const double *psi,
                        const double *gauge, int isign, int cb, long s,
                        cplx out[4][3])
{
  int c[4];
  coords(L, s, cb, c);
  memset(out, 0, sizeof(cplx) * 12);
  for (int mu = 0; mu < 4; mu++) {
    hop(L, psi, gauge, cb, c, mu, 1, isign, out);
    hop(L, psi, gauge, cb, c, mu, 0, isign, out);
  }
}

/* include/qphix/dslash_body.h:339-347 (Dslash::dslash) */
void or_dslash(const or_lattice *L, double *res, const double *psi,
               const double *gauge, int isign, int cb)
{
  long vh = or_vh(L);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx out[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, out);
    store_spinor(res, s, out);
  }
}

/* include/qphix/dslash_body.h:362-373,1160-1230: res = alpha chi - beta D psi */
void or_dslash_achimbdpsi(const or_lattice *L, double *res, const double *psi,
                          const double *chi, const double *gauge, double alpha,
                          double beta, int isign, int cb)
{
  long vh = or_vh(L);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx d[4][3], x[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, d);
    load_spinor(chi, s, x);
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) d[i][c] = alpha * x[i][c] - beta * d[i][c];
    store_spinor(res, s, d);
  }
}

/* include/qphix/dslash_body.h:1075-1157 (DPsiDir, isign fixed to +1):
   dir = 2 mu + 0 accumulates the forward-neighbour hop, 2 mu + 1 the
   backward-neighbour hop. */
void or_dslash_dir(const or_lattice *L, double *res, const double *psi,
                   const double *gauge, int cb, int dir)
{
  long vh = or_vh(L);
  int mu = dir / 2;
  int fwd = (dir % 2 == 0);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    int c[4];
    cplx out[4][3];
    coords(L, s, cb, c);
    memset(out, 0, sizeof(out));
    hop(L, psi, gauge, cb, c, mu, fwd, 1, out);
    store_spinor(res, s, out);
  }
}

/* ---- clover ------------------------------------------------------------- */

static inline void clov_site(const double *cl, cplx in[4][3], cplx out[4][3])
{
  for (int b = 0; b < 2; b++) {
    const double *blk = cl + b * 36;
    cplx A[6][6];
    for (int i = 0; i < 6; i++) A[i][i] = blk[i];
    for (int i = 1; i < 6; i++)
      for (int j = 0; j < i; j++) {
        int od = i * (i - 1) / 2 + j;
        A[i][j] = blk[6 + 2 * od] + I * blk[6 + 2 * od + 1];
        A[j][i] = conj(A[i][j]);
      }
    for (int i = 0; i < 6; i++) {
      cplx v = 0;
      for (int j = 0; j < 6; j++) v += A[i][j] * in[2 * b + j / 3][j % 3];
      out[2 * b + i / 3][i % 3] = v;
    }
  }
}

static inline void fclov_site(const double *fc, cplx in[4][3], cplx out[4][3])
{
  for (int b = 0; b < 2; b++) {
    const double *blk = fc + b * 72;
    for (int i = 0; i < 6; i++) {
      cplx v = 0;
      for (int j = 0; j < 6; j++)
        v += (blk[(i * 6 + j) * 2] + I * blk[(i * 6 + j) * 2 + 1]) *
             in[2 * b + j / 3][j % 3];
      out[2 * b + i / 3][i % 3] = v;
    }
  }
}

/* include/qphix/clover_dslash_body.h:1167 (clovMult): res = A chi */
void or_clover_apply(long vh, double *res, const double *in, const double *clov)
{
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx x[4][3], y[4][3];
    load_spinor(in, s, x);
    clov_site(clov + s * 72, x, y);
    store_spinor(res, s, y);
  }
}

void or_fullclover_apply(long vh, double *res, const double *in,
                         const double *fclov)
{
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx x[4][3], y[4][3];
    load_spinor(in, s, x);
    fclov_site(fclov + s * 144, x, y);
    store_spinor(res, s, y);
  }
}

/* include/qphix/clover_dslash_body.h:339 (ClovDslash::dslash): A^-1 D psi */
void or_clov_dslash(const or_lattice *L, double *res, const double *psi,
                    const double *gauge, const double *invclov, int isign,
                    int cb)
{
  long vh = or_vh(L);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx d[4][3], y[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, d);
    clov_site(invclov + s * 72, d, y);
    store_spinor(res, s, y);
  }
}

/* i rho gamma_5 chi for isign = +1, -i rho gamma_5 chi for isign = -1
   (codegen/dslash_common.cc:2128-2157) */
static inline void add_i_rho_g5(cplx out[4][3], cplx chi[4][3], double rho,
                                int isign)
{
  for (int sp = 0; sp < 4; sp++) {
    double g5 = (sp < 2) ? 1.0 : -1.0;
    for (int c = 0; c < 3; c++) out[sp][c] += I * rho * g5 * isign * chi[sp][c];
  }
}

/* include/qphix/clover_dslash_body.h:351: A chi + i rho (isign) g5 chi - beta D psi */
void or_clov_achimbdpsi(const or_lattice *L, double *res, const double *psi,
                        const double *chi, const double *gauge,
                        const double *clov, double beta, double rho, int isign,
                        int cb)
{
  long vh = or_vh(L);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx d[4][3], x[4][3], y[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, d);
    load_spinor(chi, s, x);
    clov_site(clov + s * 72, x, y);
    add_i_rho_g5(y, x, rho, isign);
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) y[i][c] -= beta * d[i][c];
    store_spinor(res, s, y);
  }
}

/* ---- twisted mass --------------------------------------------------------- */

/* include/qphix/tm_dslash_body.h:32-34,344 with codegen/dslash_common.cc:1482-1607:
   res = (alpha - i mu isign g5)/(alpha^2 + mu^2) D psi, alpha = 4 + mass */
void or_tm_dslash(const or_lattice *L, double *res, const double *psi,
                  const double *gauge, double mass, double twisted_mass,
                  int isign, int cb)
{
  long vh = or_vh(L);
  double alpha = 4.0 + mass;
  double dmu = twisted_mass / alpha;
  double dmu_inv = alpha / (twisted_mass * twisted_mass + alpha * alpha);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx d[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, d);
    for (int sp = 0; sp < 4; sp++) {
      double g5 = (sp < 2) ? 1.0 : -1.0;
      for (int c = 0; c < 3; c++)
        d[sp][c] = dmu_inv * (1.0 - I * dmu * g5 * isign) * d[sp][c];
    }
    store_spinor(res, s, d);
  }
}

/* include/qphix/tm_dslash_body.h:354,986 with codegen/dslash_common.cc:1612-1737:
   res = alpha (1 + i (musign mu/(4+m)) isign g5) chi - beta D psi */
void or_tm_achimbdpsi(const or_lattice *L, double *res, const double *psi,
                      const double *chi, const double *gauge, double alpha,
                      double beta, double mass, double twisted_mass, int isign,
                      int cb, double musign)
{
  long vh = or_vh(L);
  double dmu = musign * twisted_mass / (4.0 + mass);
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx d[4][3], x[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, d);
    load_spinor(chi, s, x);
    for (int sp = 0; sp < 4; sp++) {
      double g5 = (sp < 2) ? 1.0 : -1.0;
      for (int c = 0; c < 3; c++)
        d[sp][c] = alpha * (1.0 + I * dmu * g5 * isign) * x[sp][c] - beta * d[sp][c];
    }
    store_spinor(res, s, d);
  }
}

/* include/qphix/tm_clov_dslash_body.h:339-357: full inverse picked by isign
   (flavour 0): isign = +1 -> finv0, isign = -1 -> finv1 */
void or_tmclov_dslash(const or_lattice *L, double *res, const double *psi,
                      const double *gauge, const double *finv0,
                      const double *finv1, int isign, int cb)
{
  long vh = or_vh(L);
  const double *f = (isign == 1) ? finv0 : finv1;
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx d[4][3], y[4][3];
    dslash_site(L, psi, gauge, isign, cb, s, d);
    fclov_site(f + s * 144, d, y);
    store_spinor(res, s, y);
  }
}

/* ---- even-odd operators ----------------------------------------------------- */

static const double *gauge_cb(const or_operator *op, int cb)
{
  (void)cb;
  return op->gauge; /* both checkerboards live in one array */
}

long or_op_len(const or_operator *op)
{
  return 24 * or_vh(&op->L) * ((op->kind == OR_OP_NDTM || op->kind == OR_OP_NDTMCLOVER) ? 2 : 1);
}

/* include/qphix/ndtm_reuse_operator.h:68-110 (EvenOddNDTMWilsonReuseOperator):
   t_f = D_{other,target} in_f (Wilson hop, both flavours);
   t' = mu_inv [(alpha - i isign mu g5 tau3) + eps tau1] t
        (two_flav_twisted_mass, include/qphix/complex_functors.h:467-541 with
         include/qphix/blas_utils.h:77-113; mu_inv = 1/(alpha^2 + mu^2 - eps^2));
   res_f = alpha (1 + i s_f isign (mu/alpha) g5) in_f - 0.25 D t'_f - eps in_{1-f},
   s_up = +1, s_dn = -1 (two_flav_AChiMinusBDPsi, include/qphix/tm_dslash_body.h:1174-1207) */
static void ndtm_apply(const or_operator *op, double *res, const double *in, int isign, int target_cb)
{
  const or_lattice *L = &op->L;
  long vh = or_vh(L), n1 = 24 * vh;
  int other = 1 - target_cb;
  double alpha = 4.0 + op->mass, mu = op->twisted_mass, eps = op->epsilon;
  double mu_inv = 1.0 / (alpha * alpha + mu * mu - eps * eps);
  double *t = (double *)malloc(sizeof(double) * 2 * n1);
  double *tp = (double *)malloc(sizeof(double) * 2 * n1);
  for (int f = 0; f < 2; f++) or_dslash(L, t + f * n1, in + f * n1, gauge_cb(op, other), isign, other);
  double a = alpha * mu_inv, b = -isign * mu * mu_inv, e = eps * mu_inv;
#pragma omp parallel for schedule(static)
  for (long s = 0; s < vh; s++) {
    cplx up[4][3], dn[4][3], ou[4][3], od[4][3];
    load_spinor(t, s, up);
    load_spinor(t + n1, s, dn);
    for (int sp = 0; sp < 4; sp++) {
      double g5 = (sp < 2) ? 1.0 : -1.0;
      for (int c = 0; c < 3; c++) {
        ou[sp][c] = (a + I * b * g5) * up[sp][c] + e * dn[sp][c];
        od[sp][c] = (a - I * b * g5) * dn[sp][c] + e * up[sp][c];
      }
    }
    store_spinor(tp, s, ou);
    store_spinor(tp + n1, s, od);
  }
  for (int f = 0; f < 2; f++) {
    or_tm_achimbdpsi(L, res + f * n1, tp + f * n1, in + f * n1, op->gauge, alpha, 0.25, op->mass, mu, isign,
                     target_cb, f == 0 ? 1.0 : -1.0);
    for (long i = 0; i < n1; i++) res[f * n1 + i] -= eps * in[(1 - f) * n1 + i];
  }
  free(t);
  free(tp);
}

/* include/qphix/ndtm_reuse_operator_clover.h:117-128 (EvenOddNDTMCloverReuseOperator):
   t_f = D_{other,target} in_f (Wilson hop, both flavours);
   two_flav_inverse_clover_term (tm_clov_dslash_body.h:1184-1204; per site
   codegen/dslash_common.cc:1198-1341):
     u_up = F_a t_up + C t_dn, u_dn = F_b t_dn + C t_up,
     (F_a, F_b) = (finv[0], finv[1]) for isign = +1, swapped for isign = -1;
   two_flav_AChiMinusBDPsi (tm_clov_dslash_body.h:1345-1365, flavour sign of
   rho :983): res_f = A in_f + i s_f rho isign g5 in_f - 0.25 D u_f - eps in_{1-f},
   rho = twisted_mass, s_up = +1, s_dn = -1 */
static void ndtmclov_apply(const or_operator *op, double *res, const double *in, int isign, int target_cb)
{
  const or_lattice *L = &op->L;
  long vh = or_vh(L), n1 = 24 * vh;
  int other = 1 - target_cb;
  double *t = (double *)malloc(sizeof(double) * 2 * n1);
  double *u = (double *)malloc(sizeof(double) * 2 * n1);
  double *c = (double *)malloc(sizeof(double) * n1);
  for (int f = 0; f < 2; f++) or_dslash(L, t + f * n1, in + f * n1, gauge_cb(op, other), isign, other);
  const double *fa = isign == 1 ? op->finv[0] : op->finv[1];
  const double *fb = isign == 1 ? op->finv[1] : op->finv[0];
  for (int f = 0; f < 2; f++) {
    or_fullclover_apply(vh, u + f * n1, t + f * n1, f == 0 ? fa : fb);
    or_clover_apply(vh, c, t + (1 - f) * n1, op->invclov);
    for (long i = 0; i < n1; i++) u[f * n1 + i] += c[i];
  }
  for (int f = 0; f < 2; f++) {
    or_clov_achimbdpsi(L, res + f * n1, u + f * n1, in + f * n1, op->gauge, op->clov, 0.25,
                       (f == 0 ? 1.0 : -1.0) * op->twisted_mass, isign, target_cb);
    for (long i = 0; i < n1; i++) res[f * n1 + i] -= op->epsilon * in[(1 - f) * n1 + i];
  }
  free(t);
  free(u);
  free(c);
}

void or_eo_apply(const or_operator *op, double *res, const double *in,
                 int isign, int target_cb)
{
  if (op->kind == OR_OP_NDTM) {
    ndtm_apply(op, res, in, isign, target_cb);
    return;
  }
  if (op->kind == OR_OP_NDTMCLOVER) {
    ndtmclov_apply(op, res, in, isign, target_cb);
    return;
  }
  const or_lattice *L = &op->L;
  long vh = or_vh(L);
  int other = 1 - target_cb;
  double *tmp = (double *)malloc(sizeof(double) * 24 * vh);
  switch (op->kind) {
  case OR_OP_WILSON: { /* include/qphix/wilson.h:49-65 */
    double alpha = 4.0 + op->mass;
    double beta = 0.25 / alpha;
    or_dslash(L, tmp, in, gauge_cb(op, other), isign, other);
    or_dslash_achimbdpsi(L, res, tmp, in, op->gauge, alpha, beta, isign,
                         target_cb);
    break;
  }
  case OR_OP_CLOVER: /* include/qphix/clover.h:162-172 */
    or_clov_dslash(L, tmp, in, op->gauge, op->invclov, isign, other);
    or_clov_achimbdpsi(L, res, tmp, in, op->gauge, op->clov, 0.25, op->rho,
                       isign, target_cb);
    break;
  case OR_OP_TM: { /* include/qphix/twisted_mass.h:62-77 */
    double alpha = 4.0 + op->mass;
    or_tm_dslash(L, tmp, in, op->gauge, op->mass, op->twisted_mass, isign,
                 other);
    or_tm_achimbdpsi(L, res, tmp, in, op->gauge, alpha, 0.25, op->mass,
                     op->twisted_mass, isign, target_cb, 1.0);
    break;
  }
  case OR_OP_TMCLOVER: /* include/qphix/twisted_mass_clover.h:92-102 */
    or_tmclov_dslash(L, tmp, in, op->gauge, op->finv[0], op->finv[1], isign,
                     other);
    or_clov_achimbdpsi(L, res, tmp, in, op->gauge, op->clov, 0.25, op->rho,
                       isign, target_cb);
    break;
  }
  free(tmp);
}

/* ---- BLAS --------------------------------------------------------------- */

double or_norm2(long n, const double *x)
{
  double s = 0;
  for (long i = 0; i < n; i++) s += x[i] * x[i];
  return s;
}

/* <x, y> = sum conj(x) y (include/qphix/complex_functors.h:11-64) */
void or_inner(long n, const double *x, const double *y, double out[2])
{
  double re = 0, im = 0;
  for (long i = 0; i < n; i += 2) {
    re += x[i] * y[i] + x[i + 1] * y[i + 1];
    im += x[i] * y[i + 1] - x[i + 1] * y[i];
  }
  out[0] = re;
  out[1] = im;
}

static inline void cdiv(double r[2], const double a[2], const double b[2])
{
  double d = b[0] * b[0] + b[1] * b[1];
  double re = (a[0] * b[0] + a[1] * b[1]) / d;
  double im = (a[1] * b[0] - a[0] * b[1]) / d;
  r[0] = re;
  r[1] = im;
}

static inline void cmul(double r[2], const double a[2], const double b[2])
{
  double re = a[0] * b[0] - a[1] * b[1];
  double im = a[0] * b[1] + a[1] * b[0];
  r[0] = re;
  r[1] = im;
}

/* ---- solvers ------------------------------------------------------------ */

/* CG on M^+M + shift (shift = 0: or_cg).  The shifted system is the one
   MInvCG solves per shift (include/qphix/minvcg.h:77); here it is solved on
   its own with the CG recurrence of include/qphix/invcg.h:281-417, the
   operator applications taking + shift * vector, d = |Mp|^2 + shift |p|^2. */
void or_cg_shift(const or_operator *op, double *x, const double *rhs, double shift, double rsd,
                 int max_iters, int isign, int cb, or_solve_info *info)
{
  long n = or_op_len(op);
  double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
  double *mp = malloc(sizeof(double) * n), *mmp = malloc(sizeof(double) * n);
  unsigned long mv = 0;
  double chi_sq = or_norm2(n, rhs);
  double rsd_sq = rsd * rsd * chi_sq;
  or_eo_apply(op, mp, x, isign, cb);
  or_eo_apply(op, mmp, mp, -isign, cb);
  mv += 2;
  if (shift != 0.0)
    for (long i = 0; i < n; i++) mmp[i] += shift * x[i];
  for (long i = 0; i < n; i++) r[i] = rhs[i] - mmp[i];
  double cp = or_norm2(n, r);
  info->status = 0;
  if (cp <= rsd_sq) {
    info->n_iters = 0;
    info->rsd_sq_final = cp;
    info->mv_apps = mv;
    goto done;
  }
  memcpy(p, r, sizeof(double) * n);
  for (int k = 0; k <= max_iters; ++k) {
    double c = cp;
    or_eo_apply(op, mp, p, isign, cb);
    or_eo_apply(op, mmp, mp, -isign, cb);
    mv += 2;
    double d = or_norm2(n, mp);
    if (shift != 0.0) {
      d += shift * or_norm2(n, p);
      for (long i = 0; i < n; i++) mmp[i] += shift * p[i];
    }
    double a = c / d;
    cp = 0;
    for (long i = 0; i < n; i++) {
      r[i] -= a * mmp[i];
      x[i] += a * p[i];
      cp += r[i] * r[i];
    }
    if (cp < rsd_sq) {
      info->n_iters = k;
      /* true residual; the reference's own recompute sits under an #ifdef
         that is never defined (include/qphix/invcg.h:342-403), so it counts
         no operator applications for it and leaves rsd_sq_final unset */
      or_eo_apply(op, mp, x, isign, cb);
      or_eo_apply(op, mmp, mp, -isign, cb);
      if (shift != 0.0)
        for (long i = 0; i < n; i++) mmp[i] += shift * x[i];
      for (long i = 0; i < n; i++) r[i] = rhs[i] - mmp[i];
      info->rsd_sq_final = or_norm2(n, r);
      info->mv_apps = mv;
      goto done;
    }
    double b = cp / c;
    for (long i = 0; i < n; i++) p[i] = r[i] + b * p[i];
  }
  info->n_iters = max_iters;
  info->rsd_sq_final = cp;
  info->mv_apps = mv;
  info->status = 1;
done:
  free(r); free(p); free(mp); free(mmp);
}

void or_cg(const or_operator *op, double *x, const double *rhs, double rsd,
           int max_iters, int isign, int cb, or_solve_info *info)
{
  or_cg_shift(op, x, rhs, 0.0, rsd, max_iters, isign, cb, info);
}

void or_bicgstab(const or_operator *op, double *x, const double *rhs,
                 double rsd, int max_iters, int isign, int cb,
                 or_solve_info *info)
{
  long n = or_op_len(op);
  double *r0 = malloc(sizeof(double) * n), *r = malloc(sizeof(double) * n);
  double *p = calloc(n, sizeof(double)), *v = calloc(n, sizeof(double));
  double *t = malloc(sizeof(double) * n);
  unsigned long mv = 0;
  double rhs_sq = or_norm2(n, rhs);
  double rsd_sq = rsd * rsd * rhs_sq;
  or_eo_apply(op, r0, x, isign, cb);
  mv++;
  for (long i = 0; i < n; i++) r0[i] = rhs[i] - r0[i];
  double r_norm = or_norm2(n, r0);
  info->status = 0;
  if (r_norm < rsd_sq) {
    info->rsd_sq_final = r_norm;
    info->n_iters = 0;
    info->mv_apps = mv;
    goto done;
  }
  memcpy(r, r0, sizeof(double) * n);
  double rho_prev[2] = {1, 0}, alpha[2] = {1, 0}, omega[2] = {1, 0};
  double rho[2] = {0, 0};
  int conv = 0, k;
  for (k = 1; k <= max_iters && !conv; k++) {
    or_inner(n, r0, r, rho);
    if (rho[0] == 0 && rho[1] == 0) {
      info->status = 2;
      info->rsd_sq_final = r_norm;
      info->n_iters = k;
      info->mv_apps = mv;
      goto done;
    }
    double t1[2], t2[2], beta[2];
    cdiv(t1, rho, rho_prev);
    cdiv(t2, alpha, omega);
    cmul(beta, t1, t2);
    /* p = r + beta (p - omega v) */
    for (long i = 0; i < n; i += 2) {
      double tr = p[i] - (omega[0] * v[i] - omega[1] * v[i + 1]);
      double ti = p[i + 1] - (omega[0] * v[i + 1] + omega[1] * v[i]);
      p[i] = r[i] + beta[0] * tr - beta[1] * ti;
      p[i + 1] = r[i + 1] + beta[0] * ti + beta[1] * tr;
    }
    or_eo_apply(op, v, p, isign, cb);
    mv++;
    double rv[2];
    or_inner(n, r0, v, rv);
    if (rv[0] == 0 && rv[1] == 0) {
      info->status = 2;
      info->rsd_sq_final = r_norm;
      info->n_iters = k;
      info->mv_apps = mv;
      goto done;
    }
    cdiv(alpha, rho, rv);
    rho_prev[0] = rho[0];
    rho_prev[1] = rho[1];
    /* s = r - alpha v (stored in r) */
    for (long i = 0; i < n; i += 2) {
      r[i] -= alpha[0] * v[i] - alpha[1] * v[i + 1];
      r[i + 1] -= alpha[0] * v[i + 1] + alpha[1] * v[i];
    }
    or_eo_apply(op, t, r, isign, cb);
    mv++;
    double t_norm = or_norm2(n, t);
    if (t_norm == 0) {
      info->status = 2;
      info->rsd_sq_final = r_norm;
      info->n_iters = k;
      info->mv_apps = mv;
      goto done;
    }
    or_inner(n, t, r, omega);
    omega[0] /= t_norm;
    omega[1] /= t_norm;
    /* x += omega r + alpha p; r -= omega t */
    r_norm = 0;
    for (long i = 0; i < n; i += 2) {
      x[i] += omega[0] * r[i] - omega[1] * r[i + 1] + alpha[0] * p[i] - alpha[1] * p[i + 1];
      x[i + 1] += omega[0] * r[i + 1] + omega[1] * r[i] + alpha[0] * p[i + 1] + alpha[1] * p[i];
      r[i] -= omega[0] * t[i] - omega[1] * t[i + 1];
      r[i + 1] -= omega[0] * t[i + 1] + omega[1] * t[i];
      r_norm += r[i] * r[i] + r[i + 1] * r[i + 1];
    }
    if (r_norm < rsd_sq) conv = 1;
  }
  /* the reference reports the loop counter after its final increment */
  info->rsd_sq_final = r_norm;
  info->n_iters = k;
  info->mv_apps = mv;
  info->status = conv ? 0 : 1;
done:
  free(r0); free(r); free(p); free(v); free(t);
}

void or_mr(const or_operator *op, double *x, const double *rhs, double rsd,
           int max_iters, double omega, int isign, int cb, or_solve_info *info)
{
  long n = or_op_len(op);
  double *r = malloc(sizeof(double) * n), *Mr = malloc(sizeof(double) * n);
  unsigned long mv = 0;
  int k = 0;
  info->status = 0;
  if (max_iters == 0) {
    info->n_iters = 0;
    info->rsd_sq_final = -1;
    info->mv_apps = 0;
    goto done;
  }
  or_eo_apply(op, r, x, isign, cb);
  mv++;
  for (long i = 0; i < n; i++) r[i] = rhs[i] - r[i];
  double norm_chi = or_norm2(n, rhs);
  double rsd_sq = rsd * rsd * norm_chi;
  double cp = or_norm2(n, r);
  if (cp < rsd_sq) {
    info->n_iters = 0;
    info->rsd_sq_final = cp / norm_chi;
    info->mv_apps = mv;
    goto done;
  }
  int cont = 1;
  while (cont) {
    ++k;
    or_eo_apply(op, Mr, r, isign, cb);
    mv++;
    double ip[2];
    or_inner(n, Mr, r, ip);
    double d = or_norm2(n, Mr);
    double a[2] = {omega * ip[0] / d, omega * ip[1] / d};
    for (long i = 0; i < n; i += 2) {
      x[i] += a[0] * r[i] - a[1] * r[i + 1];
      x[i + 1] += a[0] * r[i + 1] + a[1] * r[i];
      r[i] -= a[0] * Mr[i] - a[1] * Mr[i + 1];
      r[i + 1] -= a[0] * Mr[i + 1] + a[1] * Mr[i];
    }
    cp = or_norm2(n, r);
    cont = (k < max_iters) && (cp > rsd_sq);
  }
  info->n_iters = k;
  info->rsd_sq_final = cp / norm_chi;
  info->mv_apps = mv;
  info->status = (cp > rsd_sq) ? 1 : 0;
done:
  free(r); free(Mr);
}

void or_minvcg(const or_operator *op, double **x, const double *rhs,
               int n_shift, const double *shifts, const double *rsd,
               int max_iters, int isign, int cb, int *n_iters,
               double *rsd_sq_final, unsigned long *mv_apps)
{
  long n = or_op_len(op);
  double *r = malloc(sizeof(double) * n), *p0 = malloc(sizeof(double) * n);
  double *mp = malloc(sizeof(double) * n), *mmp = malloc(sizeof(double) * n);
  double **p = malloc(sizeof(double *) * n_shift);
  double *zeta = malloc(sizeof(double) * n_shift);
  double *zeta_prev = malloc(sizeof(double) * n_shift);
  double *beta = malloc(sizeof(double) * n_shift);
  double *rsd_sq = malloc(sizeof(double) * n_shift);
  int *convs = calloc(n_shift, sizeof(int));
  *mv_apps = 0;
  double cp = or_norm2(n, rhs);
  for (int s = 0; s < n_shift; s++) rsd_sq[s] = rsd[s] * rsd[s] * cp;
  memcpy(r, rhs, sizeof(double) * n);
  memcpy(p0, rhs, sizeof(double) * n);
  for (int s = 0; s < n_shift; s++) {
    p[s] = malloc(sizeof(double) * n);
    memcpy(p[s], rhs, sizeof(double) * n);
    rsd_sq_final[s] = 0;
  }
  or_eo_apply(op, mp, p0, isign, cb);
  or_eo_apply(op, mmp, mp, -isign, cb);
  *mv_apps += 2;
  double d = or_norm2(n, mp);
  double b = -cp / d;
  double c = 0;
  for (long i = 0; i < n; i++) {
    r[i] += b * mmp[i];
    c += r[i] * r[i];
  }
  for (int s = 0; s < n_shift; s++) {
    zeta_prev[s] = 1;
    zeta[s] = 1.0 / (1.0 - shifts[s] * b);
    beta[s] = b / (1.0 - shifts[s] * b);
    for (long i = 0; i < n; i++) x[s][i] = -beta[s] * rhs[i];
  }
  int conv = 0, k;
  *n_iters = 0;
  for (k = 1; k < max_iters && !conv; ++k) {
    double a = c / cp;
    for (long i = 0; i < n; i++) p0[i] = r[i] + a * p0[i];
    for (int s = 0; s < n_shift; s++)
      if (!convs[s]) {
        double as = a * zeta[s] * beta[s] / (zeta_prev[s] * b);
        for (long i = 0; i < n; i++) p[s][i] = zeta[s] * r[i] + as * p[s][i];
      }
    cp = c;
    double bp = b;
    or_eo_apply(op, mp, p0, isign, cb);
    or_eo_apply(op, mmp, mp, -isign, cb);
    *mv_apps += 2;
    d = or_norm2(n, mp);
    b = -cp / d;
    c = 0;
    for (long i = 0; i < n; i++) {
      r[i] += b * mmp[i];
      c += r[i] * r[i];
    }
    conv = 1;
    for (int s = 0; s < n_shift; s++) {
      if (!convs[s]) {
        double z0 = zeta[s], z1 = zeta_prev[s];
        zeta_prev[s] = z0;
        zeta[s] = z0 * z1 * bp;
        zeta[s] /= (b * a * (z1 - z0) + z1 * bp * (1.0 - shifts[s] * b));
        beta[s] = b * zeta[s] / z0;
        for (long i = 0; i < n; i++) x[s][i] -= beta[s] * p[s][i];
        double css = c * zeta[s] * zeta[s];
        convs[s] = (css < rsd_sq[s]);
        if (convs[s]) rsd_sq_final[s] = css;
      }
      conv &= convs[s];
    }
    *n_iters = k;
  }
  for (int s = 0; s < n_shift; s++) free(p[s]);
  free(p); free(r); free(p0); free(mp); free(mmp); free(zeta); free(zeta_prev);
  free(beta); free(rsd_sq); free(convs);
}

void or_richardson_bicgstab(const or_operator *op, double *x,
                            const double *rhs, double rsd, double delta,
                            int max_iters, int inner_max_iters, int isign,
                            int cb, or_solve_info *info)
{
  long n = or_op_len(op);
  double *r = malloc(sizeof(double) * n), *tmp = malloc(sizeof(double) * n);
  double *rin = malloc(sizeof(double) * n), *dx = malloc(sizeof(double) * n);
  unsigned long mv = 0;
  double rhs_sq = or_norm2(n, rhs);
  double rsd_t = rsd * rsd * rhs_sq;
  or_eo_apply(op, tmp, x, isign, cb);
  mv++;
  double r_norm_sq = 0;
  for (long i = 0; i < n; i++) {
    r[i] = rhs[i] - tmp[i];
    r_norm_sq += r[i] * r[i];
  }
  info->status = 0;
  if (r_norm_sq < rsd_t) {
    info->n_iters = 0;
    info->rsd_sq_final = r_norm_sq;
    info->mv_apps = mv;
    goto done;
  }
  int iter;
  for (iter = 1; iter < max_iters; iter++) {
    double delta_finish = sqrt(rsd_t / r_norm_sq);
    double delta_use = delta_finish > delta ? delta_finish : delta;
    double r_norm = sqrt(r_norm_sq);
    for (long i = 0; i < n; i++) {
      rin[i] = r[i] / r_norm;
      dx[i] = 0;
    }
    or_solve_info ii;
    or_bicgstab(op, dx, rin, delta_use, inner_max_iters, isign, cb, &ii);
    mv += ii.mv_apps;
    for (long i = 0; i < n; i++) dx[i] *= r_norm;
    or_eo_apply(op, tmp, dx, isign, cb);
    mv++;
    r_norm_sq = 0;
    for (long i = 0; i < n; i++) {
      x[i] += dx[i];
      r[i] -= tmp[i];
      r_norm_sq += r[i] * r[i];
    }
    if (r_norm_sq < rsd_t) {
      or_eo_apply(op, tmp, x, isign, cb);
      mv++;
      r_norm_sq = 0;
      for (long i = 0; i < n; i++) {
        r[i] = rhs[i] - tmp[i];
        r_norm_sq += r[i] * r[i];
      }
      info->rsd_sq_final = r_norm_sq / rhs_sq;
      info->n_iters = iter;
      info->mv_apps = mv;
      goto done;
    }
  }
  or_eo_apply(op, tmp, x, isign, cb);
  mv++;
  r_norm_sq = 0;
  for (long i = 0; i < n; i++) {
    r[i] = rhs[i] - tmp[i];
    r_norm_sq += r[i] * r[i];
  }
  info->rsd_sq_final = r_norm_sq / rhs_sq;
  info->n_iters = iter;
  info->mv_apps = mv;
  info->status = 1;
done:
  free(r); free(tmp); free(rin); free(dx);
}
