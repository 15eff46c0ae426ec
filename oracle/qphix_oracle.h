/*
 * CPU oracle for the QPhiX hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C FP64 restatement of QPhiX's Wilson / clover / twisted-mass Dslash,
 * the even-odd preconditioned operators built from them, the BLAS the solvers
 * use, and the CG / BiCGStab / MR / multishift-CG / Richardson solvers.  It is
 * the checker the GPU path is compared against; nothing in the product links
 * it.  Only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark load it.
 *
 * Parity pin: the Dslash / achimbdpsi / clover / twisted-mass / EO-operator
 * restatements are checked against the reference's own CPU kernels, compiled
 * from the reference sources by oracle/ref/Makefile into oracle/_ref/ and
 * driven on identical inputs (tests/test_oracle_pin.py, golden vectors in
 * tests/golden/).  The solver recurrences follow the reference files cited
 * per function and are checked by true-residual and iteration-count tests.
 *
 * Canonical (site-major) layouts used by every function here:
 *   cb-site index   s = ((t*Nz + z)*Ny + y)*Nxh + xh,  x = 2*xh + ((y+z+t+cb)&1)
 *                   (include/qphix/qdp_packer_parscalar.h:80-90, dslash_body.h:557)
 *   spinor  (cb)    double[Vh][4 spin][3 colour][2 re/im]
 *   gauge           double[2 cb][4 mu][Vh][3 row][3 col][2]   U_mu(x), x in cb
 *   clover (packed) double[Vh][2 block][36]: diag[6] then offd[15][re,im];
 *                   block b acts on spins (2b, 2b+1), index i = 3*s2 + colour,
 *                   A[i][j] = offd[i(i-1)/2 + j] for i > j, A[j][i] = conj(A[i][j])
 *                   (include/qphix_codegen/decl_common.h:15-32,
 *                    codegen/dslash_common.cc:1346-1434)
 *   full clover     double[Vh][2 block][6][6][2], out_i = sum_j A[i][j] in_j
 *                   (decl_common.h:56-62, codegen/dslash_common.cc:1436-1480)
 */
#ifndef QPHIX_ORACLE_H
#define QPHIX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int dims[4];          /* Nx, Ny, Nz, Nt (Nx even)                      */
  double t_boundary;    /* +1 periodic, -1 antiperiodic in t             */
  double aniso_s;       /* spatial hop coefficient                      */
  double aniso_t;       /* temporal hop coefficient                     */
  int use_tbc[4];       /* twisted boundary phase per dimension          */
  double tbc[4][2];     /* the phase (re, im) applied to every hop in dim */
} or_lattice;

long or_vh(const or_lattice *L);

/* ---- Dslash family (include/qphix/dslash_def.h:35-58) ------------------ */
void or_dslash(const or_lattice *L, double *res, const double *psi,
               const double *gauge, int isign, int cb);
void or_dslash_achimbdpsi(const or_lattice *L, double *res, const double *psi,
                          const double *chi, const double *gauge, double alpha,
                          double beta, int isign, int cb);
void or_dslash_dir(const or_lattice *L, double *res, const double *psi,
                   const double *gauge, int cb, int dir);

/* ---- clover (include/qphix/clover_dslash_def.h:24-53) ----------------- */
void or_clover_apply(long vh, double *res, const double *in, const double *clov);
void or_fullclover_apply(long vh, double *res, const double *in,
                         const double *fclov);
void or_clov_dslash(const or_lattice *L, double *res, const double *psi,
                    const double *gauge, const double *invclov, int isign,
                    int cb);
void or_clov_achimbdpsi(const or_lattice *L, double *res, const double *psi,
                        const double *chi, const double *gauge,
                        const double *clov, double beta, double rho, int isign,
                        int cb);

/* ---- twisted mass (include/qphix/tm_dslash_def.h:23-49) ---------------- */
void or_tm_dslash(const or_lattice *L, double *res, const double *psi,
                  const double *gauge, double mass, double twisted_mass,
                  int isign, int cb);
void or_tm_achimbdpsi(const or_lattice *L, double *res, const double *psi,
                      const double *chi, const double *gauge, double alpha,
                      double beta, double mass, double twisted_mass, int isign,
                      int cb, double musign);

/* ---- twisted-mass clover (include/qphix/tm_clov_dslash_def.h:44-66) ---- */
void or_tmclov_dslash(const or_lattice *L, double *res, const double *psi,
                      const double *gauge, const double *finv0,
                      const double *finv1, int isign, int cb);

/* ---- even-odd operators ------------------------------------------------- */
/* OR_OP_NDTM: two-flavour (non-degenerate) twisted-mass Wilson, vectors
   [flavour up, down][Vh][24] (include/qphix/ndtm_reuse_operator.h)
   OR_OP_NDTMCLOVER: two-flavour twisted-mass clover
   (include/qphix/ndtm_reuse_operator_clover.h): clov = A (target cb),
   invclov = packed flavour-off-diagonal inverse, finv = full up / down
   flavour-diagonal inverses (other cb), twisted_mass = mu, epsilon */
enum { OR_OP_WILSON = 0, OR_OP_CLOVER = 1, OR_OP_TM = 2, OR_OP_TMCLOVER = 3, OR_OP_NDTM = 4,
       OR_OP_NDTMCLOVER = 5 };
typedef struct {
  int kind;
  or_lattice L;
  const double *gauge;      /* both checkerboards                        */
  const double *clov;       /* packed clover on the target cb (A_oo)     */
  const double *invclov;    /* packed A_ee^-1 (clover)                   */
  const double *finv[2];    /* full (A_ee +/- i mu g5)^-1 (tm clover)    */
  double mass;              /* Wilson bare mass (wilson, tm)             */
  double twisted_mass;      /* tm                                        */
  double rho;               /* prec_mass_rho (clover, tm clover)         */
  double epsilon;           /* flavour splitting (ndtm)                  */
} or_operator;

/* reals in one vector the operator acts on (24 Vh, twice that for ndtm) */
long or_op_len(const or_operator *op);

void or_eo_apply(const or_operator *op, double *res, const double *in,
                 int isign, int target_cb);

/* ---- BLAS (include/qphix/blas_new_c.h) --------------------------------- */
double or_norm2(long n, const double *x);
void or_inner(long n, const double *x, const double *y, double out[2]);

/* ---- solvers ------------------------------------------------------------ */
typedef struct {
  int n_iters;
  double rsd_sq_final;
  unsigned long mv_apps;
  int status;               /* 0 converged, 1 max iterations, 2 breakdown */
} or_solve_info;

/* include/qphix/invcg.h:88-456: CG on M^dag M (isign selects M^dag M/MM^dag) */
void or_cg(const or_operator *op, double *x, const double *rhs, double rsd,
           int max_iters, int isign, int cb, or_solve_info *info);
void or_cg_shift(const or_operator *op, double *x, const double *rhs, double shift, double rsd,
                 int max_iters, int isign, int cb, or_solve_info *info);
/* include/qphix/invbicgstab.h:80-263 */
void or_bicgstab(const or_operator *op, double *x, const double *rhs,
                 double rsd, int max_iters, int isign, int cb,
                 or_solve_info *info);
/* include/qphix/invmr.h:62-210 (terminate on residuum, relative) */
void or_mr(const or_operator *op, double *x, const double *rhs, double rsd,
           int max_iters, double omega, int isign, int cb,
           or_solve_info *info);
/* include/qphix/minvcg.h:77-387 */
void or_minvcg(const or_operator *op, double **x, const double *rhs,
               int n_shift, const double *shifts, const double *rsd,
               int max_iters, int isign, int cb, int *n_iters,
               double *rsd_sq_final, unsigned long *mv_apps);
/* include/qphix/inv_richardson_multiprec.h:42-239, inner solver BiCGStab
   run in FP64 with the relaxed tolerance delta */
void or_richardson_bicgstab(const or_operator *op, double *x,
                            const double *rhs, double rsd, double delta,
                            int max_iters, int inner_max_iters, int isign,
                            int cb, or_solve_info *info);

#ifdef __cplusplus
}
#endif
#endif
