/*
 * qphix_b200 -- C ABI of the B200 (sm_100a) implementation of QPhiX's hot
 * path: the Wilson / clover / twisted-mass (clover) Dslash, the even-odd
 * preconditioned operators and the CG / BiCGStab / MR / multishift-CG /
 * Richardson solvers.
 *
 * Plain C types only (opaque handles, pointers, sizes).  Every function
 * returns 0 on success or a negative QPHIX_GPU_E* code; the message of the
 * last failure on the calling thread is qphix_gpu_last_error().  Nothing in
 * the library calls abort() or exit().  QPhiX's own interfaces abort on
 * misuse (include/qphix/geometry.h:274-277, dslash_body.h:64-95,
 * minvcg.h:92-96); here the same conditions come back as error codes and the
 * C++ drop-in headers (include/qphix/) turn them into exceptions.
 *
 * Fields live in device memory in the library's own chunked layout; they are
 * filled from and read back into host arrays in either the canonical
 * site-major FP64 layout or QPhiX's blocked host layout (any veclen / soalen
 * / padding / compress12 / FT the reference supports).
 *
 * Each lattice carries one CUDA stream (its own non-blocking stream unless
 * the caller installs another); every call on objects of that lattice is
 * ordered on it.  A lattice stays alive until it and all of its fields have
 * been destroyed, in any order.  Objects are not
 * thread-safe: one host thread per lattice (QPhiX objects are likewise not
 * re-entrant, dslash_body.h:85-95).
 */
#ifndef QPHIX_B200_H
#define QPHIX_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define QPHIX_GPU_OK 0
#define QPHIX_GPU_EINVAL (-1)      /* bad argument / shape / combination     */
#define QPHIX_GPU_ENOMEM (-2)      /* device or pinned allocation failed     */
#define QPHIX_GPU_ECUDA (-3)       /* a CUDA runtime call failed             */
#define QPHIX_GPU_ENOTCONV (-4)    /* solver hit its iteration limit         */
#define QPHIX_GPU_EBREAKDOWN (-5)  /* solver breakdown (BiCGStab rho == 0 ...) */
#define QPHIX_GPU_EUNSUPPORTED (-6)

/* ---- enums ------------------------------------------------------------- */
/* Q16: spinors as 16-bit fixed point (q / 32767 of the site's largest |value|,
 * with that value stored per site); links and clover terms in FP16.
 * Q16F32: the same spinors with FP32 links and clover terms. */
enum { QPHIX_GPU_F64 = 0, QPHIX_GPU_F32 = 1, QPHIX_GPU_F16 = 2, QPHIX_GPU_BF16 = 3, QPHIX_GPU_Q16 = 4,
       QPHIX_GPU_Q16F32 = 5 };
enum { QPHIX_GPU_SPINOR = 0, QPHIX_GPU_GAUGE = 1, QPHIX_GPU_CLOVER = 2, QPHIX_GPU_FULLCLOVER = 3 };
/* QPHIX_GPU_NDTM: the two-flavour (non-degenerate) twisted-mass Wilson
 * operator (include/qphix/ndtm_reuse_operator.h:16-110, parameters mass,
 * twisted_mass = mu and epsilon).  Its fields hold flavour pairs: right-hand
 * side 2k is the up, 2k + 1 the down flavour.  As a Dslash kind it is the
 * Wilson hop followed by mu_inv [(alpha - i isign mu g5 tau3) + eps tau1];
 * solved with CG (flavour-coupled: the pair is one system).
 * QPHIX_GPU_NDTMCLOVER: the two-flavour twisted-mass clover operator
 * (include/qphix/ndtm_reuse_operator_clover.h:23-165; twisted_mass = mu,
 * epsilon), flavour pairs as for NDTM; its operator takes clov = A,
 * invclov = the packed flavour-off-diagonal inverse and finv0 / finv1 = the
 * full flavour-diagonal inverses (qphix_gpu_clover_invert_ndtm builds them). */
enum { QPHIX_GPU_WILSON = 0, QPHIX_GPU_CLOVER_OP = 1, QPHIX_GPU_TM = 2, QPHIX_GPU_TMCLOVER = 3,
       QPHIX_GPU_NDTM = 4, QPHIX_GPU_NDTMCLOVER = 5 };
enum { QPHIX_GPU_HOST_CANONICAL = 0, QPHIX_GPU_HOST_QPHIX = 1, QPHIX_GPU_HOST_QDP = 2 };
enum { QPHIX_GPU_HOST_F64 = 0, QPHIX_GPU_HOST_F32 = 1, QPHIX_GPU_HOST_F16 = 2 };
enum { QPHIX_GPU_SOLVER_CG = 0, QPHIX_GPU_SOLVER_BICGSTAB = 1, QPHIX_GPU_SOLVER_MR = 2 };

typedef struct qphix_gpu_lattice_s *qphix_gpu_lattice;
typedef struct qphix_gpu_field_s *qphix_gpu_field;
typedef struct qphix_gpu_eo_op_s *qphix_gpu_eo_op;

/* Host array layout for upload / download.
 * canonical: FP64 site-major (ft must be QPHIX_GPU_HOST_F64):
 *   spinor [nrhs][Vh][4 spin][3 col][2], gauge [2 cb][4 mu][Vh][3][3][2]
 *   (U_mu(x), x in cb), clover [Vh][2][36] (diag[6], offd[15] re/im),
 *   full clover [Vh][2][6][6][2].
 * qphix: the reference's Geometry<FT,V,S,compress12> arrays with padding
 *   pad_xy / pad_xyz (include/qphix/geometry.h:130-175); spinor pointers are
 *   the ones allocCBFourSpinor returns (block 0 = first site), gauge arrays
 *   are one checkerboard each (8 links per site, stored transposed).
 * qdp: QDP++ / Chroma full-lattice arrays in QDP++'s checkerboarded (CB2)
 *   site order, the order the reference's packers read
 *   (include/qphix/qdp_packer_parscalar.h:51-129,150-230): site
 *   cb * Vh + (x/2 + Nx/2 (y + Ny (z + Nz t))); FP64 or FP32.
 *   spinor [nrhs][V][4 spin][3 col][2] (LatticeFermion), gauge
 *   [4 mu][V][3][3][2] (multi1d<LatticeColorMatrix> u, row-major U_mu(x),
 *   the four directions contiguous), clover [V][72] (Chroma's
 *   PrimitiveClovTriang: diag[2][6], then offd[2][15][2]).  Spinor and
 *   clover transfers touch only checkerboard `cb` of the array (the rest is
 *   neither read nor written); gauge uploads take both checkerboards. */
typedef struct {
  int kind;        /* QPHIX_GPU_HOST_CANONICAL / _QPHIX / _QDP          */
  int ft;          /* QPHIX_GPU_HOST_F64 / _F32 / _F16                  */
  int veclen;      /* qphix only                                         */
  int soalen;
  int compress12;
  int pad_xy;
  int pad_xyz;
  int cb;          /* qdp only: the checkerboard a spinor / clover
                      transfer reads or writes (0 even, 1 odd)            */
} qphix_gpu_host_layout;

/* Operator parameters: the constructor arguments of Dslash / ClovDslash /
 * TMDslash / TMClovDslash and the EvenOdd*Operator classes. */
typedef struct {
  int kind;                 /* QPHIX_GPU_WILSON ... _TMCLOVER                 */
  double t_boundary;        /* +1 / -1                                       */
  double aniso_s, aniso_t;  /* hop coefficients                              */
  int use_tbc[4];           /* twisted boundary phase per dimension          */
  double tbc_phases[4][2];
  double mass;              /* Wilson / TM bare mass (alpha = 4 + mass)      */
  double twisted_mass;      /* TM mu                                         */
  double prec_mass_rho;     /* clover / TM clover i rho gamma_5 term         */
  double epsilon;           /* two-flavour twisted mass: flavour splitting   */
} qphix_gpu_op_params;

typedef struct {
  int n_iters;              /* as the reference solver reports it            */
  double rsd_sq_final;      /* as the reference solver reports it            */
  unsigned long site_flops; /* reference flop accounting                     */
  unsigned long mv_apps;    /* operator applications                         */
  int status;               /* 0 converged, 1 iteration limit, 2 breakdown   */
  double true_rel_resid;    /* ||b - M x|| / ||b|| recomputed in FP64        */
  double seconds;           /* device time of the solve                      */
} qphix_gpu_solve_info;

/* ---- library ------------------------------------------------------------ */
int qphix_gpu_version(void);
const char *qphix_gpu_last_error(void);
/* Select the CUDA device for the calling thread. */
int qphix_gpu_init(int device);
/* Number of kernels this library has launched in this process; a CUDA-graph
 * replay counts every kernel node it runs. */
int qphix_gpu_launch_count(unsigned long long *out);

/* ---- Dslash launch-shape autotuner (no reference counterpart: QPhiX picks
 * its blocking by hand, Geometry(..., By, Bz, NCores, Sy, Sz, ...),
 * include/qphix/geometry.h:130).  Each Dslash configuration (precision,
 * links, epilogue, lattice, nrhs) is timed over its built shapes (right-hand
 * sides per thread, lattice sites per thread) the first time it runs
 * outside CUDA-graph capture; the fastest shape is kept for the process.
 * Entries are listed in key order.  sites_per_thread = 0 (with rhs_tile = 2)
 * denotes the shape that keeps two right-hand sides of one site in the
 * float2 lanes of a thread. */
int qphix_gpu_tune_enable(int enable);
int qphix_gpu_tune_entries(int *count);
int qphix_gpu_tune_entry(int index, char *key, size_t key_len, int *rhs_tile, int *sites_per_thread,
                         double *launch_us);

/* ---- lattice (replaces Geometry<FT,V,S,c12>, include/qphix/geometry.h:130) */
int qphix_gpu_lattice_create(const int latt_size[4], qphix_gpu_lattice *out);
int qphix_gpu_lattice_destroy(qphix_gpu_lattice lat);
int qphix_gpu_lattice_set_stream(qphix_gpu_lattice lat, void *cuda_stream);
int qphix_gpu_lattice_sync(qphix_gpu_lattice lat);
long qphix_gpu_lattice_volcb(qphix_gpu_lattice lat);

/* ---- fields (replace Geometry::allocCB* / free, geometry.h:270-396) ---- */
/* recon: 12 or 18 for gauge fields, ignored otherwise.  nrhs >= 1 for
 * spinors (a block of right-hand sides), 1 otherwise.  Zero-filled. */
int qphix_gpu_field_create(qphix_gpu_lattice lat, int kind, int prec, int recon, int nrhs,
                           qphix_gpu_field *out);
int qphix_gpu_field_destroy(qphix_gpu_field f);
int qphix_gpu_field_bytes(qphix_gpu_field f, size_t *bytes);
/* cb: canonical gauge arrays carry both checkerboards (pass -1).  A qphix
 * gauge array belongs to one checkerboard and holds 8 links per site:
 * pass 0 / 1 to take the forward links U_mu(x) of that checkerboard (upload
 * both arrays to fill the field), or 2 / 3 to fill the whole field from the
 * one array of checkerboard cb - 2 (its back links U_mu(x - mu) supply the
 * other checkerboard's forward links) -- what Dslash::dslash(.., u[cb], cb)
 * needs.
 * rhs: index of one right-hand side to transfer, or -1 for all. */
int qphix_gpu_field_upload(qphix_gpu_field f, const void *host, const qphix_gpu_host_layout *layout,
                           int cb, int rhs);
int qphix_gpu_field_download(qphix_gpu_field f, void *host, const qphix_gpu_host_layout *layout, int rhs);
/* Device-to-device copy with precision conversion: dst = scale * src. */
int qphix_gpu_field_convert(qphix_gpu_field dst, qphix_gpu_field src, double scale);

/* ---- Dslash family --------------------------------------------------------
 * qphix_gpu_dslash replaces Dslash::dslash (include/qphix/dslash_def.h:35),
 *   ClovDslash::dslash (clover_dslash_def.h:34, aux = A^-1),
 *   TMDslash::dslash (tm_dslash_def.h:33) and TMClovDslash::dslash
 *   (tm_clov_dslash_def.h:44, aux = invclov[0], aux2 = invclov[1]).
 * qphix_gpu_dslash_achimbdpsi replaces the dslashAChiMinusBDPsi members
 *   (dslash_def.h:42, clover_dslash_def.h:41, tm_dslash_def.h:39,
 *   tm_clov_dslash_def.h:57; aux = the clover term A for clover kinds).
 *   For Wilson res = alpha chi - beta D psi; clover kinds
 *   res = A chi + i rho isign g5 chi - beta D psi (alpha ignored);
 *   TM res = alpha (1 + i isign musign mu/(4+m) g5) chi - beta D psi.
 * qphix_gpu_dslash_dir replaces Dslash::dslashDir (dslash_def.h:51).
 * qphix_gpu_clover_apply replaces ClovDslash::clovMult (clover_dslash_def.h:50). */
int qphix_gpu_dslash(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                     qphix_gpu_field gauge, qphix_gpu_field aux, qphix_gpu_field aux2, int isign, int cb);
int qphix_gpu_dslash_achimbdpsi(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                qphix_gpu_field chi, qphix_gpu_field gauge, qphix_gpu_field aux, double alpha,
                                double beta, int isign, int cb, double musign);
int qphix_gpu_dslash_dir(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                         qphix_gpu_field gauge, int cb, int dir);
/* qphix_gpu_dslash_achimbdpsi with the reductions the solvers fuse into its
 * epilogue (no counterpart in the reference, which calls norm2Spinor /
 * innerProduct of blas_new_c.h:278,520 on the result in separate passes):
 * per rhs r, in this order, out[nval r + 0] = |res_r|^2, then, when w is
 * given, <w_r, res_r> (re, im), then <res_r, chi_r> (re, im); nval = 3, or 5
 * with w.  Inner products are sum conj(first) second.  out == NULL leaves
 * the values in the lattice's device result buffer (no host round trip). */
int qphix_gpu_dslash_achimbdpsi_norms(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                      qphix_gpu_field chi, qphix_gpu_field gauge, qphix_gpu_field aux,
                                      double alpha, double beta, int isign, int cb, double musign, qphix_gpu_field w,
                                      double *out);
/* Two-flavour twisted-mass clover hop: the Wilson hop of both flavours of
 * each (up, down) pair followed by the two-flavour inverse clover term --
 * Dslash::dslash then TMClovDslash::two_flav_inverse_clover_term
 * (tm_clov_dslash_def.h:96-110, ndtm_reuse_operator_clover.h:121-126), one
 * kernel.  finv_up / finv_dn are used as given for isign = +1 and swapped for
 * isign = -1.  The second half of that operator is
 * qphix_gpu_dslash_achimbdpsi with kind QPHIX_GPU_NDTMCLOVER, aux = A and
 * rho = twisted_mass (two_flav_AChiMinusBDPsi, tm_clov_dslash_def.h:84-92). */
int qphix_gpu_dslash_two_flav_clover(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                     qphix_gpu_field gauge, qphix_gpu_field finv_up, qphix_gpu_field finv_dn,
                                     qphix_gpu_field clov_odiag, int isign, int cb);
int qphix_gpu_clover_apply(qphix_gpu_field res, qphix_gpu_field chi, qphix_gpu_field clov);

/* ---- multi-GPU halo mode: a lattice cut into slabs along t --------------------
 * (replaces the face packing and exchange of include/qphix/comm.h / face.h for
 * a t decomposition).  Each rank's lattice is one slab (global t offset even,
 * so local and global checkerboards agree).  A Dslash on a slab needs, from
 * its neighbours, the source field's first (next slab) and last (previous
 * slab) time slices and, once per gauge field, U_t on the previous slab's last
 * slice.  qphix_gpu_halo_pack_* copy those faces into caller-owned device
 * buffers; the caller moves them between ranks (NCCL send / recv, or device
 * copies when the slabs share a GPU) and passes the received buffers to the
 * *_halo Dslash entry points, which take every other hop from the slab.  The
 * t boundary condition applies on the slabs holding the global edges.
 * side 0 = first slice (sent to the previous slab), 1 = last slice (sent to
 * the next slab).  The packs are asynchronous on the field's lattice stream
 * (synchronise it before another stream or rank reads the buffer); dst must
 * hold qphix_gpu_halo_spinor_bytes / _link_bytes. */
typedef struct {
  const void *psi_fwd;    /* the next slab's side-0 pack of the hopped field   */
  const void *psi_bwd;    /* the previous slab's side-1 pack of it             */
  const void *links_bwd;  /* the previous slab's qphix_gpu_halo_pack_links      */
  int global_first;       /* this slab holds global t = 0                       */
  int global_last;        /* this slab holds global t = Nt - 1                  */
} qphix_gpu_halo_faces;
int qphix_gpu_halo_spinor_bytes(qphix_gpu_field psi, size_t *bytes);
int qphix_gpu_halo_pack_spinor(qphix_gpu_field psi, int side, void *dst);
int qphix_gpu_halo_link_bytes(qphix_gpu_field gauge, size_t *bytes);
int qphix_gpu_halo_pack_links(qphix_gpu_field gauge, void *dst);
int qphix_gpu_dslash_halo(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                          qphix_gpu_field gauge, qphix_gpu_field aux, qphix_gpu_field aux2, int isign, int cb,
                          const qphix_gpu_halo_faces *faces);
int qphix_gpu_dslash_achimbdpsi_halo(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                     qphix_gpu_field chi, qphix_gpu_field gauge, qphix_gpu_field aux, double alpha,
                                     double beta, int isign, int cb, double musign,
                                     const qphix_gpu_halo_faces *faces);

/* ---- halo mode for a lattice cut along any of x, y, z, t ---------------------
 * (the 4D decomposition of include/qphix/comm.h:372-437 and geometry's
 * per-direction comms flags).  Each rank's lattice is one block of a
 * Cartesian grid of blocks; every local extent is even (so local and global
 * checkerboards agree).  For each cut direction mu the Dslash needs the
 * source field's first slice along mu from the next block, its last slice
 * from the previous block, and, once per gauge field, U_mu on the previous
 * block's last slice; hops along uncut directions wrap inside the block.
 * A face lists the sites of one checkerboard of a slice, ordered
 * x: ((t Nz + z) Ny + y) / 2, y: (t Nz + z) Nx/2 + x/2,
 * z: (t Ny + y) Nx/2 + x/2, t: (z Ny + y) Nx/2 + x/2 (local coordinates).
 * qphix_gpu_halo_pack_spinor_dir packs the field's slice (side 0 first, 1
 * last) of checkerboard cb (the checkerboard the field lives on, the
 * opposite of the Dslash's target); qphix_gpu_halo_pack_links_dir packs U_mu
 * on the last slice, both checkerboards.  Packs are asynchronous on the
 * field's lattice stream; dst must hold the *_bytes_dir sizes.  A t cut
 * applies t_boundary on the blocks that hold the global t edges; without one
 * the block holds both edges. */
typedef struct {
  int cut;                  /* bit mu (0 x, 1 y, 2 z, 3 t): the lattice is cut along mu     */
  const void *psi_fwd[4];   /* cut mu: the next block's side-0 pack of the hopped field      */
  const void *psi_bwd[4];   /* cut mu: the previous block's side-1 pack of it                */
  const void *links_bwd[4]; /* cut mu: the previous block's qphix_gpu_halo_pack_links_dir    */
  int global_first_t;       /* t cut: this block holds global t = 0                          */
  int global_last_t;        /* t cut: this block holds global t = Nt - 1                     */
} qphix_gpu_halo_faces4;
int qphix_gpu_halo_face_sites(qphix_gpu_lattice lat, int mu, size_t *sites);
int qphix_gpu_halo_spinor_bytes_dir(qphix_gpu_field psi, int mu, size_t *bytes);
int qphix_gpu_halo_pack_spinor_dir(qphix_gpu_field psi, int mu, int side, int cb, void *dst);
int qphix_gpu_halo_link_bytes_dir(qphix_gpu_field gauge, int mu, size_t *bytes);
int qphix_gpu_halo_pack_links_dir(qphix_gpu_field gauge, int mu, void *dst);
int qphix_gpu_dslash_halo4(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                           qphix_gpu_field gauge, qphix_gpu_field aux, qphix_gpu_field aux2, int isign, int cb,
                           const qphix_gpu_halo_faces4 *faces);
int qphix_gpu_dslash_achimbdpsi_halo4(const qphix_gpu_op_params *p, qphix_gpu_field res, qphix_gpu_field psi,
                                      qphix_gpu_field chi, qphix_gpu_field gauge, qphix_gpu_field aux,
                                      double alpha, double beta, int isign, int cb, double musign,
                                      const qphix_gpu_halo_faces4 *faces);

/* ---- clover term on the device ----------------------------------------------
 * QPhiX takes the clover term and its inverse from its caller (Chroma's
 * QDPCloverTerm); these build them on the GPU from a resident FP64 gauge field:
 *   qphix_gpu_clover_build   A on checkerboard cb: diag_mass + sigma.F with the
 *     clover-leaf field strength (tests/mesfield.cc:25-64) and the packing /
 *     coefficient convention of tests/clover_term_qdp_w.h:114-200,325-442
 *     (isotropic Wilson-clover: diag_mass = 4 + m, csw_r = csw_t = c_sw)
 *   qphix_gpu_clover_invert  packed A^-1
 *   qphix_gpu_clover_invert_twisted  full (A + i mu g5)^-1, (A - i mu g5)^-1
 *   qphix_gpu_clover_convert precision change of a clover / full clover field */
int qphix_gpu_clover_build(qphix_gpu_field clov, qphix_gpu_field gauge, int cb, double diag_mass, double csw_r,
                           double csw_t);
int qphix_gpu_clover_invert(qphix_gpu_field dst, qphix_gpu_field src);
int qphix_gpu_clover_invert_twisted(qphix_gpu_field dst_plus, qphix_gpu_field dst_minus, qphix_gpu_field src,
                                    double mu);
/* The inverse of the two-flavour diagonal block [[A + i mu g5, -eps],
 * [-eps, A - i mu g5]] of checkerboard A: finv_up = Q (A - i mu g5), finv_dn =
 * Q (A + i mu g5) (full clover fields) and clov_odiag = eps Q (clover field),
 * Q = (A^2 + mu^2 - eps^2)^-1 -- the invclov[2] and invclov_odiag arguments of
 * EvenOddNDTMCloverReuseOperator (ndtm_reuse_operator_clover.h:38-50). */
int qphix_gpu_clover_invert_ndtm(qphix_gpu_field finv_up, qphix_gpu_field finv_dn, qphix_gpu_field clov_odiag,
                                 qphix_gpu_field src, double mu, double eps);
/* The two-flavour inverse clover term alone (no hop) on (up, down) pairs:
 * res_up = Fa psi_up + C psi_dn, res_dn = Fb psi_dn + C psi_up with
 * (Fa, Fb) = (finv_up, finv_dn), swapped for isign = -1
 * (TMClovDslash::two_flav_inverse_clover_term, tm_clov_dslash_def.h:96-110). */
int qphix_gpu_two_flav_clover_apply(qphix_gpu_field res, qphix_gpu_field psi, qphix_gpu_field finv_up,
                                    qphix_gpu_field finv_dn, qphix_gpu_field clov_odiag, int isign);
int qphix_gpu_clover_convert(qphix_gpu_field dst, qphix_gpu_field src);

/* ---- even-odd operators ----------------------------------------------------
 * Replace EvenOddWilsonOperator (include/qphix/wilson.h:20), EvenOddClover-
 * Operator (clover.h:31), EvenOddTMWilsonOperator (twisted_mass.h:22) and
 * EvenOddTMCloverOperator (twisted_mass_clover.h:29).  clov = A on the
 * target (odd) checkerboard, invclov = A^-1 on the other (even) one;
 * finv0/finv1 = (A_ee + i mu g5)^-1 / (A_ee - i mu g5)^-1 for TM clover.
 * The operator holds non-owning references to the fields and owns one
 * temporary spinor per right-hand side count it has been applied to. */
int qphix_gpu_eo_op_create(const qphix_gpu_op_params *p, qphix_gpu_field gauge, qphix_gpu_field clov,
                           qphix_gpu_field invclov, qphix_gpu_field finv0, qphix_gpu_field finv1,
                           qphix_gpu_eo_op *out);
int qphix_gpu_eo_op_destroy(qphix_gpu_eo_op op);
/* operator()(res, in, isign, target_cb) (linearOp.h:21) */
int qphix_gpu_eo_op_apply(qphix_gpu_eo_op op, qphix_gpu_field res, qphix_gpu_field in, int isign,
                          int target_cb);

/* ---- solvers ----------------------------------------------------------------
 * x holds the initial guess and receives the solution; all right-hand sides
 * of the block are solved together (info[nrhs]).  rsd_target is relative
 * (ResiduumType RELATIVE, abs_solver.h:13).
 *   cg       InvCG::operator() on M^dag M (invcg.h:88)
 *   bicgstab InvBiCGStab::operator() (invbicgstab.h:80)
 *   mr       InvMR::operator() with over-relaxation omega (invmr.h:62)
 *   mshift   MInvCG::operator() (minvcg.h:77): x[n_shift] solve
 *            (M^dag M + shifts[i]) x_i = rhs
 *   richardson InvRichardsonMultiPrec::operator()
 *            (inv_richardson_multiprec.h:42): outer operator / fields in
 *            their precision, inner solver (CG / BiCGStab / MR) on
 *            op_inner, whose fields carry the inner precision. */
int qphix_gpu_solve_cg(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target,
                       int max_iters, int isign, int cb, qphix_gpu_solve_info *info);
int qphix_gpu_solve_bicgstab(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target,
                             int max_iters, int isign, int cb, qphix_gpu_solve_info *info);
int qphix_gpu_solve_mr(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target,
                       int max_iters, double omega, int isign, int cb, qphix_gpu_solve_info *info);
/* InvMRSmoother::operator() (invmr.h:302-354): exactly n_iters MR
 * iterations with over-relaxation omega, no residual test (rsd_sq_final is
 * reported as -1, like the reference). */
int qphix_gpu_solve_mr_smoother(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, int n_iters,
                                double omega, int isign, int cb, qphix_gpu_solve_info *info);
int qphix_gpu_solve_mshift_cg(qphix_gpu_eo_op op, qphix_gpu_field *x, qphix_gpu_field rhs, int n_shift,
                              const double *shifts, const double *rsd_target, int max_iters, int isign,
                              int cb, int *n_iters, double *rsd_sq_final, unsigned long *mv_apps);
/* BiCGStab with reliable updates.  No counterpart in the reference (its
 * mixed-precision solver is InvRichardsonMultiPrec, which restarts the inner
 * Krylov solve at every outer step).  The iteration runs on op_low (fields in
 * 16-bit or FP32 storage, FP32 arithmetic); whenever a right-hand side's
 * iterated residual has dropped by `delta` since its last update, the
 * low-precision solution increment is added to x (FP64) and r is replaced by
 * the true residual b - M x computed with op, without restarting the Krylov
 * space.  Convergence (rsd_target, relative) is decided on the true
 * residual.  info: n_iters = low-precision iterations, site_flops = number
 * of reliable updates, rsd_sq_final = |b - M x|^2. */
int qphix_gpu_solve_bicgstab_mixed(qphix_gpu_eo_op op, qphix_gpu_eo_op op_low, qphix_gpu_field x,
                                   qphix_gpu_field rhs, double rsd_target, double delta, int max_iters, int isign,
                                   int cb, qphix_gpu_solve_info *info);
int qphix_gpu_solve_richardson(qphix_gpu_eo_op op_outer, qphix_gpu_eo_op op_inner, int inner_solver,
                               qphix_gpu_field x, qphix_gpu_field rhs, double rsd_target, double delta,
                               int max_iters, int inner_max_iters, int isign, int cb,
                               qphix_gpu_solve_info *info);
/* CG on shifted normal equations, one shift per right-hand side: solves
 * (M^dag M + shifts[i]) x_i = rhs_i (shifts[i] >= 0) for every right-hand
 * side i of the block at once.  No counterpart in the reference; with all
 * shifts 0 it is qphix_gpu_solve_cg.  rsd_target[i] is relative, and
 * info[i].rsd_sq_final / true_rel_resid are the shifted system's true
 * residual. */
int qphix_gpu_solve_cg_shifted(qphix_gpu_eo_op op, qphix_gpu_field x, qphix_gpu_field rhs, const double *shifts,
                               const double *rsd_target, int max_iters, int isign, int cb,
                               qphix_gpu_solve_info *info);
/* Multishift CG with low-precision iterations (no counterpart in the
 * reference; the systems are MInvCG's, minvcg.h:77): one multishift CG on
 * op_low (FP32 or 16-bit storage) to rsd_low (nullptr: rsd_target), then
 * every shift refined side by side in the precision of op and x, by
 * low-precision shifted CG solves on the normalised true residuals, until
 * every shift meets rsd_target[i] by its true residual |rhs - (M^dag M +
 * shifts[i]) x_i| / |rhs|.  x: n_shift one-rhs fields in op's precision.
 * Outputs: multishift iterations, refinement iterations (summed over the
 * rounds, the slowest shift's count per round), refinement rounds, each
 * shift's final true relative residual squared, operator applications. */
int qphix_gpu_solve_mshift_cg_mixed(qphix_gpu_eo_op op, qphix_gpu_eo_op op_low, qphix_gpu_field *x,
                                    qphix_gpu_field rhs, int n_shift, const double *shifts,
                                    const double *rsd_target, const double *rsd_low, int max_iters, int isign,
                                    int cb, int *n_iters, int *refine_iters, int *corrections,
                                    double *rel_sq_final, unsigned long *mv_apps);

/* ---- BLAS (include/qphix/blas_new_c.h) --------------------------------------
 * Per right-hand side results are written to out[nrhs] (complex: out[2*nrhs]). */
int qphix_gpu_blas_norm2(qphix_gpu_field x, double *out);                        /* :278 */
int qphix_gpu_blas_inner_product(qphix_gpu_field x, qphix_gpu_field y, double *out); /* :520 */
int qphix_gpu_blas_caxpby(const double a[2], qphix_gpu_field x, const double b[2], qphix_gpu_field y);
                                                      /* y = a x + b y: axpy :214, axpby :247, aypx :139, caxpy :696 */
int qphix_gpu_blas_copy(qphix_gpu_field dst, qphix_gpu_field src);               /* :18  */
int qphix_gpu_blas_zero(qphix_gpu_field x);                                      /* :49  */
int qphix_gpu_blas_caxpby_norm2(const double a[2], qphix_gpu_field x, const double b[2], qphix_gpu_field y,
                                double *out);          /* y = a x + b y, |y|^2: axpyNorm2 :312 */
int qphix_gpu_blas_xmy_norm2(qphix_gpu_field x, qphix_gpu_field y, qphix_gpu_field z, double *out);
                                                      /* z = x - y, |z|^2: xmyNorm2Spinor :345, xmy2Norm2Spinor :360 */
int qphix_gpu_blas_inner_product_norm(qphix_gpu_field x, qphix_gpu_field y, double *out);
                                                      /* out[3 nrhs]: <x,y> re, im, |x|^2: innerProductNorm :573 */

/* ---- squared norms without allocation ---------------------------------------
 * No counterpart in the reference.  Same result as qphix_gpu_blas_norm2, for
 * callers that cannot let the library call cudaMalloc: host codes whose
 * device memory is owned by another allocator that has already reserved the
 * free HBM, or that must not add the device-wide synchronisation cudaMalloc /
 * cudaFree can cause inside a latency-sensitive loop.  Allocates nothing: the
 * per-block partial sums live in a fixed 512 KiB array in the library's
 * device memory (held by every GPU that loads the library until exit) and
 * the nrhs results are written to out_dev, a device buffer of nrhs doubles
 * owned by the caller, asynchronously on the lattice's stream (synchronise it
 * before reading).  Limit: ceil(volcb / 128) * nrhs <= 65536, else
 * QPHIX_GPU_EINVAL.  The field's device must be the current device, and
 * out_dev device (or managed) memory of it; a host pointer is rejected with
 * QPHIX_GPU_EINVAL before anything is launched.  The first call on a device
 * looks up the array's device address; make that first call before any
 * stream capture.  Under CUDA's lazy module loading (the default since CUDA
 * 12.2) that first call is also when the device reserves the 512 KiB, so make
 * it before the caller's allocator takes the free HBM (or set
 * CUDA_MODULE_LOADING=EAGER).  Every call shares the array, so calls whose
 * kernels overlap on the GPU race. */
int qphix_gpu_blas_norm2_noalloc(qphix_gpu_field x, double *out_dev);

/* ---- serving layer (no reference counterpart: the reference is a library
 * called one solve at a time; this is a request loop on top of it) --------
 * A server keeps gauge ensembles resident on the device (FP64 and low-
 * precision 12-real links) and runs up to `slots` requests at once, each on
 * its own worker thread, CUDA stream and device memory, so that requests of
 * different lattice sizes and operators overlap on the GPU.  Request memory
 * comes from one stream-ordered pool and is admitted against
 * `hbm_budget_bytes` (ensembles included): waiting requests are taken in
 * arrival order when a slot and the budget allow; one that does not fit may
 * be passed by later requests at most `max_bypass` times.  A request builds
 * its clover term on the device from the resident FP64 links and solves
 * M x = b on the odd checkerboard (target_cb = 1, isign = +1) with
 * qphix_gpu_solve_bicgstab_mixed (low-precision iterations, FP64 reliable
 * updates with threshold `delta`).  Its arithmetic is independent of the
 * other requests in flight (fixed-order reductions).
 * Host spinors use the canonical layout [nrhs][Vh][4][3][2] (FP64); rhs and
 * x must stay valid until qphix_gpu_server_wait returns. */
typedef struct qphix_gpu_server_s *qphix_gpu_server;

enum { QPHIX_GPU_SERVE_RELIABLE_UPDATE = 0, QPHIX_GPU_SERVE_RICHARDSON = 1 };
typedef struct {
  size_t hbm_budget_bytes;
  int slots;       /* requests in flight at once, 1 .. 64 */
  int low_prec;    /* QPHIX_GPU_F32 / _F16 / _BF16 / _Q16 / _Q16F32 */
  int max_bypass;
  double delta;    /* reliable-update threshold / residual reduction per correction, (0, 1) */
  int solver;      /* QPHIX_GPU_SERVE_RELIABLE_UPDATE (BiCGStab with reliable updates) or
                      QPHIX_GPU_SERVE_RICHARDSON (InvRichardsonMultiPrec, BiCGStab inner) */
} qphix_gpu_server_config;

typedef struct {
  int ensemble;          /* id from qphix_gpu_server_add_ensemble */
  int op_kind;           /* QPHIX_GPU_WILSON / _CLOVER_OP / _TM / _TMCLOVER */
  double mass;           /* bare mass, m = 1 / (2 kappa) - 4 */
  double csw;            /* clover coefficient (clover kinds) */
  double twisted_mass;   /* mu (twisted kinds; prec_mass_rho for TM clover) */
  double t_boundary;     /* +1 periodic, -1 antiperiodic in t */
  int nrhs;              /* 1 .. 32 */
  double rsd_target;     /* relative FP64 true residual */
  int max_iters;
  const double *rhs;
  double *x;
} qphix_gpu_request;

typedef struct {
  int status;              /* QPHIX_GPU_OK, _ENOTCONV, or the failing call's code */
  int n_iters;             /* max over the request's right-hand sides */
  unsigned long mv_apps;
  double true_rel_resid;   /* worst over the request's right-hand sides */
  double queue_s;          /* submit -> admission */
  double solve_s;          /* admission -> x written */
  double latency_s;        /* submit -> x written */
  size_t bytes;            /* device memory reserved for the request */
} qphix_gpu_request_result;

typedef struct {
  long long completed, failed, waiting, bypasses;
  int running, running_peak;
  size_t resident_bytes, reserved_bytes, reserved_peak_bytes, pool_used_peak_bytes;
} qphix_gpu_server_stats;

/* The server runs on the calling thread's current device. */
int qphix_gpu_server_create(const qphix_gpu_server_config *cfg, qphix_gpu_server *out);
/* gauge: canonical layout [2 cb][4 mu][Vh][3][3][2] (FP64) */
int qphix_gpu_server_add_ensemble(qphix_gpu_server s, const int dims[4], const double *gauge_canonical,
                                  int *ensemble_id);
int qphix_gpu_server_request_bytes(qphix_gpu_server s, const qphix_gpu_request *req, size_t *bytes);
int qphix_gpu_server_submit(qphix_gpu_server s, const qphix_gpu_request *req, long long *ticket);
int qphix_gpu_server_poll(qphix_gpu_server s, long long ticket, int *done);
/* Blocks until done; returns the request's status and forgets the ticket. */
int qphix_gpu_server_wait(qphix_gpu_server s, long long ticket, qphix_gpu_request_result *res);
int qphix_gpu_server_get_stats(qphix_gpu_server s, qphix_gpu_server_stats *stats);
/* Finishes admitted requests, drops waiting ones, frees everything. */
int qphix_gpu_server_destroy(qphix_gpu_server s);

#ifdef __cplusplus
}
#endif
#endif
