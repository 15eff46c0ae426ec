// The Wilson hopping term and every operator built around it, as one kernel
// template.  One thread owns one output site of the target checkerboard and a
// tile of R right-hand sides: each link is loaded (and, for 12-real storage,
// reconstructed) once and applied to all R spinors.  Neighbour indices and the
// periodic / antiperiodic / twisted boundary factors are computed in-kernel
// from the site coordinates, so there is no offset table and no face packing.
//
// Math follows the reference generator (codegen/dslash_common.cc):
//   projection tables :848-866, reconstruction :884-990, link multiply
//   :1916-1965 (U for forward hops, U^+ for backward hops), 12 -> 18
//   reconstruction :1895-1914, twisted boundary phases :1739-1772,
//   clover epilogue :1346-1434, full clover :1436-1480, twisted-mass
//   inverse :1482-1607, twisted-mass A chi :1612-1737, a chi - b D psi
//   :2089-2183, i rho gamma_5 prec-mass term :2128-2157.
// and the drivers' coefficient handling (include/qphix/dslash_body.h:484-512,
// 718-821): spatial hops x aniso_s, temporal hops x aniso_t, times t_boundary
// on the hop that crosses the global t edge.
#pragma once

#include "qpx_common.cuh"
#include "qpx_lanes.cuh"
#include "qpx_reduce.cuh"

// Register budget of the Dslash kernels, as the minimum resident 128-thread
// blocks per SM the compiler must allow for (registers per thread capped at
// 65536 / (128 x that)).  Measured on B200 (FP16 clover, 32^3x64 and
// 16^3x32 x 8 rhs): one site per thread with 16-bit storage runs best at 4
// blocks (at most 128 registers, which it fits without spilling; left free
// it takes 135 and drops to 3 blocks, 13 % slower at 32^3x64); FP32 / FP64
// storage, which sits at the HBM roofline with ~170-255 registers, keeps the
// compiler free (1); two sites or two right-hand sides per thread with at
// most 168 (3).
#ifndef QPX_MINB1
#define QPX_MINB1 1
#endif
#ifndef QPX_MINB1_16
#define QPX_MINB1_16 4
#endif
#ifndef QPX_MINB2
#define QPX_MINB2 3
#endif
#ifndef QPX_MINBR
#define QPX_MINBR 3
#endif
#define QPX_DSLASH_BOUNDS \
  __launch_bounds__(QPX_BLOCK, (SP == 2 ? QPX_MINB2 : (R == 2 ? QPX_MINBR : (P::has_norm ? QPX_MINB1_16 : QPX_MINB1))))

namespace qpx {

// EPI_NDTM / ACHI_NDTM: the two flavours of a non-degenerate twisted-mass
// doublet are right-hand sides 2k (up) and 2k + 1 (down) and are only built
// with two right-hand sides per thread (R = 2), so both flavours of a site
// sit in one thread:
//   EPI_NDTM:  out_up = (a + i b g5) acc_up + e acc_dn,
//              out_dn = (a - i b g5) acc_dn + e acc_up   (a = alpha, b = mu,
//              e = eps of the args; include/qphix/blas_utils.h:77-113)
//   ACHI_NDTM: out_f = alpha (1 + i s_f isign mu g5) chi_f - beta acc_f
//              - eps chi_{1-f}, s_up = +1, s_dn = -1
//              (include/qphix/tm_dslash_body.h:1174-1207)
// and the two-flavour twisted-mass clover operator
// (include/qphix/ndtm_reuse_operator_clover.h:117-128):
//   EPI_NDFCLOV: out_up = F_a acc_up + C acc_dn, out_dn = F_b acc_dn + C acc_up
//              with F_a, F_b the full flavour-diagonal inverses (clov, clov2;
//              the host swaps them for isign = -1) and C the packed
//              flavour-off-diagonal inverse (clov3)
//              (tm_clov_dslash_body.h:1184-1204, codegen/dslash_common.cc:
//               1198-1341)
//   ACHI_NDCLOV: out_f = A chi_f + i s_f isign rho g5 chi_f - beta acc_f
//              - eps chi_{1-f} (tm_clov_dslash_body.h:983,1345-1365)
enum Epi : int { EPI_NONE = 0, EPI_CLOV = 1, EPI_TMINV = 2, EPI_FCLOV = 3, EPI_NDTM = 4, EPI_NDFCLOV = 5 };
enum Achi : int { ACHI_NONE = 0, ACHI_ALPHA = 1, ACHI_CLOV = 2, ACHI_TM = 3, ACHI_NDTM = 4, ACHI_NDCLOV = 5 };
__host__ __device__ inline bool is_two_flavour(int epi, int achi)
{
  return epi == EPI_NDTM || epi == EPI_NDFCLOV || achi == ACHI_NDTM || achi == ACHI_NDCLOV;
}
enum Post : int {
  POST_STORE = 0,  // store out
  POST_CG = 1,     // r -= a out ; x += a p ; |r|^2   (a = state S_A[rhs]); out not stored
  POST_RAXPY = 2,  // r += b out ; |r|^2             (b = state S_B[rhs]); out not stored
};
// reduction value bits (values appear in this order)
enum RedBit : int {
  RED_NORM_OUT = 1,   // |out|^2                   (1 value,  slot 0)
  RED_DOT_W_OUT = 2,  // <w, out> = sum conj(w) out (2 values, slots 1-2)
  RED_DOT_OUT_CHI = 4,// <out, chi>                (2 values, slots 3-4)
  RED_NORM_R = 8,     // |r_new|^2 (POST_CG)        (1 value,  slot 5)
};

__host__ __device__ inline int red_nval(int mask)
{
  return ((mask & RED_NORM_OUT) ? 1 : 0) + ((mask & RED_DOT_W_OUT) ? 2 : 0) +
         ((mask & RED_DOT_OUT_CHI) ? 2 : 0) + ((mask & RED_NORM_R) ? 1 : 0);
}

__host__ __device__ inline int red_slots(int mask)
{
  return ((mask & RED_NORM_OUT) ? 0x1 : 0) | ((mask & RED_DOT_W_OUT) ? 0x6 : 0) |
         ((mask & RED_DOT_OUT_CHI) ? 0x18 : 0) | ((mask & RED_NORM_R) ? 0x20 : 0);
}

struct DslashArgs {
  Geom geom;
  int cb;           // target checkerboard
  int isign;        // +1: D, -1: D^dagger
  int nrhs;
  unsigned dir_mask;  // bit (2 mu + 1): forward hop, bit (2 mu): backward hop
  SpinorArg out, in, chi;
  GaugeArg gauge;
  CloverArg clov;
  CloverArg clov2, clov3;  // EPI_NDFCLOV: down-flavour full inverse, off-diagonal packed inverse
  double coeff_s;       // spatial hops (aniso_s, times the caller's beta)
  double coeff_t;       // temporal hops away from the t edges (aniso_t)
  double coeff_t_edge;  // temporal hops across the global t edge (aniso_t * t_boundary)
  int tbc_mask;
  double tbc[4][2];
  double alpha, beta;   // a chi - b D psi
  double mu, mu_inv;    // twisted mass
  double rho;           // i rho gamma_5 term
  double eps;           // flavour splitting of the two-flavour twisted mass
  int post;
  int g5_out;           // 1: the result times gamma_5 (see the post section of dslash_block)
  // halo mode (general path only): the lattice is one block of a lattice cut
  // along the directions whose bit is set in `halo`; a hop that leaves the
  // block along such a direction reads a ghost face instead of wrapping.
  // ghost_fwd[mu] = psi on the next block's first slice along mu,
  // ghost_bwd[mu] = psi on the previous block's last slice, ghost_link[mu] =
  // U_mu on that slice (the backward hop's link), indexed by the face site
  // (halo_face): x: ((t nz + z) ny + y) / 2, y: (t nz + z) nx/2 + x/2,
  // z: (t ny + y) nx/2 + x/2, t: (z ny + y) nx/2 + x/2.  The forward t edge
  // takes coeff_t_edge, the backward one coeff_t_bwd_edge (aniso_t, times
  // t_boundary where the edge is the global one).
  int halo;
  SpinorArg ghost_fwd[4], ghost_bwd[4];
  GaugeArg ghost_link[4];
  double coeff_t_bwd_edge;
  SpinorArg r, x, p, w; // extra vectors for POST_CG and RED_DOT_W_OUT
  ReduceArg red;
  SolverState *state;   // nullable; supplies the done flag and POST_CG's a
};

// --- spin projection (1 + SG gamma_mu) psi -> two colour vectors, SG = +-1 ---
template <int MU, int SG, typename T>
__device__ __forceinline__ void project(const T *psi, cx<T> h[2][3])
{
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cx<T> p0 = {psi[(0 * 3 + c) * 2], psi[(0 * 3 + c) * 2 + 1]};
    cx<T> p1 = {psi[(1 * 3 + c) * 2], psi[(1 * 3 + c) * 2 + 1]};
    cx<T> p2 = {psi[(2 * 3 + c) * 2], psi[(2 * 3 + c) * 2 + 1]};
    cx<T> p3 = {psi[(3 * 3 + c) * 2], psi[(3 * 3 + c) * 2 + 1]};
    if (MU == 0) {        // h0 = p0 + SG i p3, h1 = p1 + SG i p2
      h[0][c] = SG > 0 ? cx<T>{p0.re - p3.im, p0.im + p3.re} : cx<T>{p0.re + p3.im, p0.im - p3.re};
      h[1][c] = SG > 0 ? cx<T>{p1.re - p2.im, p1.im + p2.re} : cx<T>{p1.re + p2.im, p1.im - p2.re};
    } else if (MU == 1) { // h0 = p0 - SG p3, h1 = p1 + SG p2
      h[0][c] = SG > 0 ? p0 - p3 : p0 + p3;
      h[1][c] = SG > 0 ? p1 + p2 : p1 - p2;
    } else if (MU == 2) { // h0 = p0 + SG i p2, h1 = p1 - SG i p3
      h[0][c] = SG > 0 ? cx<T>{p0.re - p2.im, p0.im + p2.re} : cx<T>{p0.re + p2.im, p0.im - p2.re};
      h[1][c] = SG > 0 ? cx<T>{p1.re + p3.im, p1.im - p3.re} : cx<T>{p1.re - p3.im, p1.im + p3.re};
    } else {              // h0 = p0 + SG p2, h1 = p1 + SG p3
      h[0][c] = SG > 0 ? p0 + p2 : p0 - p2;
      h[1][c] = SG > 0 ? p1 + p3 : p1 - p3;
    }
  }
}

// The same projection on FP16 storage, one site per thread: the raw half2
// words (re, im of spin s, colour c in word 3 s + c) are combined in half
// precision -- i p = (-p.im, p.re) is a half swap -- and only the 12 results
// are widened to FP32, instead of the 24 inputs.  Each sum adds one FP16
// rounding to inputs that already carry the FP16 storage error.
template <int MU, int SG>
__device__ __forceinline__ void project_h2(const __half2 w[12], cx<float> h[2][3])
{
  const __half2 isg = __floats2half2_rn(-(float)SG, (float)SG);  // SG i p = swap(p) (-SG, SG)
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const __half2 p0 = w[c], p1 = w[3 + c], p2 = w[6 + c], p3 = w[9 + c];
    __half2 h0, h1;
    if (MU == 0) {  // h0 = p0 + SG i p3, h1 = p1 + SG i p2
      h0 = __hfma2(__lowhigh2highlow(p3), isg, p0);
      h1 = __hfma2(__lowhigh2highlow(p2), isg, p1);
    } else if (MU == 1) {  // h0 = p0 - SG p3, h1 = p1 + SG p2
      h0 = SG > 0 ? __hsub2(p0, p3) : __hadd2(p0, p3);
      h1 = SG > 0 ? __hadd2(p1, p2) : __hsub2(p1, p2);
    } else if (MU == 2) {  // h0 = p0 + SG i p2, h1 = p1 - SG i p3
      h0 = __hfma2(__lowhigh2highlow(p2), isg, p0);
      h1 = __hfma2(__lowhigh2highlow(p3), __hneg2(isg), p1);
    } else {  // h0 = p0 + SG p2, h1 = p1 + SG p3
      h0 = SG > 0 ? __hadd2(p0, p2) : __hsub2(p0, p2);
      h1 = SG > 0 ? __hadd2(p1, p3) : __hsub2(p1, p3);
    }
    const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
    h[0][c] = {f0.x, f0.y};
    h[1][c] = {f1.x, f1.y};
  }
}

// the FP16 one-site path's loads for project_h2: the 12 raw words and the norm
__device__ __forceinline__ void load_h2(const SpinorArg &f, int rhs, long long s, __half2 w[12], float &nrm)
{
  const uint4 *p = reinterpret_cast<const uint4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
  nrm = __ldg(f.norm + rhs * f.stride + s);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint4 d = __ldg(p + k * f.stride);
    w[4 * k] = *reinterpret_cast<const __half2 *>(&d.x);
    w[4 * k + 1] = *reinterpret_cast<const __half2 *>(&d.y);
    w[4 * k + 2] = *reinterpret_cast<const __half2 *>(&d.z);
    w[4 * k + 3] = *reinterpret_cast<const __half2 *>(&d.w);
  }
}

template <typename Lane>
struct HalfProjection {
  static constexpr bool value = false;
};
template <>
struct HalfProjection<Lanes<F16, 1>> {
  static constexpr bool value = true;
};

// the same for two right-hand sides in the lanes (RhsLanes<F16>): each rhs is
// projected on its raw half2 words and the 12 results widened into the lanes
template <int MU, int SG>
__device__ __forceinline__ void project_h2_pair(const SpinorArg &f, int rhs, long long s, cx<f2> h[2][3], f2 &nrm)
{
  __half2 wa[12], wb[12];
  float na, nb;
  load_h2(f, rhs, s, wa, na);
  load_h2(f, rhs + 1, s, wb, nb);
  cx<float> ha[2][3], hb[2][3];
  project_h2<MU, SG>(wa, ha);
  project_h2<MU, SG>(wb, hb);
#pragma unroll
  for (int sp = 0; sp < 2; sp++)
#pragma unroll
    for (int c = 0; c < 3; c++)
      h[sp][c] = {make_float2(ha[sp][c].re, hb[sp][c].re), make_float2(ha[sp][c].im, hb[sp][c].im)};
  nrm = make_float2(na, nb);
}

template <typename Lane>
struct RhsHalfProjection {
  static constexpr bool value = false;
};
template <>
struct RhsHalfProjection<RhsLanes<F16>> {
  static constexpr bool value = true;
};

// a per-rhs solver coefficient in the arithmetic type: the lanes of a
// two-rhs thread take right-hand sides rr and rr + 1
template <bool RL, typename T>
__device__ __forceinline__ T rhs_coef(const double *v, int rr)
{
  if constexpr (RL)
    return make_float2((float)v[rr], (float)v[rr + 1]);
  else
    return splat<T>(v[rr]);
}

// the per-lane parts of the fused reductions of a two-rhs thread: lane 0
// belongs to right-hand side rr, lane 1 to rr + 1
__device__ __forceinline__ void red_norm_pair(const f2 *x, double &n0, double &n1)
{
  f2 n = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 24; k++) n = mad(x[k], x[k], n);
  n0 = (double)n.x;
  n1 = (double)n.y;
}
__device__ __forceinline__ void red_dot_pair(const f2 *x, const f2 *y, double *re, double *im)
{
  f2 dre = make_float2(0.f, 0.f), dim = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 24; k += 2) {
    dre = mad(x[k], y[k], mad(x[k + 1], y[k + 1], dre));
    dim = mad(x[k], y[k + 1], mad(-x[k + 1], y[k], dim));
  }
  re[0] = (double)dre.x;
  re[1] = (double)dre.y;
  im[0] = (double)dim.x;
  im[1] = (double)dim.y;
}

// --- reconstruct-accumulate of (1 + SG gamma_mu) from chi = U h -------------
// QPX_ADD(k, v): acc[k] += SG v ; QPX_SUB(k, v): acc[k] -= SG v (signs
// resolved at compile time)
template <int MU, int SG, typename T>
__device__ __forceinline__ void recons_add(const cx<T> ch[2][3], T *acc)
{
#define QPX_ADD(k, v) (SG > 0 ? (acc[k] = acc[k] + (v)) : (acc[k] = acc[k] - (v)))
#define QPX_SUB(k, v) (SG > 0 ? (acc[k] = acc[k] - (v)) : (acc[k] = acc[k] + (v)))
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cx<T> c0 = ch[0][c], c1 = ch[1][c];
    acc[(0 * 3 + c) * 2] = acc[(0 * 3 + c) * 2] + c0.re;
    acc[(0 * 3 + c) * 2 + 1] = acc[(0 * 3 + c) * 2 + 1] + c0.im;
    acc[(1 * 3 + c) * 2] = acc[(1 * 3 + c) * 2] + c1.re;
    acc[(1 * 3 + c) * 2 + 1] = acc[(1 * 3 + c) * 2 + 1] + c1.im;
    if (MU == 0) {        // o2 += -SG i c1, o3 += -SG i c0
      QPX_ADD((2 * 3 + c) * 2, c1.im);
      QPX_SUB((2 * 3 + c) * 2 + 1, c1.re);
      QPX_ADD((3 * 3 + c) * 2, c0.im);
      QPX_SUB((3 * 3 + c) * 2 + 1, c0.re);
    } else if (MU == 1) { // o2 += SG c1, o3 += -SG c0
      QPX_ADD((2 * 3 + c) * 2, c1.re);
      QPX_ADD((2 * 3 + c) * 2 + 1, c1.im);
      QPX_SUB((3 * 3 + c) * 2, c0.re);
      QPX_SUB((3 * 3 + c) * 2 + 1, c0.im);
    } else if (MU == 2) { // o2 += -SG i c0, o3 += SG i c1
      QPX_ADD((2 * 3 + c) * 2, c0.im);
      QPX_SUB((2 * 3 + c) * 2 + 1, c0.re);
      QPX_SUB((3 * 3 + c) * 2, c1.im);
      QPX_ADD((3 * 3 + c) * 2 + 1, c1.re);
    } else {              // o2 += SG c0, o3 += SG c1
      QPX_ADD((2 * 3 + c) * 2, c0.re);
      QPX_ADD((2 * 3 + c) * 2 + 1, c0.im);
      QPX_ADD((3 * 3 + c) * 2, c1.re);
      QPX_ADD((3 * 3 + c) * 2 + 1, c1.im);
    }
  }
#undef QPX_ADD
#undef QPX_SUB
}

// the same with the hop's real coefficient c folded in: acc += c x (the
// reconstruction of ch), as fused multiply-adds (no separate scaling pass)
template <int MU, int SG, typename T>
__device__ __forceinline__ void recons_add_c(const cx<T> ch[2][3], T *acc, T c)
{
  const T cp = (SG > 0) ? c : -c;  // +SG c
  const T cn = -cp;                // -SG c
#define QPX_ADD(k, v) (acc[k] = mad(cp, (v), acc[k]))
#define QPX_SUB(k, v) (acc[k] = mad(cn, (v), acc[k]))
#pragma unroll
  for (int cc = 0; cc < 3; cc++) {
    cx<T> c0 = ch[0][cc], c1 = ch[1][cc];
    acc[(0 * 3 + cc) * 2] = mad(c, c0.re, acc[(0 * 3 + cc) * 2]);
    acc[(0 * 3 + cc) * 2 + 1] = mad(c, c0.im, acc[(0 * 3 + cc) * 2 + 1]);
    acc[(1 * 3 + cc) * 2] = mad(c, c1.re, acc[(1 * 3 + cc) * 2]);
    acc[(1 * 3 + cc) * 2 + 1] = mad(c, c1.im, acc[(1 * 3 + cc) * 2 + 1]);
    if (MU == 0) {        // o2 += -SG i c1, o3 += -SG i c0
      QPX_ADD((2 * 3 + cc) * 2, c1.im);
      QPX_SUB((2 * 3 + cc) * 2 + 1, c1.re);
      QPX_ADD((3 * 3 + cc) * 2, c0.im);
      QPX_SUB((3 * 3 + cc) * 2 + 1, c0.re);
    } else if (MU == 1) { // o2 += SG c1, o3 += -SG c0
      QPX_ADD((2 * 3 + cc) * 2, c1.re);
      QPX_ADD((2 * 3 + cc) * 2 + 1, c1.im);
      QPX_SUB((3 * 3 + cc) * 2, c0.re);
      QPX_SUB((3 * 3 + cc) * 2 + 1, c0.im);
    } else if (MU == 2) { // o2 += -SG i c0, o3 += SG i c1
      QPX_ADD((2 * 3 + cc) * 2, c0.im);
      QPX_SUB((2 * 3 + cc) * 2 + 1, c0.re);
      QPX_SUB((3 * 3 + cc) * 2, c1.im);
      QPX_ADD((3 * 3 + cc) * 2 + 1, c1.re);
    } else {              // o2 += SG c0, o3 += SG c1
      QPX_ADD((2 * 3 + cc) * 2, c0.re);
      QPX_ADD((2 * 3 + cc) * 2 + 1, c0.im);
      QPX_ADD((3 * 3 + cc) * 2, c1.re);
      QPX_ADD((3 * 3 + cc) * 2 + 1, c1.im);
    }
  }
#undef QPX_ADD
#undef QPX_SUB
}

// scale the projected half spinor once by the hop's coefficient x the
// spinor's per-site norm (x the twisted-boundary phase): the link multiply is
// linear, so this equals scaling its result
template <typename T>
__device__ __forceinline__ void scale_h(cx<T> h[2][3], T coeff, bool tw, cx<T> ph)
{
  if (tw) {
    cx<T> f = {coeff * ph.re, coeff * ph.im};
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) h[s][c] = cmul(h[s][c], f);
  } else {
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) h[s][c] = rmul(coeff, h[s][c]);
  }
}

// chi = U h (ADJ: U^+ h)
template <bool ADJ, typename T>
__device__ __forceinline__ void link_mult(const cx<T> u[3][3], const cx<T> h[2][3], cx<T> ch[2][3])
{
#pragma unroll
  for (int s = 0; s < 2; s++) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
      cx<T> v;
      if (!ADJ) {
        v = cmul(u[r][0], h[s][0]);
        v = cmad(u[r][1], h[s][1], v);
        v = cmad(u[r][2], h[s][2], v);
      } else {
        v = cmulcf(u[0][r], h[s][0]);
        v = cmadc(u[1][r], h[s][1], v);
        v = cmadc(u[2][r], h[s][2], v);
      }
      ch[s][r] = v;
    }
  }
}

// --- clover block products -------------------------------------------------
// out_block = A_b in_block for the packed Hermitian 6x6 block (diag[6],
// offd[15]); in/out index i = 3 * s2 + colour within spins (2b, 2b+1)
template <typename T>
__device__ __forceinline__ void herm6_apply(const T *blk, const T *in, T *out, int b)
{
  // blk: 36 reals
  cx<T> x[6], y[6];
#pragma unroll
  for (int i = 0; i < 6; i++) x[i] = {in[((2 * b + i / 3) * 3 + i % 3) * 2], in[((2 * b + i / 3) * 3 + i % 3) * 2 + 1]};
#pragma unroll
  for (int i = 0; i < 6; i++) y[i] = rmul(blk[i], x[i]);
#pragma unroll
  for (int i = 1; i < 6; i++) {
#pragma unroll
    for (int j = 0; j < i; j++) {
      int od = i * (i - 1) / 2 + j;
      cx<T> a = {blk[6 + 2 * od], blk[6 + 2 * od + 1]};
      y[i] = cmad(a, x[j], y[i]);
      y[j] = cmadc(a, x[i], y[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 6; i++) {
    out[((2 * b + i / 3) * 3 + i % 3) * 2] = y[i].re;
    out[((2 * b + i / 3) * 3 + i % 3) * 2 + 1] = y[i].im;
  }
}

// out_block += A_b in_block (packed Hermitian block as in herm6_apply)
template <typename T>
__device__ __forceinline__ void herm6_acc(const T *blk, const T *in, T *out, int b)
{
  cx<T> x[6], y[6];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    const int k = ((2 * b + i / 3) * 3 + i % 3) * 2;
    x[i] = {in[k], in[k + 1]};
    y[i] = {mad(blk[i], x[i].re, out[k]), mad(blk[i], x[i].im, out[k + 1])};
  }
#pragma unroll
  for (int i = 1; i < 6; i++) {
#pragma unroll
    for (int j = 0; j < i; j++) {
      int od = i * (i - 1) / 2 + j;
      cx<T> a = {blk[6 + 2 * od], blk[6 + 2 * od + 1]};
      y[i] = cmad(a, x[j], y[i]);
      y[j] = cmadc(a, x[i], y[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 6; i++) {
    out[((2 * b + i / 3) * 3 + i % 3) * 2] = y[i].re;
    out[((2 * b + i / 3) * 3 + i % 3) * 2 + 1] = y[i].im;
  }
}

// full complex 6x6 block, row-major (72 reals)
template <typename T>
__device__ __forceinline__ void full6_apply(const T *blk, const T *in, T *out, int b)
{
  cx<T> x[6];
#pragma unroll
  for (int i = 0; i < 6; i++) x[i] = {in[((2 * b + i / 3) * 3 + i % 3) * 2], in[((2 * b + i / 3) * 3 + i % 3) * 2 + 1]};
#pragma unroll
  for (int i = 0; i < 6; i++) {
    cx<T> y = cmul(cx<T>{blk[i * 12], blk[i * 12 + 1]}, x[0]);
#pragma unroll
    for (int j = 1; j < 6; j++) {
      cx<T> a = {blk[(i * 6 + j) * 2], blk[(i * 6 + j) * 2 + 1]};
      y = cmad(a, x[j], y);
    }
    out[((2 * b + i / 3) * 3 + i % 3) * 2] = y.re;
    out[((2 * b + i / 3) * 3 + i % 3) * 2 + 1] = y.im;
  }
}

// rows 2j, 2j+1 of a full complex 6x6 block (24 reals, row-major) applied to
// the block-b half of `in`
template <typename T>
__device__ __forceinline__ void full6_rows(const T *rows, const T *in, T *out, int b, int j)
{
  cx<T> x[6];
#pragma unroll
  for (int i = 0; i < 6; i++) x[i] = {in[((2 * b + i / 3) * 3 + i % 3) * 2], in[((2 * b + i / 3) * 3 + i % 3) * 2 + 1]};
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int i = 2 * j + q;
    cx<T> y = cmul(cx<T>{rows[q * 12], rows[q * 12 + 1]}, x[0]);
#pragma unroll
    for (int k = 1; k < 6; k++) y = cmad(cx<T>{rows[q * 12 + 2 * k], rows[q * 12 + 2 * k + 1]}, x[k], y);
    out[((2 * b + i / 3) * 3 + i % 3) * 2] = y.re;
    out[((2 * b + i / 3) * 3 + i % 3) * 2 + 1] = y.im;
  }
}

// per-lane values of a lane-generic type from SP doubles
__device__ __forceinline__ void lanes_set(double &d, const double *v) { d = v[0]; }
__device__ __forceinline__ void lanes_set(float &d, const double *v) { d = (float)v[0]; }
__device__ __forceinline__ void lanes_set(f2 &d, const double *v) { d = make_float2((float)v[0], (float)v[1]); }

// ---------------------------------------------------------------------------
// P      storage precision (arithmetic in P::real, or float2 lanes for SP = 2)
// RECON  12- or 18-real links
// EPI, ACHI  the operator epilogue (see the enums above)
// R      right-hand sides per thread (SP = 1)
// ISIGN  +1: D, -1: D^dagger
// SP     lattice sites per thread: 1, or 2 in float2 lanes (FP32 arithmetic)
// GEN    honour a.dir_mask and twisted boundary phases.  Without GEN every
//        hop is taken and no phase applied: the hops are then straight-line
//        code and the compiler can schedule every load early.
// RL     (with SP = 2, R = 1, fast path) the float2 lanes hold two
//        right-hand sides of one site instead of two sites: links and
//        clover terms are loaded once for both (RhsLanes).
// Blocks cover (site block, rhs tile) pairs with the rhs tile varying
// fastest, so the blocks that share a site block (and its links) run
// together and the links of the later right-hand sides come from L2.  (The
// site block varying fastest instead, each tile sweeping the lattice as a
// one-tile launch would, measured 5-17 % slower at 32^3x64 with 16 rhs and
// 24^3x48 with 24 rhs.)
//
// dslash_block is the work of one block: block `vblock` of a launch of
// `nvblocks` blocks, with POST_CG / POST_RAXPY coefficients read from `st`.
// dslash_kernel runs it once per CUDA block; the persistent solver kernels
// (qpx_persist.cuh) run it over all virtual blocks of a phase from a grid
// that stays resident.
template <typename P, int RECON, int EPI, int ACHI, int R, int ISIGN, int SP, bool GEN, bool RL = false>
__device__ __forceinline__ void dslash_block(const DslashArgs &a, const SolverState *st, int vblock, int nvblocks)
{
  using L = typename std::conditional<RL, RhsLanes<P>, Lanes<P, SP>>::type;
  using T = typename L::T;
  static_assert(SP == 1 || R == 1, "two sites per thread take one right-hand side");
  static_assert(!RL || (SP == 2 && R == 1 && !GEN), "right-hand-side lanes: SP = 2, R = 1, fast path");
  constexpr int RT = RL ? 2 : R;  // right-hand sides per thread
  const int ntiles = a.nrhs / RT;
  const int tile = vblock % ntiles;
  const int sblock = vblock / ntiles;
  const int rhs0 = tile * RT;
  int s[SP];
  bool act[SP];
  if (RL) {
    s[0] = sblock * QPX_BLOCK + threadIdx.x;
    act[0] = s[0] < a.geom.vh;
    s[SP - 1] = s[0];
    act[SP - 1] = act[0];
  } else if (SP == 1) {
    s[0] = sblock * QPX_BLOCK + threadIdx.x;
    act[0] = s[0] < a.geom.vh;
  } else {
    // each warp owns 64 consecutive sites: lane l takes sites l and l + 32,
    // so every load instruction of the warp reads 32 consecutive sites
    const int base = (sblock * QPX_BLOCK + (threadIdx.x & ~31)) * 2 + (threadIdx.x & 31);
    s[0] = base;
    act[0] = base < a.geom.vh;
    act[SP - 1] = base + 32 < a.geom.vh;
    s[SP - 1] = act[SP - 1] ? base + 32 : base;
  }
  double red[RT][QPX_MAX_RED];
#pragma unroll
  for (int r = 0; r < RT; r++)
#pragma unroll
    for (int k = 0; k < QPX_MAX_RED; k++) red[r][k] = 0.0;

  if (act[0]) {
    const Geom &g = a.geom;
    const int sxy = g.nxh;
    const int sxyz = g.nxh * g.ny;
    const int sxyzt = sxyz * g.nz;
    int nb[4][2][SP];  // [mu][0 back, 1 forward][lane]
    bool tlast[SP], tfirst[SP];
    // halo mode (general path, one site per thread): per direction, whether
    // the forward / backward hop leaves the block, and the neighbour's face site
    bool hlast[4] = {false, false, false, false}, hfirst[4] = {false, false, false, false};
    int hface[4] = {0, 0, 0, 0};
#pragma unroll
    for (int l = 0; l < (RL ? 1 : SP); l++) {
      int xh, y, z, t, par;
      const int sl = s[l];
      site_coords(g, sl, a.cb, xh, y, z, t, par);
      if (GEN && l == 0 && a.halo) {
        const int x = 2 * xh + par;
        hlast[0] = x + 1 == g.nx;
        hfirst[0] = x == 0;
        hlast[1] = y + 1 == g.ny;
        hfirst[1] = y == 0;
        hlast[2] = z + 1 == g.nz;
        hfirst[2] = z == 0;
        hlast[3] = t + 1 == g.nt;
        hfirst[3] = t == 0;
        hface[0] = ((t * g.nz + z) * g.ny + y) >> 1;
        hface[1] = (t * g.nz + z) * g.nxh + xh;
        hface[2] = (t * g.ny + y) * g.nxh + xh;
        hface[3] = (z * g.ny + y) * g.nxh + xh;
      }
      const int xf = (par == 0) ? xh : ((xh + 1 == g.nxh) ? 0 : xh + 1);
      const int xb = (par == 1) ? xh : ((xh == 0) ? g.nxh - 1 : xh - 1);
      nb[0][1][l] = sl - xh + xf;
      nb[0][0][l] = sl - xh + xb;
      nb[1][1][l] = sl + ((y + 1 == g.ny) ? -(g.ny - 1) * sxy : sxy);
      nb[1][0][l] = sl + ((y == 0) ? (g.ny - 1) * sxy : -sxy);
      nb[2][1][l] = sl + ((z + 1 == g.nz) ? -(g.nz - 1) * sxyz : sxyz);
      nb[2][0][l] = sl + ((z == 0) ? (g.nz - 1) * sxyz : -sxyz);
      nb[3][1][l] = sl + ((t + 1 == g.nt) ? -(g.nt - 1) * sxyzt : sxyzt);
      nb[3][0][l] = sl + ((t == 0) ? (g.nt - 1) * sxyzt : -sxyzt);
      tlast[l] = (t + 1 == g.nt);
      tfirst[l] = (t == 0);
    }
    if (RL) {  // both lanes are the same site
#pragma unroll
      for (int mu = 0; mu < 4; mu++)
#pragma unroll
        for (int d = 0; d < 2; d++) nb[mu][d][SP - 1] = nb[mu][d][0];
      tlast[SP - 1] = tlast[0];
      tfirst[SP - 1] = tfirst[0];
    }
    const T zero = splat<T>(0.0);
    T acc[R][24];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int k = 0; k < 24; k++) acc[r][k] = zero;

#define QPX_HOP(MU)                                                                       \
  {                                                                                       \
    const bool tw = GEN && ((a.tbc_mask >> MU) & 1);                                      \
    /* forward hop: U_mu(x) (1 - isign g) psi(x + mu) */                                  \
    if (!GEN || (a.dir_mask & (1u << (2 * MU + 1)))) {                                    \
      cx<T> u[3][3];                                                                      \
      L::template load_link<RECON>(a.gauge, a.cb, MU, s, u);                              \
      T cf;                                                                               \
      {                                                                                   \
        double c[SP];                                                                     \
        _Pragma("unroll") for (int l = 0; l < SP; l++) c[l] =                             \
            (MU < 3) ? a.coeff_s : (tlast[l] ? a.coeff_t_edge : a.coeff_t);               \
        lanes_set(cf, c);                                                                 \
      }                                                                                   \
      /* halo: the next block's first slice along MU (general path, one site per thread) */ \
      const bool ghf = GEN && ((a.halo >> MU) & 1) && hlast[MU];                          \
      int ixf[SP];                                                                        \
      _Pragma("unroll") for (int l = 0; l < SP; l++) ixf[l] = ghf ? hface[MU] : nb[MU][1][l]; \
      const cx<T> ph = {splat<T>(a.tbc[MU][0]), splat<T>(a.tbc[MU][1])};                  \
      _Pragma("unroll") for (int r = 0; r < R; r++)                                       \
      {                                                                                   \
        T nrm;                                                                            \
        cx<T> h[2][3], ch[2][3];                                                          \
        if constexpr (HalfProjection<L>::value) {                                         \
          __half2 w[12];                                                                  \
          load_h2(ghf ? a.ghost_fwd[MU] : a.in, rhs0 + r, ixf[0], w, nrm);                    \
          project_h2<MU, -ISIGN>(w, h);                                                   \
        } else if constexpr (RhsHalfProjection<L>::value) {                               \
          project_h2_pair<MU, -ISIGN>(a.in, rhs0 + r, ixf[0], h, nrm);                    \
        } else {                                                                          \
          T psi[24];                                                                      \
          L::load_raw(ghf ? a.ghost_fwd[MU] : a.in, rhs0 + r, ixf, psi, nrm);                 \
          project<MU, -ISIGN>(psi, h);                                                    \
        }                                                                                 \
        if (tw || SP == 2) { /* SP = 2: the folded form costs registers (spills) */       \
          scale_h(h, cf * nrm, tw, ph);                                                   \
          link_mult<false>(u, h, ch);                                                     \
          recons_add<MU, -ISIGN>(ch, acc[r]);                                             \
        } else {                                                                          \
          link_mult<false>(u, h, ch);                                                     \
          recons_add_c<MU, -ISIGN>(ch, acc[r], cf * nrm);                                 \
        }                                                                                 \
      }                                                                                   \
    }                                                                                     \
    /* backward hop: U_mu(x - mu)^+ (1 + isign g) psi(x - mu) */                          \
    if (!GEN || (a.dir_mask & (1u << (2 * MU)))) {                                        \
      /* halo: the previous block's last slice along MU and its U_MU (general path) */    \
      const bool ghb = GEN && ((a.halo >> MU) & 1) && hfirst[MU];                         \
      int ixb[SP];                                                                        \
      _Pragma("unroll") for (int l = 0; l < SP; l++) ixb[l] = ghb ? hface[MU] : nb[MU][0][l]; \
      cx<T> u[3][3];                                                                      \
      L::template load_link<RECON>(ghb ? a.ghost_link[MU] : a.gauge, ghb ? 0 : 1 - a.cb,  \
                                   ghb ? 0 : MU, ixb, u);                                 \
      T cf;                                                                               \
      {                                                                                   \
        double c[SP];                                                                     \
        _Pragma("unroll") for (int l = 0; l < SP; l++) c[l] =                             \
            (MU < 3) ? a.coeff_s                                                          \
                     : (tfirst[l] ? ((GEN && a.halo) ? a.coeff_t_bwd_edge : a.coeff_t_edge) \
                                  : a.coeff_t);                                           \
        lanes_set(cf, c);                                                                 \
      }                                                                                   \
      const cx<T> ph = {splat<T>(a.tbc[MU][0]), splat<T>(-a.tbc[MU][1])};                 \
      _Pragma("unroll") for (int r = 0; r < R; r++)                                       \
      {                                                                                   \
        T nrm;                                                                            \
        cx<T> h[2][3], ch[2][3];                                                          \
        if constexpr (HalfProjection<L>::value) {                                         \
          __half2 w[12];                                                                  \
          load_h2(ghb ? a.ghost_bwd[MU] : a.in, rhs0 + r, ixb[0], w, nrm);                    \
          project_h2<MU, ISIGN>(w, h);                                                    \
        } else if constexpr (RhsHalfProjection<L>::value) {                               \
          project_h2_pair<MU, ISIGN>(a.in, rhs0 + r, ixb[0], h, nrm);                     \
        } else {                                                                          \
          T psi[24];                                                                      \
          L::load_raw(ghb ? a.ghost_bwd[MU] : a.in, rhs0 + r, ixb, psi, nrm);                 \
          project<MU, ISIGN>(psi, h);                                                     \
        }                                                                                 \
        if (tw || SP == 2) { /* SP = 2: the folded form costs registers (spills) */       \
          scale_h(h, cf * nrm, tw, ph);                                                   \
          link_mult<true>(u, h, ch);                                                      \
          recons_add<MU, ISIGN>(ch, acc[r]);                                              \
        } else {                                                                          \
          link_mult<true>(u, h, ch);                                                      \
          recons_add_c<MU, ISIGN>(ch, acc[r], cf * nrm);                                  \
        }                                                                                 \
      }                                                                                   \
    }                                                                                     \
  }
    QPX_HOP(0)
    QPX_HOP(1)
    QPX_HOP(2)
    QPX_HOP(3)
#undef QPX_HOP

    // ---------------- epilogue ----------------
    T res[R][24];
    if (ACHI == ACHI_NONE) {
      if (EPI == EPI_NONE) {
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int k = 0; k < 24; k++) res[r][k] = acc[r][k];
      } else if (EPI == EPI_CLOV) {
#pragma unroll
        for (int b = 0; b < 2; b++) {
          T blk[36];
          L::template load_clover<72>(a.clov, s, 36 * b, 36, blk);
#pragma unroll
          for (int r = 0; r < R; r++) herm6_apply(blk, acc[r], res[r], b);
        }
      } else if (EPI == EPI_FCLOV) {
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            T rows[24];
            L::template load_clover<144>(a.clov, s, 72 * b + 24 * j, 24, rows);
#pragma unroll
            for (int r = 0; r < R; r++) full6_rows(rows, acc[r], res[r], b, j);
          }
      } else if (EPI == EPI_NDTM) {
        if constexpr (R == 2) {
          const T ca = splat<T>(a.alpha), cb = splat<T>(a.mu), ce = splat<T>(a.eps);
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T bb = (sp < 2) ? cb : -cb;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              const int k = (sp * 3 + c) * 2;
              const T ur = acc[0][k], ui = acc[0][k + 1], dr = acc[1][k], di = acc[1][k + 1];
              // up: (a + i bb) u + e d ; down: (a - i bb) d + e u
              res[0][k] = mad(ce, dr, mad(ca, ur, -(bb * ui)));
              res[0][k + 1] = mad(ce, di, mad(ca, ui, bb * ur));
              res[1][k] = mad(ce, ur, mad(ca, dr, bb * di));
              res[1][k + 1] = mad(ce, ui, mad(ca, di, -(bb * dr)));
            }
          }
        }
      } else if (EPI == EPI_NDFCLOV) {
        if constexpr (R == 2) {
#pragma unroll
          for (int b = 0; b < 2; b++) {
#pragma unroll
            for (int j = 0; j < 3; j++) {
              T rows[24];
              L::template load_clover<144>(a.clov, s, 72 * b + 24 * j, 24, rows);
              full6_rows(rows, acc[0], res[0], b, j);
              L::template load_clover<144>(a.clov2, s, 72 * b + 24 * j, 24, rows);
              full6_rows(rows, acc[1], res[1], b, j);
            }
            T blk[36];
            L::template load_clover<72>(a.clov3, s, 36 * b, 36, blk);
            herm6_acc(blk, acc[1], res[0], b);  // up += C down
            herm6_acc(blk, acc[0], res[1], b);  // down += C up
          }
        }
      } else {  // EPI_TMINV: mu_inv (1 - i mu isign g5) acc
        const T m = splat<T>(a.mu * ISIGN), mi = splat<T>(a.mu_inv);
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T mm = (sp < 2) ? m : -m;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              T re = acc[r][(sp * 3 + c) * 2], im = acc[r][(sp * 3 + c) * 2 + 1];
              res[r][(sp * 3 + c) * 2] = mi * mad(mm, im, re);
              res[r][(sp * 3 + c) * 2 + 1] = mi * mad(-mm, re, im);
            }
          }
      }
    } else {
      const T nbeta = splat<T>(-a.beta);
      T chi[R][24];
#pragma unroll
      for (int r = 0; r < R; r++) L::load(a.chi, rhs0 + r, s, chi[r]);
      if (ACHI == ACHI_ALPHA) {
        const T al = splat<T>(a.alpha);
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int k = 0; k < 24; k++) res[r][k] = mad(nbeta, acc[r][k], al * chi[r][k]);
      } else if (ACHI == ACHI_CLOV) {
#pragma unroll
        for (int b = 0; b < 2; b++) {
          T blk[36];
          L::template load_clover<72>(a.clov, s, 36 * b, 36, blk);
#pragma unroll
          for (int r = 0; r < R; r++) herm6_apply(blk, chi[r], res[r], b);
        }
        const T rh = splat<T>(a.rho * ISIGN);
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T rr = (sp < 2) ? rh : -rh;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              int k = (sp * 3 + c) * 2;
              // res += i rr chi - beta acc
              res[r][k] = mad(nbeta, acc[r][k], mad(-rr, chi[r][k + 1], res[r][k]));
              res[r][k + 1] = mad(nbeta, acc[r][k + 1], mad(rr, chi[r][k], res[r][k + 1]));
            }
          }
      } else if (ACHI == ACHI_NDTM) {
        if constexpr (R == 2) {
          const T al = splat<T>(a.alpha), m = splat<T>(a.mu * ISIGN), ne = splat<T>(-a.eps);
#pragma unroll
          for (int f = 0; f < 2; f++) {
#pragma unroll
            for (int sp = 0; sp < 4; sp++) {
              // s_f g5 isign mu
              const T mm = ((sp < 2) == (f == 0)) ? m : -m;
#pragma unroll
              for (int c = 0; c < 3; c++) {
                const int k = (sp * 3 + c) * 2;
                const T re = chi[f][k], im = chi[f][k + 1];
                res[f][k] = mad(ne, chi[1 - f][k], mad(nbeta, acc[f][k], al * mad(-mm, im, re)));
                res[f][k + 1] = mad(ne, chi[1 - f][k + 1], mad(nbeta, acc[f][k + 1], al * mad(mm, re, im)));
              }
            }
          }
        }
      } else if (ACHI == ACHI_NDCLOV) {
        if constexpr (R == 2) {
#pragma unroll
          for (int b = 0; b < 2; b++) {
            T blk[36];
            L::template load_clover<72>(a.clov, s, 36 * b, 36, blk);
#pragma unroll
            for (int r = 0; r < 2; r++) herm6_apply(blk, chi[r], res[r], b);
          }
          const T rh = splat<T>(a.rho * ISIGN), ne = splat<T>(-a.eps);
#pragma unroll
          for (int f = 0; f < 2; f++)
#pragma unroll
            for (int sp = 0; sp < 4; sp++) {
              const T rr = ((sp < 2) == (f == 0)) ? rh : -rh;  // s_f g5 isign rho
#pragma unroll
              for (int c = 0; c < 3; c++) {
                const int k = (sp * 3 + c) * 2;
                res[f][k] = mad(ne, chi[1 - f][k], mad(nbeta, acc[f][k], mad(-rr, chi[f][k + 1], res[f][k])));
                res[f][k + 1] =
                    mad(ne, chi[1 - f][k + 1], mad(nbeta, acc[f][k + 1], mad(rr, chi[f][k], res[f][k + 1])));
              }
            }
        }
      } else {  // ACHI_TM: alpha (1 + i mu isign g5) chi - beta acc
        const T al = splat<T>(a.alpha), m = splat<T>(a.mu * ISIGN);
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T mm = (sp < 2) ? m : -m;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              int k = (sp * 3 + c) * 2;
              T re = chi[r][k], im = chi[r][k + 1];
              res[r][k] = mad(nbeta, acc[r][k], al * mad(-mm, im, re));
              res[r][k + 1] = mad(nbeta, acc[r][k + 1], al * mad(mm, re, im));
            }
          }
      }
      // <out, chi> reduction needs chi
      if (a.red.mask & RED_DOT_OUT_CHI) {
        if constexpr (RL) {
          double re[2], im[2];
          red_dot_pair(res[0], chi[0], re, im);
          red[0][3] = re[0];
          red[0][4] = im[0];
          red[1][3] = re[1];
          red[1][4] = im[1];
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) red_dot(res[r], chi[r], act, red[r][3], red[r][4]);
        }
      }
    }

    // g5_out: the result times gamma_5 = diag(1, 1, -1, -1) (spins 2 and 3
    // negated, exactly) before the post operation and the norm reductions;
    // the <out, chi> value above is taken before it, so the host never
    // combines the two.  The persistent CG applies M^+ = gamma_5 M gamma_5
    // this way with the isign = +1 kernels.
    if (a.g5_out) {
#pragma unroll
      for (int r = 0; r < R; r++)
#pragma unroll
        for (int k = 12; k < 24; k++) res[r][k] = -res[r][k];
    }

    // ---------------- post op + reductions ----------------
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int rr = rhs0 + r;
      if (rr >= a.nrhs) continue;
      if (a.red.mask & RED_NORM_OUT) {
        if constexpr (RL)
          red_norm_pair(res[0], red[0][0], red[1][0]);
        else
          red[r][0] = red_norm(res[r], act);
      }
      if (a.red.mask & RED_DOT_W_OUT) {
        T w[24];
        L::load(a.w, rr, s, w);
        if constexpr (RL) {
          double re[2], im[2];
          red_dot_pair(w, res[0], re, im);
          red[0][1] = re[0];
          red[0][2] = im[0];
          red[1][1] = re[1];
          red[1][2] = im[1];
        } else {
          red_dot(w, res[r], act, red[r][1], red[r][2]);
        }
      }
      if (a.post == POST_STORE) {
        L::store(a.out, rr, s, act, res[r]);
      } else if (a.post == POST_RAXPY) {  // r += b mmp ; |r|^2
        const T cb_ = rhs_coef<RL, T>(st->v[S_B], rr);
        T rv[24];
        L::load(a.r, rr, s, rv);
#pragma unroll
        for (int k = 0; k < 24; k++) rv[k] = mad(cb_, res[r][k], rv[k]);
        L::store(a.r, rr, s, act, rv);
        if constexpr (RL)
          red_norm_pair(rv, red[0][5], red[1][5]);
        else
          red[r][5] = red_norm(rv, act);
      } else {  // POST_CG: r -= a mmp ; x += a p ; |r|^2
        const T ca = rhs_coef<RL, T>(st->v[S_A], rr), nca = -ca;
        T rv[24], xv[24], pv[24];
        L::load(a.r, rr, s, rv);
        L::load(a.x, rr, s, xv);
        L::load(a.p, rr, s, pv);
#pragma unroll
        for (int k = 0; k < 24; k++) {
          rv[k] = mad(nca, res[r][k], rv[k]);
          xv[k] = mad(ca, pv[k], xv[k]);
        }
        L::store(a.r, rr, s, act, rv);
        L::store(a.x, rr, s, act, xv);
        if constexpr (RL)
          red_norm_pair(rv, red[0][5], red[1][5]);
        else
          red[r][5] = red_norm(rv, act);
      }
    }
  }
  if (a.red.mask)
    reduce_epilogue<RT>(a.red, a.nrhs, rhs0, red_slots(a.red.mask), red, sblock, nvblocks / ntiles);
}

template <typename P, int RECON, int EPI, int ACHI, int R, int ISIGN, int SP, bool GEN, bool RL = false>
__global__ void QPX_DSLASH_BOUNDS dslash_kernel(const __grid_constant__ DslashArgs a)
{
  pdl_wait();
  pdl_trigger();
  if (a.state && a.state->done) return;
  dslash_block<P, RECON, EPI, ACHI, R, ISIGN, SP, GEN, RL>(a, a.state, blockIdx.x, gridDim.x);
}

}  // namespace qpx
