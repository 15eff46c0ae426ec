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
#include "qpx_reduce.cuh"

namespace qpx {

enum Epi : int { EPI_NONE = 0, EPI_CLOV = 1, EPI_TMINV = 2, EPI_FCLOV = 3 };
enum Achi : int { ACHI_NONE = 0, ACHI_ALPHA = 1, ACHI_CLOV = 2, ACHI_TM = 3 };
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
  double coeff_s;       // spatial hops (aniso_s, times the caller's beta)
  double coeff_t;       // temporal hops away from the t edges (aniso_t)
  double coeff_t_edge;  // temporal hops across the global t edge (aniso_t * t_boundary)
  int tbc_mask;
  double tbc[4][2];
  double alpha, beta;   // a chi - b D psi
  double mu, mu_inv;    // twisted mass
  double rho;           // i rho gamma_5 term
  int post;
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

// --- reconstruct-accumulate of (1 + SG gamma_mu) from chi = U h -------------
template <int MU, int SG, typename T>
__device__ __forceinline__ void recons_add(const cx<T> ch[2][3], T *acc)
{
  const T sg = (T)SG;  // +-1: folded into add / subtract by the compiler
#pragma unroll
  for (int c = 0; c < 3; c++) {
    cx<T> c0 = ch[0][c], c1 = ch[1][c];
    acc[(0 * 3 + c) * 2] += c0.re;
    acc[(0 * 3 + c) * 2 + 1] += c0.im;
    acc[(1 * 3 + c) * 2] += c1.re;
    acc[(1 * 3 + c) * 2 + 1] += c1.im;
    if (MU == 0) {        // o2 += -SG i c1, o3 += -SG i c0
      acc[(2 * 3 + c) * 2] += sg * c1.im;
      acc[(2 * 3 + c) * 2 + 1] -= sg * c1.re;
      acc[(3 * 3 + c) * 2] += sg * c0.im;
      acc[(3 * 3 + c) * 2 + 1] -= sg * c0.re;
    } else if (MU == 1) { // o2 += SG c1, o3 += -SG c0
      acc[(2 * 3 + c) * 2] += sg * c1.re;
      acc[(2 * 3 + c) * 2 + 1] += sg * c1.im;
      acc[(3 * 3 + c) * 2] -= sg * c0.re;
      acc[(3 * 3 + c) * 2 + 1] -= sg * c0.im;
    } else if (MU == 2) { // o2 += -SG i c0, o3 += SG i c1
      acc[(2 * 3 + c) * 2] += sg * c0.im;
      acc[(2 * 3 + c) * 2 + 1] -= sg * c0.re;
      acc[(3 * 3 + c) * 2] -= sg * c1.im;
      acc[(3 * 3 + c) * 2 + 1] += sg * c1.re;
    } else {              // o2 += SG c0, o3 += SG c1
      acc[(2 * 3 + c) * 2] += sg * c0.re;
      acc[(2 * 3 + c) * 2 + 1] += sg * c0.im;
      acc[(3 * 3 + c) * 2] += sg * c1.re;
      acc[(3 * 3 + c) * 2 + 1] += sg * c1.im;
    }
  }
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
      for (int c = 0; c < 3; c++) h[s][c] = h[s][c] * f;
  } else {
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
      for (int c = 0; c < 3; c++) h[s][c] = coeff * h[s][c];
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
        v = u[r][0] * h[s][0];
        v = v + u[r][1] * h[s][1];
        v = v + u[r][2] * h[s][2];
      } else {
        v = cmulc(u[0][r], h[s][0]);
        v = v + cmulc(u[1][r], h[s][1]);
        v = v + cmulc(u[2][r], h[s][2]);
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
  for (int i = 0; i < 6; i++) y[i] = blk[i] * x[i];
#pragma unroll
  for (int i = 1; i < 6; i++) {
#pragma unroll
    for (int j = 0; j < i; j++) {
      int od = i * (i - 1) / 2 + j;
      cx<T> a = {blk[6 + 2 * od], blk[6 + 2 * od + 1]};
      y[i] = y[i] + a * x[j];
      y[j] = y[j] + cmulc(a, x[i]);
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
    cx<T> y = {0, 0};
#pragma unroll
    for (int j = 0; j < 6; j++) {
      cx<T> a = {blk[(i * 6 + j) * 2], blk[(i * 6 + j) * 2 + 1]};
      y = y + a * x[j];
    }
    out[((2 * b + i / 3) * 3 + i % 3) * 2] = y.re;
    out[((2 * b + i / 3) * 3 + i % 3) * 2 + 1] = y.im;
  }
}

// ---------------------------------------------------------------------------
template <typename P, int RECON, int EPI, int ACHI, int R, int ISIGN>
__global__ void __launch_bounds__(QPX_BLOCK) dslash_kernel(const DslashArgs a)
{
  using T = typename P::real;
  if (a.state && a.state->done) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs0 = blockIdx.y * R;
  const bool active = s < a.geom.vh;
  double red[R][QPX_MAX_RED];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < QPX_MAX_RED; k++) red[r][k] = 0.0;

  if (active) {
    const Geom &g = a.geom;
    int xh, y, z, t, par;
    site_coords(g, s, a.cb, xh, y, z, t, par);
    // neighbour cb indices
    const int sxy = g.nxh;
    const int sxyz = g.nxh * g.ny;
    const int sxyzt = sxyz * g.nz;
    int nb[4][2];  // [mu][0 back, 1 forward]
    {
      int xf = (par == 0) ? xh : ((xh + 1 == g.nxh) ? 0 : xh + 1);
      int xb = (par == 1) ? xh : ((xh == 0) ? g.nxh - 1 : xh - 1);
      nb[0][1] = s - xh + xf;
      nb[0][0] = s - xh + xb;
      nb[1][1] = s + ((y + 1 == g.ny) ? -(g.ny - 1) * sxy : sxy);
      nb[1][0] = s + ((y == 0) ? (g.ny - 1) * sxy : -sxy);
      nb[2][1] = s + ((z + 1 == g.nz) ? -(g.nz - 1) * sxyz : sxyz);
      nb[2][0] = s + ((z == 0) ? (g.nz - 1) * sxyz : -sxyz);
      nb[3][1] = s + ((t + 1 == g.nt) ? -(g.nt - 1) * sxyzt : sxyzt);
      nb[3][0] = s + ((t == 0) ? (g.nt - 1) * sxyzt : -sxyzt);
    }
    const T sgn = (T)ISIGN;
    T acc[R][24];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int k = 0; k < 24; k++) acc[r][k] = 0;

#define QPX_HOP(MU)                                                                       \
  {                                                                                       \
    const T cs = (MU == 3) ? (T)0 : (T)a.coeff_s;                                         \
    const bool tw = (a.tbc_mask >> MU) & 1;                                               \
    /* forward hop: U_mu(x) (1 - isign g) psi(x + mu) */                                  \
    if (a.dir_mask & (1u << (2 * MU + 1))) {                                              \
      cx<T> u[3][3];                                                                      \
      GaugeIO<P, RECON>::load(a.gauge, a.cb, MU, s, u);                                   \
      T cf = cs;                                                                          \
      if (MU == 3) cf = (T)((t + 1 == g.nt) ? a.coeff_t_edge : a.coeff_t);                \
      cx<T> ph = {(T)a.tbc[MU][0], (T)a.tbc[MU][1]};                                      \
      _Pragma("unroll") for (int r = 0; r < R; r++)                                       \
      {                                                                                   \
        T psi[24], nrm;                                                                   \
        SpinorIO<P>::load_raw(a.in, rhs0 + r, nb[MU][1], psi, nrm);                      \
        cx<T> h[2][3], ch[2][3];                                                          \
        project<MU, -ISIGN>(psi, h);                                                      \
        scale_h(h, cf * nrm, tw, ph);                                                     \
        link_mult<false>(u, h, ch);                                                       \
        recons_add<MU, -ISIGN>(ch, acc[r]);                                               \
      }                                                                                   \
    }                                                                                     \
    /* backward hop: U_mu(x - mu)^+ (1 + isign g) psi(x - mu) */                          \
    if (a.dir_mask & (1u << (2 * MU))) {                                                  \
      cx<T> u[3][3];                                                                      \
      GaugeIO<P, RECON>::load(a.gauge, 1 - a.cb, MU, nb[MU][0], u);                       \
      T cf = cs;                                                                          \
      if (MU == 3) cf = (T)((t == 0) ? a.coeff_t_edge : a.coeff_t);                       \
      cx<T> ph = {(T)a.tbc[MU][0], -(T)a.tbc[MU][1]};                                     \
      _Pragma("unroll") for (int r = 0; r < R; r++)                                       \
      {                                                                                   \
        T psi[24], nrm;                                                                   \
        SpinorIO<P>::load_raw(a.in, rhs0 + r, nb[MU][0], psi, nrm);                      \
        cx<T> h[2][3], ch[2][3];                                                          \
        project<MU, ISIGN>(psi, h);                                                       \
        scale_h(h, cf * nrm, tw, ph);                                                     \
        link_mult<true>(u, h, ch);                                                        \
        recons_add<MU, ISIGN>(ch, acc[r]);                                                \
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
          CloverIO<P, 72>::load(a.clov, s, 36 * b, 36, blk);
#pragma unroll
          for (int r = 0; r < R; r++) herm6_apply(blk, acc[r], res[r], b);
        }
      } else if (EPI == EPI_FCLOV) {
#pragma unroll
        for (int b = 0; b < 2; b++) {
          T blk[72];
          CloverIO<P, 144>::load(a.clov, s, 72 * b, 72, blk);
#pragma unroll
          for (int r = 0; r < R; r++) full6_apply(blk, acc[r], res[r], b);
        }
      } else {  // EPI_TMINV: mu_inv (1 - i mu isign g5) acc
        const T m = (T)a.mu * sgn, mi = (T)a.mu_inv;
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T mm = (sp < 2) ? m : -m;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              T re = acc[r][(sp * 3 + c) * 2], im = acc[r][(sp * 3 + c) * 2 + 1];
              res[r][(sp * 3 + c) * 2] = mi * (re + mm * im);
              res[r][(sp * 3 + c) * 2 + 1] = mi * (im - mm * re);
            }
          }
      }
    } else {
      const T beta = (T)a.beta;
      T chi[R][24];
#pragma unroll
      for (int r = 0; r < R; r++) SpinorIO<P>::load(a.chi, rhs0 + r, s, chi[r]);
      if (ACHI == ACHI_ALPHA) {
        const T al = (T)a.alpha;
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int k = 0; k < 24; k++) res[r][k] = al * chi[r][k] - beta * acc[r][k];
      } else if (ACHI == ACHI_CLOV) {
#pragma unroll
        for (int b = 0; b < 2; b++) {
          T blk[36];
          CloverIO<P, 72>::load(a.clov, s, 36 * b, 36, blk);
#pragma unroll
          for (int r = 0; r < R; r++) herm6_apply(blk, chi[r], res[r], b);
        }
        const T rh = (T)a.rho * sgn;
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T rr = (sp < 2) ? rh : -rh;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              int k = (sp * 3 + c) * 2;
              res[r][k] += -rr * chi[r][k + 1] - beta * acc[r][k];
              res[r][k + 1] += rr * chi[r][k] - beta * acc[r][k + 1];
            }
          }
      } else {  // ACHI_TM: alpha (1 + i mu isign g5) chi - beta acc
        const T al = (T)a.alpha, m = (T)a.mu * sgn;
#pragma unroll
        for (int r = 0; r < R; r++)
#pragma unroll
          for (int sp = 0; sp < 4; sp++) {
            const T mm = (sp < 2) ? m : -m;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              int k = (sp * 3 + c) * 2;
              T re = chi[r][k], im = chi[r][k + 1];
              res[r][k] = al * (re - mm * im) - beta * acc[r][k];
              res[r][k + 1] = al * (im + mm * re) - beta * acc[r][k + 1];
            }
          }
      }
      // <out, chi> reduction needs chi
      if (a.red.mask & RED_DOT_OUT_CHI) {
#pragma unroll
        for (int r = 0; r < R; r++) {
          double dre = 0, dim = 0;
#pragma unroll
          for (int k = 0; k < 24; k += 2) {
            dre += (double)res[r][k] * chi[r][k] + (double)res[r][k + 1] * chi[r][k + 1];
            dim += (double)res[r][k] * chi[r][k + 1] - (double)res[r][k + 1] * chi[r][k];
          }
          red[r][3] = dre;
          red[r][4] = dim;
        }
      }
    }

    // ---------------- post op + reductions ----------------
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int rr = rhs0 + r;
      if (rr >= a.nrhs) continue;
      if (a.red.mask & RED_NORM_OUT) {
        double n2 = 0;
#pragma unroll
        for (int k = 0; k < 24; k++) n2 += (double)res[r][k] * res[r][k];
        red[r][0] = n2;
      }
      if (a.red.mask & RED_DOT_W_OUT) {
        T w[24];
        SpinorIO<P>::load(a.w, rr, s, w);
        double dre = 0, dim = 0;
#pragma unroll
        for (int k = 0; k < 24; k += 2) {
          dre += (double)w[k] * res[r][k] + (double)w[k + 1] * res[r][k + 1];
          dim += (double)w[k] * res[r][k + 1] - (double)w[k + 1] * res[r][k];
        }
        red[r][1] = dre;
        red[r][2] = dim;
      }
      if (a.post == POST_STORE) {
        SpinorIO<P>::store(a.out, rr, s, res[r]);
      } else if (a.post == POST_RAXPY) {  // r += b mmp ; |r|^2
        const T cb_ = (T)a.state->v[S_B][rr];
        T rv[24];
        SpinorIO<P>::load(a.r, rr, s, rv);
        double n2 = 0;
#pragma unroll
        for (int k = 0; k < 24; k++) {
          rv[k] += cb_ * res[r][k];
          n2 += (double)rv[k] * rv[k];
        }
        SpinorIO<P>::store(a.r, rr, s, rv);
        red[r][5] = n2;
      } else {  // POST_CG: r -= a mmp ; x += a p ; |r|^2
        const T ca = (T)a.state->v[S_A][rr];
        T rv[24], xv[24], pv[24];
        SpinorIO<P>::load(a.r, rr, s, rv);
        SpinorIO<P>::load(a.x, rr, s, xv);
        SpinorIO<P>::load(a.p, rr, s, pv);
        double n2 = 0;
#pragma unroll
        for (int k = 0; k < 24; k++) {
          rv[k] -= ca * res[r][k];
          xv[k] += ca * pv[k];
          n2 += (double)rv[k] * rv[k];
        }
        SpinorIO<P>::store(a.r, rr, s, rv);
        SpinorIO<P>::store(a.x, rr, s, xv);
        red[r][5] = n2;
      }
    }
  }
  if (a.red.mask) reduce_epilogue<R>(a.red, a.state, a.nrhs, rhs0, red_slots(a.red.mask), red);
}

}  // namespace qpx
