// Streaming BLAS over checkerboarded spinor fields, each fused the way the
// reference fuses it (include/qphix/blas_new_c.h, real_functors.h,
// complex_functors.h): one pass over the vectors, arithmetic in the field's
// compute type, reductions accumulated in FP64 and folded deterministically
// by reduce_epilogue.  Coefficients come either from the launch (host values)
// or from a SolverState slot (device-resident Krylov scalars), per rhs.
#pragma once

#include "qpx_common.cuh"
#include "qpx_reduce.cuh"

namespace qpx {

// complex coefficient: state slot pointers (per rhs) if set, else the value
struct Coef {
  double re, im;
  const double *pre, *pim;
  __device__ __forceinline__ double r(int rhs) const { return pre ? pre[rhs] : re; }
  __device__ __forceinline__ double i(int rhs) const { return pim ? pim[rhs] : im; }
};

enum BlasOp : int {
  B_NORM2 = 0,     // red: |x|^2
  B_DOT,           // red: <x, y>
  B_DOTNORM,       // red: <x, y>, |x|^2           (innerProductNorm)
  B_COPY,          // y = x
  B_ZERO,          // x = 0
  B_CAXPBY,        // y = a x + b y                (ax, axy, axpy, axpby, aypx, caxpy)
  B_CAXPBY_NORM,   // y = a x + b y, red |y|^2     (axpyNorm2)
  B_XMY_NORM,      // z = x - y, red |z|^2          (xmyNorm2Spinor)
  B_BICG_P,        // p = r + beta (p - omega v)    (bicgstab_p_update)
  B_BICG_S,        // r = r - alpha v               (bicgstab_s_update)
  B_BICG_RX,       // x += omega r + alpha p ; r -= omega t ; red |r|^2, <w, r>
  B_CG_P,          // p = r + b p                   (aypx with device b)
  B_MR_RX,         // x += a r ; r -= a Mr ; red |r|^2
  B_RICH_RX,       // x += dx ; r -= t ; red |r|^2  (richardson_rxupdateNormR)
  B_G5,            // y = gamma_5 x
  B_CG_RX,         // x += a p ; r -= a (q + s p) ; red |r|^2   (CG on M^+M + s, s per rhs)
};

// BLAS reductions use red.mask directly as the slot set: B_NORM2 / the
// *_NORM ops fill slot 0, B_DOT slots 0-1, B_DOTNORM / B_BICG_RX slots 0-2.
struct BlasArgs {
  int op;
  int vh;
  int nrhs;
  SpinorArg x, y, z, w, v;  // operand roles documented per op
  Coef a, b, c;
  ReduceArg red;
  SolverState *state;
};

template <typename T>
__device__ __forceinline__ void caxpy_(T *y, double ar, double ai, const T *x)
{
  const T r = (T)ar, i = (T)ai;
#pragma unroll
  for (int k = 0; k < 24; k += 2) {
    T xr = x[k], xi = x[k + 1];
    y[k] += r * xr - i * xi;
    y[k + 1] += r * xi + i * xr;
  }
}

// Reduction terms of one site: FP64 fields keep their element loops (pairs
// of reals where the reference's functors pair them); FP32-arithmetic fields
// sum in FP32 per thread and convert once (red_norm / red_dot).
template <bool PAIRS, typename T>
__device__ __forceinline__ double blas_norm(const T *x)
{
  if constexpr (std::is_same<T, double>::value) {
    double n = 0;
    if (PAIRS) {
#pragma unroll
      for (int k = 0; k < 24; k += 2) n += (double)x[k] * x[k] + (double)x[k + 1] * x[k + 1];
    } else {
#pragma unroll
      for (int k = 0; k < 24; k++) n += (double)x[k] * x[k];
    }
    return n;
  } else {
    const bool one[1] = {true};
    return red_norm(x, one);
  }
}

template <typename T>
__device__ __forceinline__ void blas_dot(const T *x, const T *y, double &re, double &im)
{
  if constexpr (std::is_same<T, double>::value) {
    double dr = 0, di = 0;
#pragma unroll
    for (int k = 0; k < 24; k += 2) {
      dr += (double)x[k] * y[k] + (double)x[k + 1] * y[k + 1];
      di += (double)x[k] * y[k + 1] - (double)x[k + 1] * y[k];
    }
    re = dr;
    im = di;
  } else {
    const bool one[1] = {true};
    red_dot(x, y, one, re, im);
  }
}

template <typename P>
__global__ void __launch_bounds__(QPX_BLOCK) blas_kernel(const BlasArgs a)
{
  using T = typename P::real;
  using IO = SpinorIO<P>;
  pdl_wait();
  pdl_trigger();
  if (a.state && a.state->done) return;
  const int rhs = blockIdx.y;
  double red[1][QPX_MAX_RED];
#pragma unroll
  for (int k = 0; k < QPX_MAX_RED; k++) red[0][k] = 0;
  // grid-stride over the sites: a launch with fewer blocks than Vh / 128
  // gives each thread several sites (and the fold fewer block partials); a
  // thread's per-site values are added in site order
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < a.vh; s += gridDim.x * blockDim.x) {
    double sr[1][QPX_MAX_RED];
#pragma unroll
    for (int k = 0; k < QPX_MAX_RED; k++) sr[0][k] = 0;
    T x[24], y[24];
    switch (a.op) {
    case B_NORM2: {
      IO::load(a.x, rhs, s, x);
      sr[0][0] = blas_norm<false>(x);
      break;
    }
    case B_DOT:
    case B_DOTNORM: {
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      blas_dot(x, y, sr[0][0], sr[0][1]);
      if (a.op == B_DOTNORM) sr[0][2] = blas_norm<true>(x);
      break;
    }
    case B_COPY:
      IO::load(a.x, rhs, s, x);
      IO::store(a.y, rhs, s, x);
      break;
    case B_ZERO:
#pragma unroll
      for (int k = 0; k < 24; k++) x[k] = 0;
      IO::store(a.x, rhs, s, x);
      break;
    case B_CAXPBY:
    case B_CAXPBY_NORM: {
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      const T ar = (T)a.a.r(rhs), ai = (T)a.a.i(rhs), br = (T)a.b.r(rhs), bi = (T)a.b.i(rhs);
#pragma unroll
      for (int k = 0; k < 24; k += 2) {
        T yr = ar * x[k] - ai * x[k + 1] + br * y[k] - bi * y[k + 1];
        T yi = ar * x[k + 1] + ai * x[k] + br * y[k + 1] + bi * y[k];
        y[k] = yr;
        y[k + 1] = yi;
      }
      IO::store(a.y, rhs, s, y);
      if (a.op == B_CAXPBY_NORM) sr[0][0] = blas_norm<true>(y);
      break;
    }
    case B_XMY_NORM: {
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
#pragma unroll
      for (int k = 0; k < 24; k++) x[k] -= y[k];
      IO::store(a.z, rhs, s, x);
      sr[0][0] = blas_norm<false>(x);
      break;
    }
    case B_BICG_P: {  // x = r, y = p, z = v ; a = beta, b = omega
      T v[24];
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      IO::load(a.z, rhs, s, v);
      const T br = (T)a.a.r(rhs), bi = (T)a.a.i(rhs), orr = (T)a.b.r(rhs), oi = (T)a.b.i(rhs);
#pragma unroll
      for (int k = 0; k < 24; k += 2) {
        T tr = y[k] - (orr * v[k] - oi * v[k + 1]);
        T ti = y[k + 1] - (orr * v[k + 1] + oi * v[k]);
        y[k] = x[k] + br * tr - bi * ti;
        y[k + 1] = x[k + 1] + br * ti + bi * tr;
      }
      IO::store(a.y, rhs, s, y);
      break;
    }
    case B_BICG_S: {  // x = r (in/out), y = v ; a = alpha
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      caxpy_(x, -a.a.r(rhs), -a.a.i(rhs), y);
      IO::store(a.x, rhs, s, x);
      break;
    }
    case B_BICG_RX: {  // x = x, y = r, z = t, v = p, w = r0 ; a = omega, b = alpha
      T t[24], p[24];
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      IO::load(a.z, rhs, s, t);
      IO::load(a.v, rhs, s, p);
      const double orr = a.a.r(rhs), oi = a.a.i(rhs);
      caxpy_(x, orr, oi, y);
      caxpy_(x, a.b.r(rhs), a.b.i(rhs), p);
      caxpy_(y, -orr, -oi, t);
      IO::store(a.x, rhs, s, x);
      IO::store(a.y, rhs, s, y);
      T w[24];
      IO::load(a.w, rhs, s, w);
      sr[0][0] = blas_norm<true>(y);
      blas_dot(w, y, sr[0][1], sr[0][2]);
      break;
    }
    case B_CG_P: {  // x = r, y = p ; a = b ; with a reduction: |p|^2 (shifted CG)
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      const T b = (T)a.a.r(rhs);
#pragma unroll
      for (int k = 0; k < 24; k++) y[k] = x[k] + b * y[k];
      IO::store(a.y, rhs, s, y);
      if (a.red.mask) sr[0][0] = blas_norm<false>(y);
      break;
    }
    case B_CG_RX: {  // x = x, y = r, z = q = M^+M p, v = p ; a = alpha, b = shift
      T q[24], p[24];
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      IO::load(a.z, rhs, s, q);
      IO::load(a.v, rhs, s, p);
      const T al = (T)a.a.r(rhs), sg = (T)a.b.r(rhs);
#pragma unroll
      for (int k = 0; k < 24; k++) {
        x[k] += al * p[k];
        y[k] -= al * (q[k] + sg * p[k]);
      }
      IO::store(a.x, rhs, s, x);
      IO::store(a.y, rhs, s, y);
      sr[0][0] = blas_norm<false>(y);
      break;
    }
    case B_MR_RX: {  // x = x, y = r, z = Mr ; a = a
      T mr[24];
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      IO::load(a.z, rhs, s, mr);
      const double ar = a.a.r(rhs), ai = a.a.i(rhs);
      caxpy_(x, ar, ai, y);
      caxpy_(y, -ar, -ai, mr);
      IO::store(a.x, rhs, s, x);
      IO::store(a.y, rhs, s, y);
      sr[0][0] = blas_norm<false>(y);
      break;
    }
    case B_RICH_RX: {  // x = x, y = r, z = dx, w = t
      T dx[24], t[24];
      IO::load(a.x, rhs, s, x);
      IO::load(a.y, rhs, s, y);
      IO::load(a.z, rhs, s, dx);
      IO::load(a.w, rhs, s, t);
#pragma unroll
      for (int k = 0; k < 24; k++) {
        x[k] += dx[k];
        y[k] -= t[k];
      }
      IO::store(a.x, rhs, s, x);
      IO::store(a.y, rhs, s, y);
      sr[0][0] = blas_norm<false>(y);
      break;
    }
    case B_G5: {
      IO::load(a.x, rhs, s, x);
#pragma unroll
      for (int k = 12; k < 24; k++) x[k] = -x[k];
      IO::store(a.y, rhs, s, x);
      break;
    }
    default:
      break;
    }
#pragma unroll
    for (int k = 0; k < QPX_MAX_RED; k++) red[0][k] += sr[0][k];
  }
  if (a.red.mask) reduce_epilogue<1>(a.red, a.nrhs, rhs, a.red.mask, red);
}

// Multishift CG vector update (include/qphix/minvcg.h:279-384), fused across
// iterations: the x update of iteration k (x_s -= beta_s p_s, with
// xcoef_s = beta_s for shifts still active in k, else 0) and the p updates of
// iteration k+1 (p_s = zeta_s r + as_s p_s for shifts not yet converged;
// p0 = r + a p0) in one pass over r, p0 and every (x_s, p_s).
constexpr int QPX_MAX_SHIFTS = 32;
struct MShiftArgs {
  int vh;
  int nshift;
  int x_only;          // 1: apply only the pending x update (after the last iteration)
  SpinorArg r, p0;
  SpinorArg x[QPX_MAX_SHIFTS], p[QPX_MAX_SHIFTS];
  SolverState *state;  // coefficients; its done flag stops the update unless x_only
};

template <typename P>
__global__ void __launch_bounds__(QPX_BLOCK) mshift_update_kernel(const MShiftArgs a)
{
  using T = typename P::real;
  using IO = SpinorIO<P>;
  const SolverState *st = a.state;
  if (!a.x_only && st->done) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.vh) return;
  T r[24];
  if (!a.x_only) IO::load(a.r, 0, s, r);
  for (int sh = 0; sh < a.nshift; sh++) {
    const T xc = (T)st->v[S_AUX6][sh];
    const bool pact = !a.x_only && !st->rhs_done[sh];
    if (xc == (T)0 && !pact) continue;
    T p[24];
    IO::load(a.p[sh], 0, s, p);
    if (xc != (T)0) {
      T x[24];
      IO::load(a.x[sh], 0, s, x);
#pragma unroll
      for (int k = 0; k < 24; k++) x[k] -= xc * p[k];
      IO::store(a.x[sh], 0, s, x);
    }
    if (pact) {
      const T z = (T)st->v[S_AUX0][sh], as = (T)st->v[S_AUX2][sh];
#pragma unroll
      for (int k = 0; k < 24; k++) p[k] = z * r[k] + as * p[k];
      IO::store(a.p[sh], 0, s, p);
    }
  }
  if (!a.x_only) {
    T p0[24];
    IO::load(a.p0, 0, s, p0);
    const T aa = (T)st->v[S_A][0];
#pragma unroll
    for (int k = 0; k < 24; k++) p0[k] = r[k] + aa * p0[k];
    IO::store(a.p0, 0, s, p0);
  }
}

// y (precision Q) = scale * x (precision P): the precision conversion of
// InvRichardsonMultiPrec (blas_new_c.h:852-960), scale = 1/|r| going down
// and |r| coming back up.  `scale` may be a per-rhs device value.
// accumulate = 1: y += scale * x (folds a low-precision solution increment
// into a high-precision solution).
template <typename P, typename Q>
__global__ void __launch_bounds__(QPX_BLOCK) convert_kernel(int vh, SpinorArg x, SpinorArg y, Coef scale,
                                                            SolverState *state, int accumulate)
{
  if (state && state->done) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  if (s >= vh) return;
  typename P::real xv[24];
  typename Q::real yv[24];
  SpinorIO<P>::load(x, rhs, s, xv);
  const double sc = scale.r(rhs);
  if (accumulate) {
    SpinorIO<Q>::load(y, rhs, s, yv);
#pragma unroll
    for (int k = 0; k < 24; k++) yv[k] = (typename Q::real)((double)yv[k] + (double)xv[k] * sc);
  } else {
#pragma unroll
    for (int k = 0; k < 24; k++) yv[k] = (typename Q::real)((double)xv[k] * sc);
  }
  SpinorIO<Q>::store(y, rhs, s, yv);
}

}  // namespace qpx
