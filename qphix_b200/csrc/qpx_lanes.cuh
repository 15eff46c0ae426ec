// Field access for kernels that process SP lattice sites per thread.
//
// SP = 1: one site, arithmetic in P::real (double or float).
// SP = 2: two sites (lanes), arithmetic in f2 = float2 whose .x holds the
//         value of site s[0] and .y the value of site s[1]; only for the
//         FP32-arithmetic precisions (F32 storage, F16 / BF16 / Q16 storage
//         with per-site norms).  Each lane's data is loaded with the same
//         coalesced per-site loads as the one-site path and converted
//         straight into its lane.
// A lane whose site lies past the end of the checkerboard is given a copy of
// lane 0's site index by the kernel (valid loads, identical arithmetic) and
// is skipped on store.
#pragma once

#include "qpx_common.cuh"

namespace qpx {

template <typename P, int SP>
struct Lanes;

template <typename P>
struct Lanes<P, 1> {
  using T = typename P::real;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, const int *s, T v[24], T &nrm)
  {
    SpinorIO<P>::load_raw(f, rhs, s[0], v, nrm);
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, const int *s, T v[24])
  {
    SpinorIO<P>::load(f, rhs, s[0], v);
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, const int *s, const bool *act,
                                               const T v[24])
  {
    (void)act;
    SpinorIO<P>::store(f, rhs, s[0], v);
  }
  template <int RECON>
  __device__ __forceinline__ static void load_link(const GaugeArg &g, int cb, int mu, const int *s, cx<T> u[3][3])
  {
    GaugeIO<P, RECON>::load(g, cb, mu, s[0], u);
  }
  template <int NR>
  __device__ __forceinline__ static void load_clover(const CloverArg &c, const int *s, int k0, int n, T *v)
  {
    CloverIO<P, NR>::load(c, s[0], k0, n, v);
  }
};

// ---- two lanes -------------------------------------------------------------
// element 0 / 1 of a word of two 16-bit values, as float
__device__ __forceinline__ float lo_f(uint32_t w, F16) { return __low2float(*reinterpret_cast<const __half2 *>(&w)); }
__device__ __forceinline__ float hi_f(uint32_t w, F16) { return __high2float(*reinterpret_cast<const __half2 *>(&w)); }
__device__ __forceinline__ float lo_f(uint32_t w, BF16) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float hi_f(uint32_t w, BF16) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ float lo_f(uint32_t w, Q16) { return q16_lo(w); }
__device__ __forceinline__ float hi_f(uint32_t w, Q16) { return q16_hi(w); }

// v[0] = (a.lo, b.lo), v[1] = (a.hi, b.hi): the same element of sites A and B
template <typename H>
__device__ __forceinline__ void lanes_from_words(uint32_t a, uint32_t b, f2 *v)
{
  v[0] = make_float2(lo_f(a, H()), lo_f(b, H()));
  v[1] = make_float2(hi_f(a, H()), hi_f(b, H()));
}

// S: spinor storage (F16, BF16, Q16); H: link and clover storage (F16, BF16)
template <typename S, typename H>
struct Lanes16 {
  using T = f2;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, const int *s, f2 v[24], f2 &nrm)
  {
    const uint4 *p = reinterpret_cast<const uint4 *>(f.data) + rhs * f.rhs_stride_chunks;
    nrm = make_float2(__ldg(f.norm + rhs * f.stride + s[0]), __ldg(f.norm + rhs * f.stride + s[1]));
#pragma unroll
    for (int k = 0; k < 3; k++) {
      uint4 da = __ldg(p + k * f.stride + s[0]);
      uint4 db = __ldg(p + k * f.stride + s[1]);
      lanes_from_words<S>(da.x, db.x, v + 8 * k);
      lanes_from_words<S>(da.y, db.y, v + 8 * k + 2);
      lanes_from_words<S>(da.z, db.z, v + 8 * k + 4);
      lanes_from_words<S>(da.w, db.w, v + 8 * k + 6);
    }
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, const int *s, f2 v[24])
  {
    f2 nrm;
    load_raw(f, rhs, s, v, nrm);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] = v[k] * nrm;
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, const int *s, const bool *act,
                                               const f2 v[24])
  {
    float ma = 0.f, mb = 0.f;
#pragma unroll
    for (int k = 0; k < 24; k++) {
      ma = fmaxf(ma, fabsf(v[k].x));
      mb = fmaxf(mb, fabsf(v[k].y));
    }
    const f2 inv = make_float2(ma > 0.f ? 1.0f / ma : 0.f, mb > 0.f ? 1.0f / mb : 0.f);
    f2 w[24];
#pragma unroll
    for (int k = 0; k < 24; k++) w[k] = v[k] * inv;
    uint4 *p = reinterpret_cast<uint4 *>(f.data) + rhs * f.rhs_stride_chunks;
#pragma unroll
    for (int l = 0; l < 2; l++) {
      if (!act[l]) continue;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        float q[8];
#pragma unroll
        for (int i = 0; i < 8; i++) q[i] = lane(w[8 * k + i], l);
        p[k * f.stride + s[l]] = pack8(q, S());
      }
      f.norm[rhs * f.stride + s[l]] = (l ? mb : ma) * site_norm_scale<S>();
    }
  }
  template <int RECON>
  __device__ __forceinline__ static void load_link(const GaugeArg &g, int cb, int mu, const int *s, cx<f2> u[3][3])
  {
    if (RECON == 12) {
      const uint2 *p = reinterpret_cast<const uint2 *>(g.data) + (cb * 4 + mu) * g.mu_stride;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        uint2 da = __ldg(p + k * g.stride + s[0]);
        uint2 db = __ldg(p + k * g.stride + s[1]);
        f2 t[4];
        lanes_from_words<H>(da.x, db.x, t);
        lanes_from_words<H>(da.y, db.y, t + 2);
        u[(2 * k) / 3][(2 * k) % 3] = {t[0], t[1]};
        u[(2 * k + 1) / 3][(2 * k + 1) % 3] = {t[2], t[3]};
      }
      recon12(u);
    } else {
      const uint32_t *p = reinterpret_cast<const uint32_t *>(g.data) + (cb * 4 + mu) * g.mu_stride;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        f2 t[2];
        lanes_from_words<H>(__ldg(p + k * g.stride + s[0]), __ldg(p + k * g.stride + s[1]), t);
        u[k / 3][k % 3] = {t[0], t[1]};
      }
    }
  }
  // reals [k0, k0 + n), k0 and n multiples of 4: every 16-byte chunk that
  // overlaps the range is loaded once and the needed halves converted
  template <int NR>
  __device__ __forceinline__ static void load_clover(const CloverArg &c, const int *s, int k0, int n, f2 *v)
  {
    const uint4 *p = reinterpret_cast<const uint4 *>(c.data);
#pragma unroll
    for (int q = (k0 / 8) * 8; q < k0 + n; q += 8) {
      uint4 da = __ldg(p + (q / 8) * c.stride + s[0]);
      uint4 db = __ldg(p + (q / 8) * c.stride + s[1]);
      if (q >= k0) {
        lanes_from_words<H>(da.x, db.x, v + (q - k0));
        lanes_from_words<H>(da.y, db.y, v + (q - k0) + 2);
      }
      if (q + 4 < k0 + n && q + 4 >= k0) {
        lanes_from_words<H>(da.z, db.z, v + (q + 4 - k0));
        lanes_from_words<H>(da.w, db.w, v + (q + 4 - k0) + 2);
      }
    }
  }
};

template <>
struct Lanes<F16, 2> : Lanes16<F16, F16> {};
template <>
struct Lanes<BF16, 2> : Lanes16<BF16, BF16> {};
template <>
struct Lanes<Q16, 2> : Lanes16<Q16, F16> {};

template <>
struct Lanes<F32, 2> {
  using T = f2;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, const int *s, f2 v[24], f2 &nrm)
  {
    load(f, rhs, s, v);
    nrm = make_float2(1.f, 1.f);
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, const int *s, f2 v[24])
  {
    const float4 *p = reinterpret_cast<const float4 *>(f.data) + rhs * f.rhs_stride_chunks;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      float4 a = __ldg(p + k * f.stride + s[0]);
      float4 b = __ldg(p + k * f.stride + s[1]);
      v[4 * k] = make_float2(a.x, b.x);
      v[4 * k + 1] = make_float2(a.y, b.y);
      v[4 * k + 2] = make_float2(a.z, b.z);
      v[4 * k + 3] = make_float2(a.w, b.w);
    }
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, const int *s, const bool *act,
                                               const f2 v[24])
  {
    float4 *p = reinterpret_cast<float4 *>(f.data) + rhs * f.rhs_stride_chunks;
#pragma unroll
    for (int l = 0; l < 2; l++) {
      if (!act[l]) continue;
#pragma unroll
      for (int k = 0; k < 6; k++)
        p[k * f.stride + s[l]] = make_float4(lane(v[4 * k], l), lane(v[4 * k + 1], l), lane(v[4 * k + 2], l),
                                             lane(v[4 * k + 3], l));
    }
  }
  template <int RECON>
  __device__ __forceinline__ static void load_link(const GaugeArg &g, int cb, int mu, const int *s, cx<f2> u[3][3])
  {
    if (RECON == 12) {
      const float4 *p = reinterpret_cast<const float4 *>(g.data) + (cb * 4 + mu) * g.mu_stride;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        float4 a = __ldg(p + k * g.stride + s[0]);
        float4 b = __ldg(p + k * g.stride + s[1]);
        u[(2 * k) / 3][(2 * k) % 3] = {make_float2(a.x, b.x), make_float2(a.y, b.y)};
        u[(2 * k + 1) / 3][(2 * k + 1) % 3] = {make_float2(a.z, b.z), make_float2(a.w, b.w)};
      }
      recon12(u);
    } else {
      const float2 *p = reinterpret_cast<const float2 *>(g.data) + (cb * 4 + mu) * g.mu_stride;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        float2 a = __ldg(p + k * g.stride + s[0]);
        float2 b = __ldg(p + k * g.stride + s[1]);
        u[k / 3][k % 3] = {make_float2(a.x, b.x), make_float2(a.y, b.y)};
      }
    }
  }
  // reals [k0, k0 + n), k0 and n multiples of 4
  template <int NR>
  __device__ __forceinline__ static void load_clover(const CloverArg &c, const int *s, int k0, int n, f2 *v)
  {
    const float4 *p = reinterpret_cast<const float4 *>(c.data);
#pragma unroll
    for (int q = 0; q < n; q += 4) {
      float4 a = __ldg(p + ((k0 + q) / 4) * c.stride + s[0]);
      float4 b = __ldg(p + ((k0 + q) / 4) * c.stride + s[1]);
      v[q] = make_float2(a.x, b.x);
      v[q + 1] = make_float2(a.y, b.y);
      v[q + 2] = make_float2(a.z, b.z);
      v[q + 3] = make_float2(a.w, b.w);
    }
  }
};

// ---- two right-hand sides in the lanes ---------------------------------------
// RhsLanes<P>: one lattice site per thread and two right-hand sides, rhs and
// rhs + 1, in the .x / .y lanes of f2, so the paired FP32 instructions do the
// arithmetic of both while every link and clover element is loaded,
// converted and (12-real) reconstructed once for the pair and broadcast to
// both lanes.  Both lanes are active or neither (`act` holds the site's
// flag twice).  For the FP32-arithmetic precisions only.
template <typename P>
struct RhsLanes {
  using T = f2;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, const int *s, f2 v[24], f2 &nrm)
  {
    float a[24], b[24], na, nb;
    SpinorIO<P>::load_raw(f, rhs, s[0], a, na);
    SpinorIO<P>::load_raw(f, rhs + 1, s[0], b, nb);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] = make_float2(a[k], b[k]);
    nrm = make_float2(na, nb);
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, const int *s, f2 v[24])
  {
    float a[24], b[24];
    SpinorIO<P>::load(f, rhs, s[0], a);
    SpinorIO<P>::load(f, rhs + 1, s[0], b);
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] = make_float2(a[k], b[k]);
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, const int *s, const bool *act,
                                               const f2 v[24])
  {
    if (!act[0]) return;
    float a[24], b[24];
#pragma unroll
    for (int k = 0; k < 24; k++) {
      a[k] = v[k].x;
      b[k] = v[k].y;
    }
    SpinorIO<P>::store(f, rhs, s[0], a);
    SpinorIO<P>::store(f, rhs + 1, s[0], b);
  }
  template <int RECON>
  __device__ __forceinline__ static void load_link(const GaugeArg &g, int cb, int mu, const int *s, cx<f2> u[3][3])
  {
    cx<float> w[3][3];
    GaugeIO<P, RECON>::load(g, cb, mu, s[0], w);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) u[i][j] = {make_float2(w[i][j].re, w[i][j].re), make_float2(w[i][j].im, w[i][j].im)};
  }
  template <int NR>
  __device__ __forceinline__ static void load_clover(const CloverArg &c, const int *s, int k0, int n, f2 *v)
  {
    float w[144];
    CloverIO<P, NR>::load(c, s[0], k0, n, w);
#pragma unroll
    for (int k = 0; k < n; k++) v[k] = make_float2(w[k], w[k]);
  }
};

// Q16 spinors, FP32 links and clover terms
template <>
struct Lanes<Q16F32, 2> {
  using T = f2;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, const int *s, f2 v[24], f2 &nrm)
  {
    Lanes16<Q16, F16>::load_raw(f, rhs, s, v, nrm);
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, const int *s, f2 v[24])
  {
    Lanes16<Q16, F16>::load(f, rhs, s, v);
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, const int *s, const bool *act,
                                               const f2 v[24])
  {
    Lanes16<Q16, F16>::store(f, rhs, s, act, v);
  }
  template <int RECON>
  __device__ __forceinline__ static void load_link(const GaugeArg &g, int cb, int mu, const int *s, cx<f2> u[3][3])
  {
    Lanes<F32, 2>::load_link<RECON>(g, cb, mu, s, u);
  }
  template <int NR>
  __device__ __forceinline__ static void load_clover(const CloverArg &c, const int *s, int k0, int n, f2 *v)
  {
    Lanes<F32, 2>::load_clover<NR>(c, s, k0, n, v);
  }
};

}  // namespace qpx
