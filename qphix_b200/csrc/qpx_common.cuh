// Device-side building blocks shared by every kernel of the library:
// precision traits, the chunked structure-of-arrays field layouts in HBM,
// complex helpers and the lattice geometry passed to kernels.
//
// Layouts (one checkerboard of Vh sites, `stride` >= Vh, a multiple of 64):
//   spinor  [rhs][chunk][stride] of Chunk, 24 reals per site ordered
//           (spin, colour, re/im); FP64 12 x double2, FP32 6 x float4,
//           half / bf16 3 x 16-byte chunks (8 values) + float norm[rhs][stride]
//   gauge   [cb][mu][chunk][stride]: U_mu(x) for x in cb, row-major (row, col,
//           re/im); 18 reals, or 12 (rows 0 and 1; row 2 = conj(row0 x row1))
//   clover  [chunk][stride], 72 reals = 2 blocks x (diag[6], offd[15] re/im)
//   full    [chunk][stride], 144 reals = 2 blocks x 6 x 6 complex, row-major
// A warp therefore reads 32 consecutive sites x 16 (or 8) bytes per chunk.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <type_traits>

namespace qpx {

// ---------------------------------------------------------------------------
// Programmatic dependent launch (sm_90 and later).  The Dslash, BLAS and fold
// kernels of a solver iteration are launched with the programmatic stream
// serialisation attribute (launch_pdl): each may be scheduled while its
// predecessor on the stream is still finishing its last blocks, instead of
// after it has drained.  pdl_wait() blocks until the predecessor grid has
// completed and its writes are visible, and comes before the kernel reads
// anything its predecessors wrote; pdl_trigger() lets the successor start
// launching.  For a kernel launched without the attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// The attribute pays off where a launch's predecessor ends in a partial last
// wave of many blocks (measured on B200: the 16^3x32, 8-rhs solve runs 2 %
// faster with it); behind small launches (an 8^4 lattice's 16-block grids)
// the dependent wait costs more than the ordinary launch boundary (8^4 CG
// 10 % slower), so launches of fewer than kPdlMinBlocks blocks, and folds of
// fewer partials, go the ordinary way.  QPHIX_GPU_PDL=0 turns it off.
constexpr int kPdlMinBlocks = 296;
inline bool pdl_enabled()
{
  static const bool on = [] {
    const char *e = std::getenv("QPHIX_GPU_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}
// set while the autotuner times launch shapes: its back-to-back timed
// launches must not overlap one another
inline bool &pdl_suspended()
{
  static thread_local bool off = false;
  return off;
}

// `size`: the block count that decides whether the attribute is set
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, long long size,
                       Args &&...args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (pdl_enabled() && !pdl_suspended() && size >= kPdlMinBlocks) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

enum Prec : int { PREC_F64 = 0, PREC_F32 = 1, PREC_F16 = 2, PREC_BF16 = 3, PREC_Q16 = 4, PREC_Q16F32 = 5 };

// ---------------------------------------------------------------------------
// complex arithmetic on plain structs (kept in registers)
// ---------------------------------------------------------------------------
template <typename T>
struct cx {
  T re, im;
};

template <typename T>
__device__ __forceinline__ cx<T> cmake(T r, T i) { return cx<T>{r, i}; }
template <typename T>
__device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
__device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T>
__device__ __forceinline__ cx<T> operator*(cx<T> a, cx<T> b)
{
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__device__ __forceinline__ cx<T> operator*(T s, cx<T> a) { return {s * a.re, s * a.im}; }
template <typename T>
__device__ __forceinline__ cx<T> conj(cx<T> a) { return {a.re, -a.im}; }
// conj(a) * b
template <typename T>
__device__ __forceinline__ cx<T> cmulc(cx<T> a, cx<T> b)
{
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
// i * a
template <typename T>
__device__ __forceinline__ cx<T> itimes(cx<T> a) { return {-a.im, a.re}; }

// ---------------------------------------------------------------------------
// Two sites per thread: the lanes of a float2 hold the same component of two
// lattice sites, so that Blackwell's paired FP32 instructions (FADD2, FMUL2,
// FFMA2; IEEE round-to-nearest per lane, like their scalar forms) do the
// work of two scalar instructions.  Every operation below is lane-wise.
// ---------------------------------------------------------------------------
using f2 = float2;
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 operator-(f2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ f2 operator*(f2 a, f2 b) { return __fmul2_rn(a, b); }

// fused multiply-add c + a b for every arithmetic type
__device__ __forceinline__ double mad(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float mad(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ f2 mad(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }

// a scalar broadcast to the arithmetic type (both lanes for f2)
template <typename T>
__device__ __forceinline__ T splat(double v) { return (T)v; }
template <>
__device__ __forceinline__ f2 splat<f2>(double v) { return make_float2((float)v, (float)v); }

// lane l of a value (l = 0 for scalar types)
__device__ __forceinline__ double lane(double v, int) { return v; }
__device__ __forceinline__ float lane(float v, int) { return v; }
__device__ __forceinline__ float lane(f2 v, int l) { return l ? v.y : v.x; }

// ---- per-thread terms of the fused reductions ------------------------------
// A thread sums the products of its own spinor elements in its arithmetic
// type -- FP32 (float or float2 lanes) for 16-bit and FP32 storage, FP64 for
// FP64 storage -- and converts each value to FP64 once; everything after
// that (warps, blocks, the fold over blocks) adds in FP64.  Converting every
// element instead costs two float -> double conversions per product on the
// slow conversion pipe.  The FP64 forms are the plain element loops.
// `act` masks the lanes of a two-site thread whose second site is past the
// end of the lattice.
__device__ __forceinline__ double red_total(float v, const bool *) { return (double)v; }
__device__ __forceinline__ double red_total(f2 v, const bool *act)
{
  return (act[0] ? (double)v.x : 0.0) + (act[1] ? (double)v.y : 0.0);
}

// sum |x_k|^2 over the 24 reals of a thread's site(s)
template <typename T>
__device__ __forceinline__ double red_norm(const T *x, const bool *act)
{
  if constexpr (std::is_same<T, double>::value) {
    double n = 0;
#pragma unroll
    for (int k = 0; k < 24; k++) n += x[k] * x[k];
    return n;
  } else {
    T n = splat<T>(0.0);
#pragma unroll
    for (int k = 0; k < 24; k++) n = mad(x[k], x[k], n);
    return red_total(n, act);
  }
}

// <x, y> = sum conj(x) y over the 12 complex elements of a thread's site(s)
template <typename T>
__device__ __forceinline__ void red_dot(const T *x, const T *y, const bool *act, double &re, double &im)
{
  if constexpr (std::is_same<T, double>::value) {
    double dre = 0, dim = 0;
#pragma unroll
    for (int k = 0; k < 24; k += 2) {
      dre += x[k] * y[k] + x[k + 1] * y[k + 1];
      dim += x[k] * y[k + 1] - x[k + 1] * y[k];
    }
    re = dre;
    im = dim;
  } else {
    T dre = splat<T>(0.0), dim = splat<T>(0.0);
#pragma unroll
    for (int k = 0; k < 24; k += 2) {
      dre = mad(x[k], y[k], mad(x[k + 1], y[k + 1], dre));
      dim = mad(x[k], y[k + 1], mad(-x[k + 1], y[k], dim));
    }
    re = red_total(dre, act);
    im = red_total(dim, act);
  }
}

// complex products with explicit fused multiply-adds
// c + a b
template <typename T>
__device__ __forceinline__ cx<T> cmad(cx<T> a, cx<T> b, cx<T> c)
{
  return {mad(a.re, b.re, mad(-a.im, b.im, c.re)), mad(a.re, b.im, mad(a.im, b.re, c.im))};
}
// c + conj(a) b
template <typename T>
__device__ __forceinline__ cx<T> cmadc(cx<T> a, cx<T> b, cx<T> c)
{
  return {mad(a.re, b.re, mad(a.im, b.im, c.re)), mad(a.re, b.im, mad(-a.im, b.re, c.im))};
}
// a b
template <typename T>
__device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b)
{
  return {mad(a.re, b.re, -(a.im * b.im)), mad(a.re, b.im, a.im * b.re)};
}
// conj(a) b
template <typename T>
__device__ __forceinline__ cx<T> cmulcf(cx<T> a, cx<T> b)
{
  return {mad(a.re, b.re, a.im * b.im), mad(a.re, b.im, -(a.im * b.re))};
}
// real s times complex a
template <typename T>
__device__ __forceinline__ cx<T> rmul(T s, cx<T> a) { return {s * a.re, s * a.im}; }

// ---------------------------------------------------------------------------
// precision traits
// ---------------------------------------------------------------------------
struct F64 {
  using real = double;       // arithmetic type
  static constexpr int prec = PREC_F64;
  static constexpr bool has_norm = false;
};
struct F32 {
  using real = float;
  static constexpr int prec = PREC_F32;
  static constexpr bool has_norm = false;
};
struct F16 {
  using real = float;
  static constexpr int prec = PREC_F16;
  static constexpr bool has_norm = true;
};
struct BF16 {
  using real = float;
  static constexpr int prec = PREC_BF16;
  static constexpr bool has_norm = true;
};
// 16-bit fixed-point spinors with a per-site scale (links and clover terms
// stay FP16): a spinor value is q * norm with q an integer in [-32767, 32767]
// and norm = (max |value| of the site) / 32767, so every component is held to
// 1/65534 of the site's largest one (FP16: ~1/4096)
struct Q16 {
  using real = float;
  static constexpr int prec = PREC_Q16;
  static constexpr bool has_norm = true;
};
// Q16 spinors with FP32 links and clover terms: the operator at FP32
// accuracy, the Krylov vectors at 16 bits (for many right-hand sides, whose
// spinor traffic outweighs the shared links and clover terms)
struct Q16F32 {
  using real = float;
  static constexpr int prec = PREC_Q16F32;
  static constexpr bool has_norm = true;
};

// the per-site norm stored for a site whose largest |value| is m
template <typename H>
__host__ __device__ constexpr float site_norm_scale() { return 1.0f; }
template <>
__host__ __device__ constexpr float site_norm_scale<Q16>() { return 1.0f / 32767.0f; }

// Q16 words hold u = q + 32768 in each 16-bit half.  As the low 16 mantissa
// bits of a float with exponent 2^23 they give 2^23 + u exactly, so one byte
// permute and one subtraction recover q as a float (and one fused
// multiply-add plus a byte permute store it).
constexpr float QPX_Q16_BIAS = 8421376.0f;  // 2^23 + 32768
__device__ __forceinline__ float q16_lo(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B00u, 0x5410)) - QPX_Q16_BIAS; }
__device__ __forceinline__ float q16_hi(uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B00u, 0x5432)) - QPX_Q16_BIAS; }
// a and b in [-1, 1] (already divided by the site's max): the word of
// round(32767 a), round(32767 b) (round to nearest even)
__device__ __forceinline__ uint32_t q16_pack(float a, float b)
{
  const uint32_t ua = __float_as_uint(fmaf(a, 32767.0f, QPX_Q16_BIAS));
  const uint32_t ub = __float_as_uint(fmaf(b, 32767.0f, QPX_Q16_BIAS));
  return __byte_perm(ua, ub, 0x5410);
}

// 16-bit conversions --------------------------------------------------------
__device__ __forceinline__ void unpack8(const uint4 &v, float out[8], Q16)
{
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    out[2 * i] = q16_lo(w[i]);
    out[2 * i + 1] = q16_hi(w[i]);
  }
}
__device__ __forceinline__ uint4 pack8(const float in[8], Q16)
{
  return make_uint4(q16_pack(in[0], in[1]), q16_pack(in[2], in[3]), q16_pack(in[4], in[5]), q16_pack(in[6], in[7]));
}
__device__ __forceinline__ void unpack8(const uint4 &v, float out[8], F16)
{
  const __half2 *h = reinterpret_cast<const __half2 *>(&v);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float2 f = __half22float2(h[i]);
    out[2 * i] = f.x;
    out[2 * i + 1] = f.y;
  }
}
__device__ __forceinline__ void unpack8(const uint4 &v, float out[8], BF16)
{
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float2 f = __bfloat1622float2(h[i]);
    out[2 * i] = f.x;
    out[2 * i + 1] = f.y;
  }
}
__device__ __forceinline__ uint4 pack8(const float in[8], F16)
{
  uint4 v;
  __half2 *h = reinterpret_cast<__half2 *>(&v);
#pragma unroll
  for (int i = 0; i < 4; i++) h[i] = __floats2half2_rn(in[2 * i], in[2 * i + 1]);
  return v;
}
__device__ __forceinline__ uint4 pack8(const float in[8], BF16)
{
  uint4 v;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v);
#pragma unroll
  for (int i = 0; i < 4; i++) h[i] = __floats2bfloat162_rn(in[2 * i], in[2 * i + 1]);
  return v;
}
__device__ __forceinline__ void unpack4(const uint2 &v, float out[4], F16)
{
  const __half2 *h = reinterpret_cast<const __half2 *>(&v);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    float2 f = __half22float2(h[i]);
    out[2 * i] = f.x;
    out[2 * i + 1] = f.y;
  }
}
__device__ __forceinline__ void unpack4(const uint2 &v, float out[4], BF16)
{
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    float2 f = __bfloat1622float2(h[i]);
    out[2 * i] = f.x;
    out[2 * i + 1] = f.y;
  }
}
__device__ __forceinline__ uint2 pack4(const float in[4], F16)
{
  uint2 v;
  __half2 *h = reinterpret_cast<__half2 *>(&v);
  h[0] = __floats2half2_rn(in[0], in[1]);
  h[1] = __floats2half2_rn(in[2], in[3]);
  return v;
}
__device__ __forceinline__ uint2 pack4(const float in[4], BF16)
{
  uint2 v;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&v);
  h[0] = __floats2bfloat162_rn(in[0], in[1]);
  h[1] = __floats2bfloat162_rn(in[2], in[3]);
  return v;
}
__device__ __forceinline__ void unpack2(const uint32_t &v, float out[2], F16)
{
  float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&v));
  out[0] = f.x;
  out[1] = f.y;
}
__device__ __forceinline__ void unpack2(const uint32_t &v, float out[2], BF16)
{
  float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v));
  out[0] = f.x;
  out[1] = f.y;
}
__device__ __forceinline__ uint32_t pack2(const float in[2], F16)
{
  __half2 h = __floats2half2_rn(in[0], in[1]);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t pack2(const float in[2], BF16)
{
  __nv_bfloat162 h = __floats2bfloat162_rn(in[0], in[1]);
  return *reinterpret_cast<uint32_t *>(&h);
}

// ---------------------------------------------------------------------------
// spinor fields
// ---------------------------------------------------------------------------
struct SpinorArg {
  void *data;         // chunk array
  float *norm;        // per-site norm (16-bit storage only)
  long long stride;   // sites per chunk row
  long long rhs_stride_chunks;  // chunk rows per right-hand side (= nchunk * stride)
};

template <typename P>
struct SpinorIO;

// load_raw(f, rhs, s, v, nrm): the stored values and the per-site scale
// separately (v * nrm are the spinor's components); nrm == 1 without a norm.
template <>
struct SpinorIO<F64> {
  static constexpr int nchunk = 12;
  static constexpr size_t chunk_bytes = 16;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, long long s, double v[24], double &nrm)
  {
    load(f, rhs, s, v);
    nrm = 1.0;
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, long long s, double v[24])
  {
    const double2 *p = reinterpret_cast<const double2 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 d = __ldg(p + k * f.stride);
      v[2 * k] = d.x;
      v[2 * k + 1] = d.y;
    }
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, long long s, const double v[24])
  {
    double2 *p = reinterpret_cast<double2 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 12; k++) p[k * f.stride] = make_double2(v[2 * k], v[2 * k + 1]);
  }
};

template <>
struct SpinorIO<F32> {
  static constexpr int nchunk = 6;
  static constexpr size_t chunk_bytes = 16;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, long long s, float v[24], float &nrm)
  {
    load(f, rhs, s, v);
    nrm = 1.0f;
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, long long s, float v[24])
  {
    const float4 *p = reinterpret_cast<const float4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      float4 d = __ldg(p + k * f.stride);
      v[4 * k] = d.x;
      v[4 * k + 1] = d.y;
      v[4 * k + 2] = d.z;
      v[4 * k + 3] = d.w;
    }
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, long long s, const float v[24])
  {
    float4 *p = reinterpret_cast<float4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 6; k++) p[k * f.stride] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
  }
};

// 16-bit storage with a per-site scale: stored = value / norm, |stored| <= 1
template <typename H>
struct SpinorIO16 {
  static constexpr int nchunk = 3;
  static constexpr size_t chunk_bytes = 16;
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, long long s, float v[24], float &nrm)
  {
    const uint4 *p = reinterpret_cast<const uint4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
    nrm = __ldg(f.norm + rhs * f.stride + s);
#pragma unroll
    for (int k = 0; k < 3; k++) unpack8(__ldg(p + k * f.stride), v + 8 * k, H());
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, long long s, float v[24])
  {
    const uint4 *p = reinterpret_cast<const uint4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
    float nrm = __ldg(f.norm + rhs * f.stride + s);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      uint4 d = __ldg(p + k * f.stride);
      unpack8(d, v + 8 * k, H());
    }
#pragma unroll
    for (int k = 0; k < 24; k++) v[k] *= nrm;
  }
  __device__ __forceinline__ static void store(const SpinorArg &f, int rhs, long long s, const float v[24])
  {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 24; k++) m = fmaxf(m, fabsf(v[k]));
    float inv = (m > 0.f) ? 1.0f / m : 0.f;
    float w[24];
#pragma unroll
    for (int k = 0; k < 24; k++) w[k] = v[k] * inv;
    uint4 *p = reinterpret_cast<uint4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 3; k++) p[k * f.stride] = pack8(w + 8 * k, H());
    f.norm[rhs * f.stride + s] = m * site_norm_scale<H>();
  }
};
template <>
struct SpinorIO<F16> : SpinorIO16<F16> {};
template <>
struct SpinorIO<BF16> : SpinorIO16<BF16> {};
template <>
struct SpinorIO<Q16> : SpinorIO16<Q16> {};
template <>
struct SpinorIO<Q16F32> : SpinorIO16<Q16> {};

// ---------------------------------------------------------------------------
// gauge links
// ---------------------------------------------------------------------------
struct GaugeArg {
  const void *data;
  long long stride;     // sites per chunk row
  long long mu_stride;  // chunk rows per (cb, mu) = nchunk * stride
};

// reconstruct row 2 = conj(row0 x row1)
template <typename T>
__device__ __forceinline__ void recon12(cx<T> u[3][3])
{
  // a b - c d with fused products: cmad(-c, d, a b)
  const cx<T> n02 = {-u[0][2].re, -u[0][2].im}, n00 = {-u[0][0].re, -u[0][0].im}, n01 = {-u[0][1].re, -u[0][1].im};
  u[2][0] = conj(cmad(n02, u[1][1], cmul(u[0][1], u[1][2])));
  u[2][1] = conj(cmad(n00, u[1][2], cmul(u[0][2], u[1][0])));
  u[2][2] = conj(cmad(n01, u[1][0], cmul(u[0][0], u[1][1])));
}

template <typename P, int RECON>
struct GaugeIO;

template <>
struct GaugeIO<F64, 18> {
  static constexpr int nchunk = 9;
  static constexpr size_t chunk_bytes = 16;
  __device__ __forceinline__ static void load(const GaugeArg &g, int cb, int mu, long long s, cx<double> u[3][3])
  {
    const double2 *p = reinterpret_cast<const double2 *>(g.data) + (cb * 4 + mu) * g.mu_stride + s;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 d = __ldg(p + k * g.stride);
      u[k / 3][k % 3] = {d.x, d.y};
    }
  }
};
template <>
struct GaugeIO<F64, 12> {
  static constexpr int nchunk = 6;
  static constexpr size_t chunk_bytes = 16;
  __device__ __forceinline__ static void load(const GaugeArg &g, int cb, int mu, long long s, cx<double> u[3][3])
  {
    const double2 *p = reinterpret_cast<const double2 *>(g.data) + (cb * 4 + mu) * g.mu_stride + s;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      double2 d = __ldg(p + k * g.stride);
      u[k / 3][k % 3] = {d.x, d.y};
    }
    recon12(u);
  }
};
template <>
struct GaugeIO<F32, 18> {
  static constexpr int nchunk = 9;
  static constexpr size_t chunk_bytes = 8;
  __device__ __forceinline__ static void load(const GaugeArg &g, int cb, int mu, long long s, cx<float> u[3][3])
  {
    const float2 *p = reinterpret_cast<const float2 *>(g.data) + (cb * 4 + mu) * g.mu_stride + s;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float2 d = __ldg(p + k * g.stride);
      u[k / 3][k % 3] = {d.x, d.y};
    }
  }
};
template <>
struct GaugeIO<F32, 12> {
  static constexpr int nchunk = 3;
  static constexpr size_t chunk_bytes = 16;
  __device__ __forceinline__ static void load(const GaugeArg &g, int cb, int mu, long long s, cx<float> u[3][3])
  {
    const float4 *p = reinterpret_cast<const float4 *>(g.data) + (cb * 4 + mu) * g.mu_stride + s;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float4 d = __ldg(p + k * g.stride);
      u[(2 * k) / 3][(2 * k) % 3] = {d.x, d.y};
      u[(2 * k + 1) / 3][(2 * k + 1) % 3] = {d.z, d.w};
    }
    recon12(u);
  }
};
template <typename H>
struct GaugeIO16_18 {
  static constexpr int nchunk = 9;
  static constexpr size_t chunk_bytes = 4;
  __device__ __forceinline__ static void load(const GaugeArg &g, int cb, int mu, long long s, cx<float> u[3][3])
  {
    const uint32_t *p = reinterpret_cast<const uint32_t *>(g.data) + (cb * 4 + mu) * g.mu_stride + s;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float f[2];
      unpack2(__ldg(p + k * g.stride), f, H());
      u[k / 3][k % 3] = {f[0], f[1]};
    }
  }
};
template <typename H>
struct GaugeIO16_12 {
  static constexpr int nchunk = 3;
  static constexpr size_t chunk_bytes = 8;
  __device__ __forceinline__ static void load(const GaugeArg &g, int cb, int mu, long long s, cx<float> u[3][3])
  {
    const uint2 *p = reinterpret_cast<const uint2 *>(g.data) + (cb * 4 + mu) * g.mu_stride + s;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      float f[4];
      unpack4(__ldg(p + k * g.stride), f, H());
      u[(2 * k) / 3][(2 * k) % 3] = {f[0], f[1]};
      u[(2 * k + 1) / 3][(2 * k + 1) % 3] = {f[2], f[3]};
    }
    recon12(u);
  }
};
template <>
struct GaugeIO<F16, 18> : GaugeIO16_18<F16> {};
template <>
struct GaugeIO<F16, 12> : GaugeIO16_12<F16> {};
template <>
struct GaugeIO<BF16, 18> : GaugeIO16_18<BF16> {};
template <>
struct GaugeIO<BF16, 12> : GaugeIO16_12<BF16> {};
// Q16 keeps links (and clover terms) in FP16
template <>
struct GaugeIO<Q16, 18> : GaugeIO16_18<F16> {};
template <>
struct GaugeIO<Q16, 12> : GaugeIO16_12<F16> {};
template <int RECON>
struct GaugeIO<Q16F32, RECON> : GaugeIO<F32, RECON> {};

// ---------------------------------------------------------------------------
// clover fields (NR = 72 packed Hermitian, NR = 144 full blocks)
// ---------------------------------------------------------------------------
struct CloverArg {
  const void *data;
  long long stride;
};

template <typename P, int NR>
struct CloverIO;

template <int NR>
struct CloverIO<F64, NR> {
  static constexpr int nchunk = NR / 2;
  static constexpr size_t chunk_bytes = 16;
  // load reals [k0, k0+n) (n even, k0 even)
  __device__ __forceinline__ static void load(const CloverArg &c, long long s, int k0, int n, double *v)
  {
    const double2 *p = reinterpret_cast<const double2 *>(c.data) + s;
    for (int k = 0; k < n; k += 2) {
      double2 d = __ldg(p + ((k0 + k) / 2) * c.stride);
      v[k] = d.x;
      v[k + 1] = d.y;
    }
  }
};
template <int NR>
struct CloverIO<F32, NR> {
  static constexpr int nchunk = NR / 4;
  static constexpr size_t chunk_bytes = 16;
  // k0, n multiples of 4
  __device__ __forceinline__ static void load(const CloverArg &c, long long s, int k0, int n, float *v)
  {
    const float4 *p = reinterpret_cast<const float4 *>(c.data) + s;
    for (int k = 0; k < n; k += 4) {
      float4 d = __ldg(p + ((k0 + k) / 4) * c.stride);
      v[k] = d.x;
      v[k + 1] = d.y;
      v[k + 2] = d.z;
      v[k + 3] = d.w;
    }
  }
};
template <typename H, int NR>
struct CloverIO16 {
  static constexpr int nchunk = NR / 8;
  static constexpr size_t chunk_bytes = 16;
  // k0, n multiples of 4: every 16-byte chunk overlapping [k0, k0 + n) is
  // loaded once and the needed halves unpacked
  __device__ __forceinline__ static void load(const CloverArg &c, long long s, int k0, int n, float *v)
  {
    const uint4 *p = reinterpret_cast<const uint4 *>(c.data) + s;
#pragma unroll
    for (int q = (k0 / 8) * 8; q < k0 + n; q += 8) {
      uint4 d = __ldg(p + (q / 8) * c.stride);
      if (q >= k0) unpack4(make_uint2(d.x, d.y), v + (q - k0), H());
      if (q + 4 < k0 + n && q + 4 >= k0) unpack4(make_uint2(d.z, d.w), v + (q + 4 - k0), H());
    }
  }
};
template <int NR>
struct CloverIO<F16, NR> : CloverIO16<F16, NR> {};
template <int NR>
struct CloverIO<BF16, NR> : CloverIO16<BF16, NR> {};
template <int NR>
struct CloverIO<Q16, NR> : CloverIO16<F16, NR> {};
template <int NR>
struct CloverIO<Q16F32, NR> : CloverIO<F32, NR> {};

// Coherent<P>: precision P with its spinor loads taken through L2
// (ld.global.cg) instead of the read-only non-coherent path, for kernels that
// read spinors written earlier in the same launch (the persistent solver
// kernels, across their grid barriers).  Links and clover terms stay
// read-only for a whole solve and keep P's loads.
template <typename P>
struct Coherent : P {};
template <typename P, int RECON>
struct GaugeIO<Coherent<P>, RECON> : GaugeIO<P, RECON> {};
template <typename P, int NR>
struct CloverIO<Coherent<P>, NR> : CloverIO<P, NR> {};

template <>
struct SpinorIO<Coherent<F64>> : SpinorIO<F64> {
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, long long s, double v[24], double &nrm)
  {
    load(f, rhs, s, v);
    nrm = 1.0;
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, long long s, double v[24])
  {
    const double2 *p = reinterpret_cast<const double2 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 d = __ldcg(p + k * f.stride);
      v[2 * k] = d.x;
      v[2 * k + 1] = d.y;
    }
  }
};

template <>
struct SpinorIO<Coherent<F32>> : SpinorIO<F32> {
  __device__ __forceinline__ static void load_raw(const SpinorArg &f, int rhs, long long s, float v[24], float &nrm)
  {
    load(f, rhs, s, v);
    nrm = 1.0f;
  }
  __device__ __forceinline__ static void load(const SpinorArg &f, int rhs, long long s, float v[24])
  {
    const float4 *p = reinterpret_cast<const float4 *>(f.data) + rhs * f.rhs_stride_chunks + s;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      float4 d = __ldcg(p + k * f.stride);
      v[4 * k] = d.x;
      v[4 * k + 1] = d.y;
      v[4 * k + 2] = d.z;
      v[4 * k + 3] = d.w;
    }
  }
};

// ---------------------------------------------------------------------------
// lattice geometry as seen by a kernel
// ---------------------------------------------------------------------------
// Division by a divisor fixed at launch, as a multiply-high, an add and a
// shift (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, section 4): for 1 <= d < 2^31 and
// 0 <= n < 2^31, with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1
// (m < 2^32), n / d = (umulhi(m, n) + n) >> l, and the sum stays below 2^32.
// A run-time integer division costs a few tens of instructions instead.
struct DivU {
  uint32_t m;
  int l;
};
inline DivU make_divu(int d)
{
  int l = 0;
  while ((1ull << l) < (unsigned long long)d) l++;
  const unsigned long long m =
      ((1ull << 32) * ((1ull << l) - (unsigned long long)d)) / (unsigned long long)d + 1;
  return DivU{(uint32_t)m, l};
}
__device__ __forceinline__ int div_by(int n, DivU d)
{
  return (int)((__umulhi(d.m, (uint32_t)n) + (uint32_t)n) >> d.l);
}

struct Geom {
  int nx, ny, nz, nt, nxh;
  int vh;
  DivU div_nxh, div_ny, div_nz;  // make_divu of nxh, ny, nz
};

__device__ __forceinline__ void site_coords(const Geom &g, int s, int cb, int &xh, int &y, int &z,
                                            int &t, int &par)
{
  const int r = div_by(s, g.div_nxh);
  xh = s - r * g.nxh;
  const int r2 = div_by(r, g.div_ny);
  y = r - r2 * g.ny;
  t = div_by(r2, g.div_nz);
  z = r2 - t * g.nz;
  par = (y + z + t + cb) & 1;  // x = 2 xh + par
}

}  // namespace qpx
