// Host-layout <-> device-layout conversion kernels.  A host array is copied
// as-is into a device staging buffer; these kernels gather it into (or
// scatter it out of) the chunked device layout, converting precision and
// rebuilding the third row / column of compressed links.  Two host layouts
// are understood:
//   canonical  site-major FP64 (spinor [rhs][Vh][4][3][2], gauge
//              [2][4][Vh][3][3][2], clover [Vh][72], full clover [Vh][144])
//   qphix      the reference's blocked SoA host layout
//              (include/qphix_codegen/decl_common.h:9-62, geometry.h:156-175,
//               qdp_packer_parscalar.h:51-129,150-230,232-328)
//   qdp        QDP++ CB2 full-lattice arrays (site = cb Vh + cb index, the
//              order qdp_packer_parscalar.h:94-110 reads); spinor and clover
//              halves of one checkerboard arrive compacted in the staging
//              buffer ([rhs][Vh][24], [Vh][72]), gauge arrays whole
//              [4][2][Vh][18]; clover sites in Chroma's triangle order
//              (diag[2][6], offd[2][15][2])
#pragma once

#include "qpx_common.cuh"

namespace qpx {

enum HostKind : int { HOST_CANONICAL = 0, HOST_QPHIX = 1, HOST_QDP = 2 };
enum HostFT : int { HFT_F64 = 0, HFT_F32 = 1, HFT_F16 = 2 };

struct HostLayout {
  int kind;
  int ft;
  int V, S, c12;
  int nvecs, ngy, pxy, pxyz;
  int cb;  // qdp: checkerboard of the full-lattice spinor / clover array
};

// qdp clover: offset within a site of canonical value k (block b = k / 36:
// diag[6] then offd[15][2]) in Chroma's PrimitiveClovTriang order
__host__ __device__ __forceinline__ int qdp_clover_off(int k)
{
  int b = k / 36, j = k % 36;
  return j < 6 ? b * 6 + j : 12 + b * 30 + (j - 6);
}

__device__ __forceinline__ double host_read(const void *p, long long off, int ft)
{
  if (ft == HFT_F64) return reinterpret_cast<const double *>(p)[off];
  if (ft == HFT_F32) return (double)reinterpret_cast<const float *>(p)[off];
  return (double)__half2float(reinterpret_cast<const __half *>(p)[off]);
}
__device__ __forceinline__ void host_write(void *p, long long off, int ft, double v)
{
  if (ft == HFT_F64)
    reinterpret_cast<double *>(p)[off] = v;
  else if (ft == HFT_F32)
    reinterpret_cast<float *>(p)[off] = (float)v;
  else
    reinterpret_cast<__half *>(p)[off] = __float2half((float)v);
}

// offset of spinor real k = (spin*3 + col)*2 + ri of cb-site s, rhs
__device__ __forceinline__ long long host_spinor_off(const HostLayout &L, const Geom &g, int rhs, int s,
                                                     int k)
{
  if (L.kind != HOST_QPHIX) return ((long long)rhs * g.vh + s) * 24 + k;  // canonical / compacted qdp
  int xh = s % g.nxh, r = s / g.nxh;
  int y = r % g.ny;
  r /= g.ny;
  int z = r % g.nz, t = r / g.nz;
  long long blk = (long long)t * L.pxyz + (long long)z * L.pxy + (long long)y * L.nvecs + xh / L.S;
  int lane = xh % L.S;
  int spin = k / 6, col = (k / 2) % 3, ri = k & 1;
  long long per_rhs = (long long)L.pxyz * g.nt * 24 * L.S;
  return rhs * per_rhs + blk * 24 * L.S + ((col * 4 + spin) * 2 + ri) * L.S + lane;
}

// block / lane of a gauge- or clover-type QPhiX array for cb-site s
__device__ __forceinline__ void host_gblock(const HostLayout &L, const Geom &g, int s, long long &blk,
                                            int &lane)
{
  int xh = s % g.nxh, r = s / g.nxh;
  int y = r % g.ny;
  r /= g.ny;
  int z = r % g.nz, t = r / g.nz;
  blk = ((long long)t * L.pxyz + (long long)z * L.pxy) / L.ngy + (long long)(y / L.ngy) * L.nvecs + xh / L.S;
  lane = (y % L.ngy) * L.S + xh % L.S;
}

// ---------------------------------------------------------------------------
template <typename P>
__global__ void spinor_in_kernel(Geom g, HostLayout L, const void *host, SpinorArg f, int nrhs)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  if (s >= g.vh || rhs >= nrhs) return;
  typename P::real v[24];
#pragma unroll
  for (int k = 0; k < 24; k++) v[k] = (typename P::real)host_read(host, host_spinor_off(L, g, rhs, s, k), L.ft);
  SpinorIO<P>::store(f, rhs, s, v);
}

template <typename P>
__global__ void spinor_out_kernel(Geom g, HostLayout L, void *host, SpinorArg f, int nrhs)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int rhs = blockIdx.y;
  if (s >= g.vh || rhs >= nrhs) return;
  typename P::real v[24];
  SpinorIO<P>::load(f, rhs, s, v);
#pragma unroll
  for (int k = 0; k < 24; k++) host_write(host, host_spinor_off(L, g, rhs, s, k), L.ft, (double)v[k]);
}

// --- element stores into the chunked device layouts --------------------------
// value k of site s in an array of chunks holding `vpc` values each
template <typename P>
__device__ __forceinline__ void dev_store_real(void *base, long long stride, int vpc, long long s, int k,
                                               double val)
{
  long long chunk = k / vpc, within = k % vpc;
  long long e = (chunk * stride + s) * vpc + within;
  if (P::prec == PREC_F64)
    reinterpret_cast<double *>(base)[e] = val;
  else if (P::prec == PREC_F32 || P::prec == PREC_Q16F32)  // Q16F32 links / clover terms are FP32
    reinterpret_cast<float *>(base)[e] = (float)val;
  else if (P::prec == PREC_F16 || P::prec == PREC_Q16)  // Q16 links / clover terms are FP16
    reinterpret_cast<__half *>(base)[e] = __float2half((float)val);
  else
    reinterpret_cast<__nv_bfloat16 *>(base)[e] = __float2bfloat16((float)val);
}

template <typename P>
__device__ __forceinline__ double dev_load_real(const void *base, long long stride, int vpc, long long s, int k)
{
  long long chunk = k / vpc, within = k % vpc;
  long long e = (chunk * stride + s) * vpc + within;
  if (P::prec == PREC_F64) return reinterpret_cast<const double *>(base)[e];
  if (P::prec == PREC_F32 || P::prec == PREC_Q16F32) return reinterpret_cast<const float *>(base)[e];
  if (P::prec == PREC_F16 || P::prec == PREC_Q16) return __half2float(reinterpret_cast<const __half *>(base)[e]);
  return __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(base)[e]);
}

// Gauge: reads U_mu(x) for x in checkerboard `cb` (canonical: both cbs in one
// array, `cb` selects; qphix: the array of that cb, forward slot 2 mu + 1,
// stored [c][c2] = U(c2, c), compressed arrays keep columns 0 and 1).
//
// back = 1 (qphix only): read the back-link slot 2 mu of checkerboard cb,
// U_mu(x - mu) (qdp_packer_parscalar.h:94-110), and store it as the forward
// link of site x - mu in the other checkerboard's slab.
template <typename P>
__global__ void gauge_in_kernel(Geom g, HostLayout L, const void *host, void *dev, long long stride,
                                long long slab_bytes, int vpc, int recon, int cb, int back)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (s >= g.vh) return;
  int dst_cb = cb, dst_s = s;
  if (back) {
    int xh, y, z, t, par;
    site_coords(g, s, cb, xh, y, z, t, par);
    int c[4] = {2 * xh + par, y, z, t};
    int n[4] = {g.nx, g.ny, g.nz, g.nt};
    c[mu] = (c[mu] - 1 + n[mu]) % n[mu];
    dst_cb = 1 - cb;
    dst_s = ((c[3] * g.nz + c[2]) * g.ny + c[1]) * g.nxh + c[0] / 2;
  }
  double u[3][3][2];
  if (L.kind != HOST_QPHIX) {
    long long base = L.kind == HOST_CANONICAL ? (((long long)cb * 4 + mu) * g.vh + s) * 18
                                              : (((long long)mu * 2 + cb) * g.vh + s) * 18;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++)
        for (int ri = 0; ri < 2; ri++) u[r][c][ri] = host_read(host, base + (r * 3 + c) * 2 + ri, L.ft);
  } else {
    long long blk;
    int lane;
    host_gblock(L, g, s, blk, lane);
    int nc = L.c12 ? 2 : 3;
    long long bsz = 8LL * nc * 3 * 2 * L.V;
    int slot = back ? 2 * mu : 2 * mu + 1;
    for (int c = 0; c < nc; c++)
      for (int c2 = 0; c2 < 3; c2++)
        for (int ri = 0; ri < 2; ri++)
          u[c2][c][ri] =
              host_read(host, blk * bsz + (((long long)(slot * nc + c) * 3 + c2) * 2 + ri) * L.V + lane, L.ft);
    if (L.c12) {  // column 2 = conj(col0 x col1)
      for (int r = 0; r < 3; r++) {
        int r1 = (r + 1) % 3, r2 = (r + 2) % 3;
        double ar = u[r1][0][0], ai = u[r1][0][1], br = u[r2][1][0], bi = u[r2][1][1];
        double cr = u[r2][0][0], ci = u[r2][0][1], dr = u[r1][1][0], di = u[r1][1][1];
        double re = (ar * br - ai * bi) - (cr * dr - ci * di);
        double im = (ar * bi + ai * br) - (cr * di + ci * dr);
        u[r][2][0] = re;
        u[r][2][1] = -im;
      }
    }
  }
  char *slab = reinterpret_cast<char *>(dev) + ((long long)dst_cb * 4 + mu) * slab_bytes;
  int nstore = (recon == 12) ? 2 : 3;
  for (int r = 0; r < nstore; r++)
    for (int c = 0; c < 3; c++)
      for (int ri = 0; ri < 2; ri++) dev_store_real<P>(slab, stride, vpc, dst_s, (r * 3 + c) * 2 + ri, u[r][c][ri]);
}

// clover / full clover: NR reals per site, canonical [Vh][NR] or qphix
// CloverBlock / FullCloverBlock (both keep the canonical order, V innermost)
template <typename P>
__global__ void clover_in_kernel(Geom g, HostLayout L, const void *host, void *dev, long long stride, int vpc,
                                 int nr)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.vh) return;
  if (L.kind == HOST_CANONICAL) {
    for (int k = 0; k < nr; k++) dev_store_real<P>(dev, stride, vpc, s, k, host_read(host, (long long)s * nr + k, L.ft));
  } else if (L.kind == HOST_QDP) {
    for (int k = 0; k < nr; k++)
      dev_store_real<P>(dev, stride, vpc, s, k, host_read(host, (long long)s * nr + qdp_clover_off(k), L.ft));
  } else {
    long long blk;
    int lane;
    host_gblock(L, g, s, blk, lane);
    for (int k = 0; k < nr; k++)
      dev_store_real<P>(dev, stride, vpc, s, k, host_read(host, blk * nr * L.V + (long long)k * L.V + lane, L.ft));
  }
}

// canonical FP64 [Vh][NR], or (qdp) the compacted checkerboard half in
// Chroma's triangle order, FP64 or FP32
template <typename P>
__global__ void clover_out_kernel(Geom g, HostLayout L, void *host, const void *dev, long long stride, int vpc,
                                  int nr)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.vh) return;
  const bool qdp = L.kind == HOST_QDP;
  for (int k = 0; k < nr; k++)
    host_write(host, (long long)s * nr + (qdp ? qdp_clover_off(k) : k), L.ft, dev_load_real<P>(dev, stride, vpc, s, k));
}

}  // namespace qpx
