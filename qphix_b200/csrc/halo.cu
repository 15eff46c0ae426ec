// Face packing of the halo mode for a lattice cut along any direction: the
// sites of one checkerboard of a slice x = k, y = k, z = k or t = k, in the
// face order the Dslash kernel's ghost reads use (DslashArgs::halo).  One
// thread per face site copies every chunk row (right-hand sides x chunks, or
// one link's chunks) and, for 16-bit spinors, the per-site norms.
#include "qpx_host.h"

namespace qpx {

struct FaceMap {
  Geom g;
  int mu;     // direction of the slice
  int slice;  // its coordinate along mu
  int cb;     // checkerboard of the packed field (decides the x face's sites)
};

// checkerboard site index of face site j
__device__ __forceinline__ long long face_site(const FaceMap &m, int j)
{
  const Geom &g = m.g;
  int xh, y, z, t;
  if (m.mu == 3) {
    t = m.slice;
    xh = j % g.nxh;
    const int r = j / g.nxh;
    y = r % g.ny;
    z = r / g.ny;
  } else if (m.mu == 2) {
    z = m.slice;
    xh = j % g.nxh;
    const int r = j / g.nxh;
    y = r % g.ny;
    t = r / g.ny;
  } else if (m.mu == 1) {
    y = m.slice;
    xh = j % g.nxh;
    const int r = j / g.nxh;
    z = r % g.nz;
    t = r / g.nz;
  } else {
    // x = slice: for each (z, t) the sites of checkerboard cb take every
    // other y, those with (x + y + z + t) even for cb 0, odd for cb 1
    const int x = m.slice, nyh = g.ny / 2;
    const int jy = j % nyh, r = j / nyh;
    z = r % g.nz;
    t = r / g.nz;
    y = 2 * jy + ((m.cb + x + z + t) & 1);
    xh = x >> 1;
  }
  return ((long long)(t * g.nz + z) * g.ny + y) * g.nxh + xh;
}

template <typename W>
__global__ void __launch_bounds__(QPX_BLOCK) face_pack_kernel(FaceMap m, const W *src, long long src_stride,
                                                             int rows, long long face, W *dst, const float *nsrc,
                                                             float *ndst, int nrows)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= face) return;
  const long long s = face_site(m, j);
  for (int row = blockIdx.y; row < rows; row += gridDim.y) dst[row * face + j] = src[row * src_stride + s];
  if (nsrc && blockIdx.y == 0)
    for (int r = 0; r < nrows; r++) ndst[r * face + j] = nsrc[r * src_stride + s];
}

void launch_face_pack(const Geom &g, int mu, int slice, int cb, const void *src, long long src_stride, int rows,
                      int chunk_bytes, long long face, void *dst, const float *nsrc, float *ndst, int nrows,
                      cudaStream_t st)
{
  FaceMap m{g, mu, slice, cb};
  const dim3 grid((unsigned)((face + QPX_BLOCK - 1) / QPX_BLOCK), (unsigned)(rows < 65535 ? rows : 65535));
  switch (chunk_bytes) {
  case 16:
    face_pack_kernel<uint4><<<grid, QPX_BLOCK, 0, st>>>(m, static_cast<const uint4 *>(src), src_stride, rows, face,
                                                        static_cast<uint4 *>(dst), nsrc, ndst, nrows);
    break;
  case 8:
    face_pack_kernel<uint2><<<grid, QPX_BLOCK, 0, st>>>(m, static_cast<const uint2 *>(src), src_stride, rows, face,
                                                        static_cast<uint2 *>(dst), nsrc, ndst, nrows);
    break;
  case 4:
    face_pack_kernel<uint32_t><<<grid, QPX_BLOCK, 0, st>>>(m, static_cast<const uint32_t *>(src), src_stride, rows,
                                                           face, static_cast<uint32_t *>(dst), nsrc, ndst, nrows);
    break;
  default:
    throw Error(QPHIX_GPU_EINVAL, "face pack: unsupported chunk size");
  }
}

}  // namespace qpx
