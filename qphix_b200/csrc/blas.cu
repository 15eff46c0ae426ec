// Launchers for the streaming BLAS, precision conversion and host-layout
// conversion kernels, for every storage precision.
#include "qpx_finalize.cuh"
#include "qpx_host.h"

namespace qpx {

ChunkSpec spinor_spec(int prec)
{
  switch (prec) {
  case PREC_F64: return {12, 16, 2};
  case PREC_F32: return {6, 16, 4};
  default: return {3, 16, 8};
  }
}

ChunkSpec gauge_spec(int prec, int recon)
{
  if (prec == PREC_Q16F32) prec = PREC_F32;  // FP32 links
  if (recon == 18) {
    switch (prec) {
    case PREC_F64: return {9, 16, 2};
    case PREC_F32: return {9, 8, 2};
    default: return {9, 4, 2};
    }
  }
  switch (prec) {
  case PREC_F64: return {6, 16, 2};
  case PREC_F32: return {3, 16, 4};
  default: return {3, 8, 4};
  }
}

ChunkSpec clover_spec(int prec, int nreal)
{
  if (prec == PREC_Q16F32) prec = PREC_F32;  // FP32 clover terms
  switch (prec) {
  case PREC_F64: return {nreal / 2, 16, 2};
  case PREC_F32: return {nreal / 4, 16, 4};
  default: return {nreal / 8, 16, 8};
  }
}

#define QPX_PREC_SWITCH(prec, CALL)                                \
  switch (prec) {                                                  \
  case PREC_F64: { using P = F64; CALL; } break;                   \
  case PREC_F32: { using P = F32; CALL; } break;                   \
  case PREC_F16: { using P = F16; CALL; } break;                   \
  case PREC_BF16: { using P = BF16; CALL; } break;                 \
  case PREC_Q16: { using P = Q16; CALL; } break;                   \
  case PREC_Q16F32: { using P = Q16F32; CALL; } break;             \
  default: throw Error(QPHIX_GPU_EINVAL, "bad precision");         \
  }

void launch_blas(int prec, const BlasArgs &a, dim3 grid, cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (blas_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(a)));
}

template <typename P>
static void conv_from(int pdst, int vh, SpinorArg src, SpinorArg dst, Coef scale, SolverState *state, int acc,
                      dim3 grid, cudaStream_t st)
{
  switch (pdst) {
  case PREC_F64: convert_kernel<P, F64><<<grid, QPX_BLOCK, 0, st>>>(vh, src, dst, scale, state, acc); break;
  case PREC_F32: convert_kernel<P, F32><<<grid, QPX_BLOCK, 0, st>>>(vh, src, dst, scale, state, acc); break;
  case PREC_F16: convert_kernel<P, F16><<<grid, QPX_BLOCK, 0, st>>>(vh, src, dst, scale, state, acc); break;
  case PREC_BF16: convert_kernel<P, BF16><<<grid, QPX_BLOCK, 0, st>>>(vh, src, dst, scale, state, acc); break;
  case PREC_Q16: convert_kernel<P, Q16><<<grid, QPX_BLOCK, 0, st>>>(vh, src, dst, scale, state, acc); break;
  case PREC_Q16F32: convert_kernel<P, Q16F32><<<grid, QPX_BLOCK, 0, st>>>(vh, src, dst, scale, state, acc); break;
  default: throw Error(QPHIX_GPU_EINVAL, "bad precision");
  }
}

void launch_convert(int pdst, int psrc, int vh, SpinorArg src, SpinorArg dst, Coef scale, SolverState *state,
                    dim3 grid, cudaStream_t st, int accumulate)
{
  QPX_PREC_SWITCH(psrc, (conv_from<P>(pdst, vh, src, dst, scale, state, accumulate, grid, st)));
}

void launch_spinor_in(int prec, Geom g, HostLayout L, const void *host, SpinorArg f, int nrhs, dim3 grid,
                      cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (spinor_in_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(g, L, host, f, nrhs)));
}

void launch_spinor_out(int prec, Geom g, HostLayout L, void *host, SpinorArg f, int nrhs, dim3 grid,
                       cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (spinor_out_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(g, L, host, f, nrhs)));
}

void launch_gauge_in(int prec, Geom g, HostLayout L, const void *host, void *dev, long long stride,
                     long long slab_bytes, int vpc, int recon, int cb, int back, dim3 grid, cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (gauge_in_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(g, L, host, dev, stride, slab_bytes, vpc,
                                                                          recon, cb, back)));
}

void launch_clover_in(int prec, Geom g, HostLayout L, const void *host, void *dev, long long stride, int vpc,
                      int nr, dim3 grid, cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (clover_in_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(g, L, host, dev, stride, vpc, nr)));
}

void launch_clover_out(int prec, Geom g, HostLayout L, void *host, const void *dev, long long stride, int vpc,
                       int nr, dim3 grid, cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (clover_out_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(g, L, host, dev, stride, vpc, nr)));
}

void launch_mshift(int prec, const MShiftArgs &a, dim3 grid, cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (mshift_update_kernel<P><<<grid, QPX_BLOCK, 0, st>>>(a)));
}

bool launch_dslash_f64(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                      cudaStream_t st);
bool launch_dslash_f32(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                      cudaStream_t st);
bool launch_dslash_f16(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                      cudaStream_t st);
bool launch_dslash_bf16(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                       cudaStream_t st);
bool launch_dslash_q16(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                      cudaStream_t st);
bool launch_dslash_q16f32(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                         cudaStream_t st);

bool launch_dslash(int prec, int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                   cudaStream_t st)
{
  switch (prec) {
  case PREC_F64: return launch_dslash_f64(recon, epi, achi, sh, a, grid, st);
  case PREC_F32: return launch_dslash_f32(recon, epi, achi, sh, a, grid, st);
  case PREC_F16: return launch_dslash_f16(recon, epi, achi, sh, a, grid, st);
  case PREC_BF16: return launch_dslash_bf16(recon, epi, achi, sh, a, grid, st);
  case PREC_Q16: return launch_dslash_q16(recon, epi, achi, sh, a, grid, st);
  case PREC_Q16F32: return launch_dslash_q16f32(recon, epi, achi, sh, a, grid, st);
  }
  return false;
}

}  // namespace qpx
