// Explicit instantiation of the Dslash kernel family for one precision; each
// precision lives in its own translation unit so they compile in parallel.
#pragma once

#include "qpx_finalize.cuh"
#include "qpx_host.h"

namespace qpx {

template <typename P, int RECON, int R, int S>
void launch_dslash_prs(int epi, int achi, const DslashArgs &a, dim3 grid, cudaStream_t st)
{
  dim3 block(QPX_BLOCK);
  if (achi == ACHI_NONE) {
    switch (epi) {
    case EPI_NONE: dslash_kernel<P, RECON, EPI_NONE, ACHI_NONE, R, S><<<grid, block, 0, st>>>(a); return;
    case EPI_CLOV: dslash_kernel<P, RECON, EPI_CLOV, ACHI_NONE, R, S><<<grid, block, 0, st>>>(a); return;
    case EPI_TMINV: dslash_kernel<P, RECON, EPI_TMINV, ACHI_NONE, R, S><<<grid, block, 0, st>>>(a); return;
    case EPI_FCLOV: dslash_kernel<P, RECON, EPI_FCLOV, ACHI_NONE, R, S><<<grid, block, 0, st>>>(a); return;
    }
  } else if (epi == EPI_NONE) {
    switch (achi) {
    case ACHI_ALPHA: dslash_kernel<P, RECON, EPI_NONE, ACHI_ALPHA, R, S><<<grid, block, 0, st>>>(a); return;
    case ACHI_CLOV: dslash_kernel<P, RECON, EPI_NONE, ACHI_CLOV, R, S><<<grid, block, 0, st>>>(a); return;
    case ACHI_TM: dslash_kernel<P, RECON, EPI_NONE, ACHI_TM, R, S><<<grid, block, 0, st>>>(a); return;
    }
  }
  throw Error(QPHIX_GPU_EINVAL, "unsupported dslash epilogue combination");
}

// isign is a template parameter: the projector signs become adds / subtracts
template <typename P, int RECON, int R>
void launch_dslash_pr(int epi, int achi, const DslashArgs &a, dim3 grid, cudaStream_t st)
{
  if (a.isign == 1)
    launch_dslash_prs<P, RECON, R, 1>(epi, achi, a, grid, st);
  else
    launch_dslash_prs<P, RECON, R, -1>(epi, achi, a, grid, st);
}

template <typename P, int R>
void launch_dslash_r(int recon, int epi, int achi, const DslashArgs &a, dim3 grid, cudaStream_t st)
{
  if (recon == 12)
    launch_dslash_pr<P, 12, R>(epi, achi, a, grid, st);
  else
    launch_dslash_pr<P, 18, R>(epi, achi, a, grid, st);
}

}  // namespace qpx
