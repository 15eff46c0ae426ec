// Explicit instantiation of the Dslash kernel family for one precision; each
// precision lives in its own translation unit so they compile in parallel.
#pragma once

#include <type_traits>

#include "qpx_finalize.cuh"
#include "qpx_host.h"

namespace qpx {

inline void check_pdl(cudaError_t e)
{
  if (e != cudaSuccess) throw Error(QPHIX_GPU_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

template <typename P, int RECON, int R, int S, int SP, bool GEN, bool RL = false>
void launch_dslash_k(int epi, int achi, const DslashArgs &a, dim3 grid, cudaStream_t st)
{
  dim3 block(QPX_BLOCK);
  if (achi == ACHI_NONE) {
    switch (epi) {
    case EPI_NONE: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NONE, ACHI_NONE, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    case EPI_CLOV: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_CLOV, ACHI_NONE, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    case EPI_TMINV: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_TMINV, ACHI_NONE, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    case EPI_FCLOV: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_FCLOV, ACHI_NONE, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    }
  } else if (epi == EPI_NONE) {
    switch (achi) {
    case ACHI_ALPHA: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NONE, ACHI_ALPHA, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    case ACHI_CLOV: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NONE, ACHI_CLOV, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    case ACHI_TM: check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NONE, ACHI_TM, R, S, SP, GEN, RL>, grid, block, st, (long long)grid.x * grid.y, a)); return;
    }
  }
  throw Error(QPHIX_GPU_EINVAL, "unsupported dslash epilogue combination");
}

// the two-flavour twisted-mass kernels (two right-hand sides per thread)
template <typename P, int RECON, int S>
void launch_dslash_nd(int epi, int achi, const DslashArgs &a, dim3 grid, cudaStream_t st)
{
  dim3 block(QPX_BLOCK);
  if (achi == ACHI_NONE && epi == EPI_NDTM)
    check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NDTM, ACHI_NONE, 2, S, 1, false>, grid, block, st, (long long)grid.x * grid.y, a));
  else if (epi == EPI_NONE && achi == ACHI_NDTM)
    check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NONE, ACHI_NDTM, 2, S, 1, false>, grid, block, st, (long long)grid.x * grid.y, a));
  else if (achi == ACHI_NONE && epi == EPI_NDFCLOV)
    check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NDFCLOV, ACHI_NONE, 2, S, 1, false>, grid, block, st, (long long)grid.x * grid.y, a));
  else if (epi == EPI_NONE && achi == ACHI_NDCLOV)
    check_pdl(launch_pdl(dslash_kernel<P, RECON, EPI_NONE, ACHI_NDCLOV, 2, S, 1, false>, grid, block, st, (long long)grid.x * grid.y, a));
  else
    throw Error(QPHIX_GPU_EINVAL, "unsupported two-flavour dslash combination");
}

// isign is a template parameter: the projector signs become adds / subtracts
template <typename P, int RECON, int R, int SP, bool GEN, bool RL = false>
void launch_dslash_s(int epi, int achi, const DslashArgs *a, dim3 grid, cudaStream_t st)
{
  if (!a) return;  // shape query
  if (a->isign == 1)
    launch_dslash_k<P, RECON, R, 1, SP, GEN, RL>(epi, achi, *a, grid, st);
  else
    launch_dslash_k<P, RECON, R, -1, SP, GEN, RL>(epi, achi, *a, grid, st);
}

// The shapes built for storage P.  a == nullptr: only report whether the
// shape exists.  Returns false for a shape that is not built.
//   general path (dir mask, twisted phases): R = 1, SP = 1
//   fast path: R = 1 SP = 1 for every precision; for FP32 arithmetic also
//   SP = 2 (both link kinds), R = 2 (12-real links) and two right-hand sides
//   in the float2 lanes (rl, 12-real links, even nrhs)
template <typename P>
bool launch_dslash_p(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                     cudaStream_t st)
{
  constexpr bool fp32 = std::is_same<typename P::real, float>::value;
  if (recon != 12 && recon != 18) return false;
  if (is_two_flavour(epi, achi)) {  // two-flavour twisted mass (clover): R = 2 only
    if (sh.R != 2 || sh.SP != 1 || sh.gen) return false;
    if (!a) return true;
    const bool plus = a->isign == 1;
    if (recon == 12)
      plus ? launch_dslash_nd<P, 12, 1>(epi, achi, *a, grid, st) : launch_dslash_nd<P, 12, -1>(epi, achi, *a, grid, st);
    else
      plus ? launch_dslash_nd<P, 18, 1>(epi, achi, *a, grid, st) : launch_dslash_nd<P, 18, -1>(epi, achi, *a, grid, st);
    return true;
  }
  if (sh.rl) {
    if constexpr (fp32) {
      if (sh.R != 1 || sh.SP != 2 || sh.gen || recon != 12) return false;
      if (a && a->nrhs % 2) return false;
      launch_dslash_s<P, 12, 1, 2, false, true>(epi, achi, a, grid, st);
      return true;
    }
    return false;
  }
  if (sh.gen) {
    if (sh.R != 1 || sh.SP != 1) return false;
    if (recon == 12)
      launch_dslash_s<P, 12, 1, 1, true>(epi, achi, a, grid, st);
    else
      launch_dslash_s<P, 18, 1, 1, true>(epi, achi, a, grid, st);
    return true;
  }
  if (sh.R == 1 && sh.SP == 1) {
    if (recon == 12)
      launch_dslash_s<P, 12, 1, 1, false>(epi, achi, a, grid, st);
    else
      launch_dslash_s<P, 18, 1, 1, false>(epi, achi, a, grid, st);
    return true;
  }
  if constexpr (fp32) {
    if (sh.R == 1 && sh.SP == 2) {
      if (recon == 12)
        launch_dslash_s<P, 12, 1, 2, false>(epi, achi, a, grid, st);
      else
        launch_dslash_s<P, 18, 1, 2, false>(epi, achi, a, grid, st);
      return true;
    }
    if (sh.R == 2 && sh.SP == 1 && recon == 12) {
      launch_dslash_s<P, 12, 2, 1, false>(epi, achi, a, grid, st);
      return true;
    }
  }
  return false;
}

}  // namespace qpx
