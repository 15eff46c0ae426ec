// Deterministic global reductions fused into the epilogue of any kernel, and
// the device-resident solver scalars they feed.
//
// Every reducing kernel computes up to QPX_MAX_RED doubles per right-hand
// side per thread, reduces them over the block (warp shuffles, then a fixed
// order over warps, one barrier for all values) and writes one partial per
// (block, rhs, value).  fold_kernel (blas.cu), launched next on the
// same stream, adds the partials of every value in a fixed order -- a group
// of warps per value, lane l of warp g taking site blocks in a fixed stride,
// then shuffle trees and the group's warps in order -- and runs a finalize
// step on thread 0.  The order of every addition is fixed by the launch
// shape, so results are bitwise reproducible run to run.
//
// The finalize step updates a SolverState in device memory (Krylov scalars
// alpha, beta, omega, rho, residual norms, convergence flags) so that a
// solver iteration is a fixed sequence of launches with no host round trip:
// it can be captured once in a CUDA graph and replayed.
#pragma once

#include "qpx_common.cuh"

namespace qpx {

constexpr int QPX_MAX_RHS = 32;
constexpr int QPX_MAX_RED = 6;
constexpr int QPX_NSLOT = 24;
constexpr int QPX_BLOCK = 128;

// scalar slots (per rhs)
enum Slot : int {
  S_RHO_RE = 0, S_RHO_IM, S_RHOP_RE, S_RHOP_IM, S_ALPHA_RE, S_ALPHA_IM,
  S_OMEGA_RE, S_OMEGA_IM, S_BETA_RE, S_BETA_IM, S_RNORM, S_TNORM,
  S_A, S_B, S_C, S_D, S_RSD, S_AUX0, S_AUX1, S_AUX2, S_AUX3, S_AUX4, S_AUX5, S_AUX6
};

struct SolverState {
  int done;       // 1: stop issuing work (all rhs converged, broke down or hit max)
  int iter;       // completed iterations
  int max_iter;
  int status;     // 0 converged / running, 1 max iterations, 2 breakdown
  int nrhs;
  int coupled;    // 1: right-hand sides 2k, 2k+1 are one two-flavour system
  int pad[2];
  int rhs_done[QPX_MAX_RHS];
  int rhs_iter[QPX_MAX_RHS];
  double v[QPX_NSLOT][QPX_MAX_RHS];
};

// finalize operations (solver-specific scalar recurrences)
enum FinOp : int {
  FIN_NONE = 0,
  FIN_CG_A,        // d = |Mp|^2 ; a = c / d
  FIN_CG_R,        // cp = |r|^2 ; converged? ; b = cp / c ; c = cp
  FIN_BICG_ALPHA,  // <r0,v> -> alpha = rho / <r0,v>, rho_prev = rho
  FIN_BICG_OMEGA,  // |t|^2, <t,s> -> omega
  FIN_BICG_RX,     // |r|^2, <r0,r> -> converged? ; rho ; beta
  FIN_MR_A,        // |Mr|^2, <Mr,r> -> a = Omega <Mr,r>/|Mr|^2
  FIN_MR_R,        // |r|^2 -> converged?
  FIN_STORE,       // plain reduction: result only
  FIN_MCG_D,       // multishift CG: d = |Mp|^2, b = -cp/d
  FIN_MCG_R,       // multishift CG: c = |r|^2, zeta/beta per shift, convergence
  FIN_BICG_RU,     // BiCGStab with reliable updates: as FIN_BICG_RX, asks for an update
  FIN_CG_P,        // shifted CG: |p|^2 of the new p, for the next FIN_CG_A
};

struct ReduceArg {
  int mask;            // which values (bit order fixed by the producing kernel)
  int nval;            // number of doubles per rhs
  int fin;             // FinOp
  double *partials;    // [nrhs][nval][nblocks]
  double *result;      // [nrhs][nval]
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Called by every thread of every block after the block's per-thread values
// are final.  Values live in fixed slots val[r][k] (k < QPX_MAX_RED, compile-
// time indices so they stay in registers); `slots` (ReduceArg::mask of the
// producing kernel, translated by it into a slot bit set) says which slots
// are live, and they are packed in slot order into nval doubles per rhs.
// rhs0 = first rhs of the block's tile.  Each block writes one partial per
// (rhs, value) under site-block index `sblock` of `nsblocks` (default:
// blockIdx.x of gridDim.x; kernels whose blocks cover (site block, rhs tile)
// pairs in one grid dimension pass their own), value-major so that the fold
// reads every value's partials contiguously, and is done: the partials are
// folded, and the solver's finalize step run, by fold_kernel, launched after
// the producing kernel on the same stream.  Blocks therefore never wait on
// one another or on a device-wide fence, and the fold runs with a full block
// of threads.
// A block partial is written with L2 evict-last priority: the fold kernel
// reads it after the rest of the producing launch has streamed its fields
// (up to ~190 MB for the 16^3x32, 8-rhs BLAS passes) through the 126 MB L2,
// which with normal priority pushes the early blocks' partials out to DRAM.
__device__ __forceinline__ void store_partial(double *p, double v)
{
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}

template <int R>
__device__ __forceinline__ void reduce_epilogue(const ReduceArg &ra, int nrhs, int rhs0, int slots,
                                                const double val[R][QPX_MAX_RED], int sblock = -1,
                                                int nsblocks = -1)
{
  constexpr int NW = QPX_BLOCK / 32;  // launches of these kernels use QPX_BLOCK threads
  __shared__ double wpart[NW][R * QPX_MAX_RED];
  if (sblock < 0) {
    sblock = blockIdx.x;
    nsblocks = gridDim.x;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // every live value's warp sum, then one barrier and a fixed-order sum over warps
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < QPX_MAX_RED; k++)
      if (slots & (1 << k)) {
        const double s = warp_sum(val[r][k]);
        if (lane == 0) wpart[wid][r * QPX_MAX_RED + k] = s;
      }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int r = 0; r < R; r++) {
      int o = 0;
#pragma unroll
      for (int k = 0; k < QPX_MAX_RED; k++) {
        if (slots & (1 << k)) {
          double s = 0.0;
          for (int w = 0; w < NW; w++) s += wpart[w][r * QPX_MAX_RED + k];
          if (rhs0 + r < nrhs) store_partial(ra.partials + ((long long)(rhs0 + r) * ra.nval + o) * nsblocks + sblock, s);
          o++;
        }
      }
    }
  }
}

constexpr int QPX_FOLD_THREADS = 1024;

}  // namespace qpx
