// Persistent-kernel CG on M^+ M (include/qphix/invcg.h:281-417) for lattices
// too small to fill the GPU, where a launch per Dslash, fold and BLAS step
// costs more than the step itself.  One cooperative launch runs every
// iteration: the grid stays resident, the phases of an iteration are
// separated by grid barriers, and every block folds the reductions itself
// and keeps its own shared-memory copy of the solver state, so no block
// waits on another for a scalar.
//
// One iteration (the graph-captured iteration of solve_cg, as phases):
//   0  tmp = D p                      (first kernel of M, other checkerboard)
//   1  mp = g5 M p, partials of |mp|^2  (second kernel of M, result times g5)
//      barrier; every block: fold |mp|^2, FIN_CG_A -> a
//   2  tmp = D mp
//   3  mmp = g5 M mp = M^+ M p; r -= a mmp; x += a p; partials of |r|^2
//      barrier; every block: fold |r|^2, FIN_CG_R -> b, convergence
//   4  p = r + b p
// M^+ = g5 M g5 (gamma_5-hermiticity of the Wilson and clover even-odd
// operators; g5 = diag(1, 1, -1, -1) commutes with the clover term and turns
// D(+1) into D(-1)), so phases 2 and 3 run the same two kernel bodies as
// phases 0 and 1 with isign = +1: half the code, which matters because the
// kernel's phases otherwise evict one another from the instruction cache.
// The sign flips are exact, so the iterates are bit for bit those of the
// graph path's D(-1) launches.
// Phases 0-3 run the Dslash kernel's own per-block code (dslash_block) over
// all virtual blocks of a launch of the regular kernel's shape (one site and
// one right-hand side per thread); the folds add the partials in the order
// fold_kernel uses, and the finalize is the same finalize_warp, so the
// iterates are those of the graph-captured solver.
//
// Every block computes the same scalars from the same partials, so the
// copies agree without communication; block 0 writes the final state back.
// Spinors written inside the launch are read through L2 (Coherent<P>).
// A grid barrier waits at most kBarrierSpins polls (after the first 1024,
// each followed by a __nanosleep); a block that gives up sets bar->error and
// leaves, and the others see the flag while they wait and leave too.
#pragma once

#include "qpx_dslash.cuh"
#include "qpx_finalize.cuh"

namespace qpx {

struct GridBarrier {
  unsigned int count;  // arrivals since the launch began (monotonic)
  int error;           // 1: a block gave up waiting
  int where;           // the barrier it gave up at
  int pad;
};

struct CgPersistArgs {
  DslashArgs d[4];  // phases 0-3, as captured from the regular solver's launches (d[1], d[3]: g5_out)
  SpinorArg r, p;   // phase 4
  SolverState *state;
  GridBarrier *bar;
  int nrhs;
  int vh;
  int nsb;  // site blocks of QPX_BLOCK sites
};

constexpr long long kBarrierSpins = 1ll << 22;

// Grid barrier on a counter that only grows: barrier k of the launch is
// passed once the counter reaches k x gridDim.x (`target`, advanced by every
// call).  Thread 0 of each block adds its arrival with release semantics and
// polls with acquire semantics; the block barriers on both sides order the
// other threads' memory accesses with them (the cooperative-groups grid
// barrier's pattern).  No reset is needed between barriers, so an arrival is
// one fire-and-forget reduction and the last one releases every waiter at
// their next poll.
__device__ __forceinline__ bool grid_barrier(GridBarrier *b, unsigned int &target, int where)
{
  __shared__ int ok;
  target += gridDim.x;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&b->count) : "memory");
    volatile int *verr = &b->error;
    long long n = 0;
    while (true) {
      unsigned int c;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(&b->count) : "memory");
      if ((int)(c - target) >= 0) break;
      ++n;
      if ((n & 63) == 0 && *verr) {
        good = 0;
        break;
      }
      if (n > kBarrierSpins) {
        atomicExch(&b->where, where);
        atomicExch(&b->error, 1);
        good = 0;
        break;
      }
      if (n > 1024) __nanosleep(64);
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// The nrhs x nval values of one reduction, from partials [value][nsb], into
// res: the per-value arithmetic of fold_kernel (G = max(1, 32 / nres) groups,
// group g's lane l adding site blocks 32 g + l, 32 g + l + 32 G, ..., a
// shuffle tree per group, the groups added in order).
__device__ __forceinline__ void fold_in_block(const ReduceArg &ra, int nrhs, int nsb, double *res)
{
  const int nres = nrhs * ra.nval;
  const int G = nres >= 32 ? 1 : 32 / nres;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = wid; v < nres; v += QPX_BLOCK / 32) {
    const double *p = ra.partials + (long long)v * nsb;
    double t = 0.0;
    for (int g = 0; g < G; g++) {
      double acc = 0.0;
      for (int b = 32 * g + lane; b < nsb; b += 32 * G) acc += __ldcg(p + b);
      t += warp_sum(acc);
    }
    if (lane == 0) res[v] = t;
  }
  __syncthreads();
}

template <typename P, int RECON, int EPI, int ACHI, int ISIGN>
__global__ void __launch_bounds__(QPX_BLOCK) cg_persistent_kernel(const __grid_constant__ CgPersistArgs a)
{
  using PC = Coherent<P>;
  using T = typename P::real;
  __shared__ SolverState sst;
  __shared__ double res[QPX_MAX_RHS * QPX_MAX_RED];
  constexpr int kStateWords = sizeof(SolverState) / sizeof(int);
  for (int i = threadIdx.x; i < kStateWords; i += blockDim.x)
    reinterpret_cast<int *>(&sst)[i] = __ldcg(reinterpret_cast<const int *>(a.state) + i);
  __syncthreads();
  const int nvb = a.nsb * a.nrhs;  // virtual blocks of a Dslash phase: (site block, rhs)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned int target = 0;  // this block's grid-barrier count
  while (!sst.done) {
    // the two halves of an iteration (M p, then M^+ on its result) run the
    // same code: one call site per kernel body, the half's arguments
    // selected at run time
    bool ok = true;
#pragma unroll 1
    for (int half = 0; half < 2 && ok; half++) {
      const DslashArgs &da = a.d[2 * half], &db = a.d[2 * half + 1];
      for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        dslash_block<PC, RECON, EPI, ACHI_NONE, 1, ISIGN, 1, false>(da, &sst, vb, nvb);
        __syncthreads();
      }
      if (!grid_barrier(a.bar, target, 2 * half)) {
        ok = false;
        break;
      }
      for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        dslash_block<PC, RECON, EPI_NONE, ACHI, 1, ISIGN, 1, false>(db, &sst, vb, nvb);
        __syncthreads();
      }
      if (!grid_barrier(a.bar, target, 2 * half + 1)) {
        ok = false;
        break;
      }
      fold_in_block(db.red, a.nrhs, a.nsb, res);
      if (wid == 0) {
        if (half == 0)
          finalize_warp<FIN_CG_A>(&sst, res, a.nrhs, db.red.nval, lane);
        else
          finalize_warp<FIN_CG_R>(&sst, res, a.nrhs, db.red.nval, lane);
      }
      __syncthreads();
    }
    if (!ok || sst.done) break;
    // p = r + b p, the arithmetic of blas_kernel's B_CG_P
    const long long n = (long long)a.vh * a.nrhs;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
      const int rhs = (int)(i / a.vh);
      const long long s = i - (long long)rhs * a.vh;
      T x[24], y[24];
      SpinorIO<PC>::load(a.r, rhs, s, x);
      SpinorIO<PC>::load(a.p, rhs, s, y);
      const T b = (T)sst.v[S_B][rhs];
#pragma unroll
      for (int k = 0; k < 24; k++) y[k] = x[k] + b * y[k];
      SpinorIO<PC>::store(a.p, rhs, s, y);
    }
    if (!grid_barrier(a.bar, target, 4)) break;
  }
  if (blockIdx.x == 0) {
    __syncthreads();
    for (int i = threadIdx.x; i < kStateWords; i += blockDim.x)
      reinterpret_cast<int *>(a.state)[i] = reinterpret_cast<const int *>(&sst)[i];
  }
}

}  // namespace qpx
