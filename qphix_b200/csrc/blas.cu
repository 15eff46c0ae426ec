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

static void check_pdl_launch(cudaError_t e)
{
  if (e != cudaSuccess) throw Error(QPHIX_GPU_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

void launch_blas(int prec, const BlasArgs &a, dim3 grid, cudaStream_t st)
{
  QPX_PREC_SWITCH(prec, (check_pdl_launch(launch_pdl(blas_kernel<P>, grid, dim3(QPX_BLOCK), st, (long long)grid.x * grid.y, a))));
}

// Folds the block partials of one reducing launch (reduce_epilogue,
// qpx_reduce.cuh) into ra.result and runs the solver's finalize step; one
// block of QPX_FOLD_THREADS threads, launched right after the producing
// kernel on its stream, instantiated per finalize step (FIN) so that each
// carries only its own recurrence.  The nres = nrhs x nval values share the
// 32 warps, a group of G = max(1, 32 / nres) warps per value (further rounds
// when nres > 32): lane l of warp g of a group adds site blocks 32 g + l,
// 32 g + l + 32 G, ... in that order, then a shuffle tree per warp and the
// group's warps in order.  Warp 0 then runs the finalize, a lane per
// right-hand side.  A solver state that is already done makes it write
// nothing, as the producing kernel did.
template <int FIN>
__global__ void __launch_bounds__(QPX_FOLD_THREADS) fold_kernel(const ReduceArg ra, SolverState *st, int nrhs,
                                                                int nparts)
{
  __shared__ double gsum[QPX_FOLD_THREADS / 32];
  __shared__ double res[QPX_MAX_RHS * QPX_MAX_RED];
  __shared__ SolverState sst;
  constexpr int kStateWords = sizeof(SolverState) / sizeof(int);
  static_assert(sizeof(SolverState) % sizeof(int) == 0, "SolverState is copied as 32-bit words");
  constexpr bool kFinalize = FIN != FIN_NONE && FIN != FIN_STORE;  // steps that update the state
  const int nres = nrhs * ra.nval;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  pdl_trigger();
  pdl_wait();
  // the solver state is read and written by the finalize step below: a
  // shared copy turns its chains of dependent global accesses into
  // shared-memory ones.  Its loads and the partials' loads are all issued
  // before anything waits on them (a done solver is recognised afterwards,
  // from the copy: its producing launch wrote no partials, and nothing is
  // written back).
  if (st) {
    if (kFinalize)
      for (int i = threadIdx.x; i < kStateWords; i += blockDim.x)
        reinterpret_cast<int *>(&sst)[i] = reinterpret_cast<const int *>(st)[i];
    else if (threadIdx.x == 0) {
      sst.done = st->done;
      sst.coupled = st->coupled;
    }
  }
  const int G = nres >= 32 ? 1 : 32 / nres;
  const int vpr = 32 / G;  // values per round
  for (int v0 = 0; v0 < nres; v0 += vpr) {
    const int slot = wid / G, g = wid % G;
    const int v = v0 + slot;
    double acc = 0.0;
    if (slot < vpr && v < nres) {
      const double *p = ra.partials + (long long)v * nparts;  // value-major: coalesced across the lanes
#pragma unroll 8
      for (int b = 32 * g + lane; b < nparts; b += 32 * G) acc += __ldcg(p + b);
    }
    acc = warp_sum(acc);
    if (lane == 0) gsum[wid] = acc;
    __syncthreads();
    if ((int)threadIdx.x < vpr && v0 + (int)threadIdx.x < nres) {
      double t = 0.0;
      for (int k = 0; k < G; k++) t += gsum[threadIdx.x * G + k];
      res[v0 + threadIdx.x] = t;
    }
    __syncthreads();
  }
  __syncthreads();
  if (st && sst.done) return;  // uniform: every thread reads the same shared flag
  const bool use_state = kFinalize && st;
  if (wid == 0 && st) {
    // two-flavour systems: each flavour pair's reductions are one sum (the
    // reference's num_flav = 2 BLAS), so both get the same solver scalars
    if (sst.coupled) {
      const int r = lane & ~1;
      double t[QPX_MAX_RED];
#pragma unroll
      for (int k = 0; k < QPX_MAX_RED; k++)
        if (k < ra.nval && r + 1 < nrhs) t[k] = res[r * ra.nval + k] + res[(r + 1) * ra.nval + k];
      __syncwarp();
#pragma unroll
      for (int k = 0; k < QPX_MAX_RED; k++)
        if (k < ra.nval && r + 1 < nrhs && lane < nrhs) res[lane * ra.nval + k] = t[k];
      __syncwarp();
    }
    if (use_state) finalize_warp<FIN>(&sst, res, nrhs, ra.nval, lane);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nres; i += blockDim.x) ra.result[i] = res[i];
  if (use_state)
    for (int i = threadIdx.x; i < kStateWords; i += blockDim.x)
      reinterpret_cast<int *>(st)[i] = reinterpret_cast<const int *>(&sst)[i];
}

void launch_fold(const ReduceArg &ra, SolverState *state, int nrhs, int nparts, cudaStream_t st)
{
#define QPX_FOLD_CASE(F) \
  case F: check_pdl_launch(launch_pdl(fold_kernel<F>, dim3(1), dim3(QPX_FOLD_THREADS), st, (long long)nparts * nrhs, ra, state, nrhs, nparts)); break;
  switch (ra.fin) {
    QPX_FOLD_CASE(FIN_NONE)
    QPX_FOLD_CASE(FIN_CG_A)
    QPX_FOLD_CASE(FIN_CG_R)
    QPX_FOLD_CASE(FIN_BICG_ALPHA)
    QPX_FOLD_CASE(FIN_BICG_OMEGA)
    QPX_FOLD_CASE(FIN_BICG_RX)
    QPX_FOLD_CASE(FIN_BICG_RU)
    QPX_FOLD_CASE(FIN_MR_A)
    QPX_FOLD_CASE(FIN_MR_R)
    QPX_FOLD_CASE(FIN_STORE)
    QPX_FOLD_CASE(FIN_MCG_D)
    QPX_FOLD_CASE(FIN_MCG_R)
    QPX_FOLD_CASE(FIN_CG_P)
  default: throw Error(QPHIX_GPU_EINVAL, "bad finalize step");
  }
#undef QPX_FOLD_CASE
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
