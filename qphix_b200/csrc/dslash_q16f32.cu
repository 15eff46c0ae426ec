// Dslash kernels, Q16F32 storage (16-bit fixed-point spinors, FP32 links and clover).
#include "dslash_inst.cuh"

namespace qpx {

bool launch_dslash_q16f32(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                         cudaStream_t st)
{
  return launch_dslash_p<Q16F32>(recon, epi, achi, sh, a, grid, st);
}

}  // namespace qpx
