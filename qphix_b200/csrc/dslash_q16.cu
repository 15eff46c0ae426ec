// Dslash kernels, Q16 storage (16-bit fixed-point spinors, FP16 links and clover).
#include "dslash_inst.cuh"

namespace qpx {

bool launch_dslash_q16(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                      cudaStream_t st)
{
  return launch_dslash_p<Q16>(recon, epi, achi, sh, a, grid, st);
}

}  // namespace qpx
