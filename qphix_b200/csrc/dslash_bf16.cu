// Dslash kernels, BF16 storage.
#include "dslash_inst.cuh"

namespace qpx {

bool launch_dslash_bf16(int recon, int epi, int achi, const DslashShape &sh, const DslashArgs *a, dim3 grid,
                     cudaStream_t st)
{
  return launch_dslash_p<BF16>(recon, epi, achi, sh, a, grid, st);
}

}  // namespace qpx
