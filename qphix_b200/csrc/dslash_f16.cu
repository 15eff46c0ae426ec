// Dslash kernels, F16 storage.
#include "dslash_inst.cuh"

namespace qpx {

void launch_dslash_f16(int recon, int epi, int achi, int R, const DslashArgs &a, dim3 grid, cudaStream_t st)
{
  switch (R) {
  case 1: launch_dslash_r<F16, 1>(recon, epi, achi, a, grid, st); return;
  case 2: launch_dslash_r<F16, 2>(recon, epi, achi, a, grid, st); return;
  }
  throw Error(QPHIX_GPU_EINVAL, "unsupported rhs tile for F16");
}

}  // namespace qpx
