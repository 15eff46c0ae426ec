// Persistent CG kernels, F64 storage (qpx_persist.cuh): Wilson and clover
// even-odd operators, 12- and 18-real links, isign = +1.
#include "qpx_host.h"
#include "qpx_persist.cuh"

namespace qpx {

const void *cg_persistent_kernel_f64(int recon, bool clover)
{
  if (recon == 12)
    return clover ? (const void *)cg_persistent_kernel<F64, 12, EPI_CLOV, ACHI_CLOV, 1>
                  : (const void *)cg_persistent_kernel<F64, 12, EPI_NONE, ACHI_ALPHA, 1>;
  if (recon == 18)
    return clover ? (const void *)cg_persistent_kernel<F64, 18, EPI_CLOV, ACHI_CLOV, 1>
                  : (const void *)cg_persistent_kernel<F64, 18, EPI_NONE, ACHI_ALPHA, 1>;
  return nullptr;
}

}  // namespace qpx
