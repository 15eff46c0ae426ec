// Drop-in spinor BLAS (reference: include/qphix/blas_new_c.h): QPhiX's
// user-level BLAS on Geometry's host arrays, computed on the device -- each
// call uploads its operands, runs the C-ABI kernel and downloads the result.
// n_blas_simt (OpenMP SIMT threads) and globalSum (the multi-node sum) are
// accepted and have no effect on one GPU.  Inner products are <x, y> =
// sum conj(x) y, as in the reference.
#pragma once

#include "qphix/geometry.h"

namespace QPhiX
{

namespace gpu
{
template <typename FT, int V, int S, bool C>
using Spinor = typename Geometry<FT, V, S, C>::FourSpinorBlock;

// y = a x + b y on host arrays; out (optional) = |y|^2
template <typename FT, int V, int S, bool C>
void host_caxpby(const double a[2], const Spinor<FT, V, S, C> *x, const double b[2], Spinor<FT, V, S, C> *y,
                 const Geometry<FT, V, S, C> &geom, double *norm2 = nullptr)
{
  auto dx = geom.upload_spinor(x);
  auto dy = geom.upload_spinor(y);
  if (norm2)
    check(qphix_gpu_blas_caxpby_norm2(a, dx.get(), b, dy.get(), norm2), "caxpby_norm2");
  else
    check(qphix_gpu_blas_caxpby(a, dx.get(), b, dy.get()), "caxpby");
  geom.download_spinor(dy, y);
}
}  // namespace gpu

// res = src (blas_new_c.h:17-46)
template <typename FT, int V, int S, bool C>
void copySpinor(gpu::Spinor<FT, V, S, C> *res, const gpu::Spinor<FT, V, S, C> *src,
                const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  auto d = geom.upload_spinor(src);
  geom.download_spinor(d, res);
}

// res = 0 (:48-57)
template <typename FT, int V, int S, bool C>
void zeroSpinor(gpu::Spinor<FT, V, S, C> *res, const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  gpu::Field d(geom.lattice(), QPHIX_GPU_SPINOR, Geometry<FT, V, S, C>::device_prec(), 0);
  gpu::check(qphix_gpu_blas_zero(d.get()), "zero");
  geom.download_spinor(d, res);
}

// y = alpha x (:69-99)
template <typename FT, int V, int S, bool C>
void axy(const double alpha, const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y,
         const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {alpha, 0.0}, b[2] = {0.0, 0.0};
  auto dx = geom.upload_spinor(x);
  gpu::Field dy(geom.lattice(), QPHIX_GPU_SPINOR, Geometry<FT, V, S, C>::device_prec(), 0);
  gpu::check(qphix_gpu_blas_zero(dy.get()), "zero");
  gpu::check(qphix_gpu_blas_caxpby(a, dx.get(), b, dy.get()), "axy");
  geom.download_spinor(dy, y);
}

// x = alpha x (:101-111)
template <typename FT, int V, int S, bool C>
void ax(const double alpha, gpu::Spinor<FT, V, S, C> *x, const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {0.0, 0.0}, b[2] = {alpha, 0.0};
  gpu::host_caxpby(a, x, b, x, geom);
}

// y = y + x (:113-123)
template <typename FT, int V, int S, bool C>
void ypeqx(gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y, const Geometry<FT, V, S, C> &geom,
           int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {1.0, 0.0}, b[2] = {1.0, 0.0};
  gpu::host_caxpby(a, x, b, y, geom);
}

// y = y - x (:125-135)
template <typename FT, int V, int S, bool C>
void ymeqx(gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y, const Geometry<FT, V, S, C> &geom,
           int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {-1.0, 0.0}, b[2] = {1.0, 0.0};
  gpu::host_caxpby(a, x, b, y, geom);
}

// y = alpha y + x (:137-155)
template <typename FT, int V, int S, bool C>
void aypx(const double alpha, const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y,
          const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {1.0, 0.0}, b[2] = {alpha, 0.0};
  gpu::host_caxpby(a, x, b, y, geom);
}

// y = alpha x + y (:212-243)
template <typename FT, int V, int S, bool C>
void axpy(const double alpha, const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y,
          const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {alpha, 0.0}, b[2] = {1.0, 0.0};
  gpu::host_caxpby(a, x, b, y, geom);
}

// y = alpha x + beta y (:245-274)
template <typename FT, int V, int S, bool C>
void axpby(const double alpha, const gpu::Spinor<FT, V, S, C> *x, const double beta, gpu::Spinor<FT, V, S, C> *y,
           const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {alpha, 0.0}, b[2] = {beta, 0.0};
  gpu::host_caxpby(a, x, b, y, geom);
}

// n2 = |x|^2 (:276-308)
template <typename FT, int V, int S, bool C>
void norm2Spinor(double &n2, const gpu::Spinor<FT, V, S, C> *x, const Geometry<FT, V, S, C> &geom,
                 int n_blas_simt, bool globalSum = true)
{
  (void)n_blas_simt;
  (void)globalSum;
  auto dx = geom.upload_spinor(x);
  gpu::check(qphix_gpu_blas_norm2(dx.get(), &n2), "norm2");
}

// y = alpha x + y, norm2y = |y|^2 (:310-341)
template <typename FT, int V, int S, bool C>
void axpyNorm2(const double alpha, const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y, double &norm2y,
               const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double a[2] = {alpha, 0.0}, b[2] = {1.0, 0.0};
  gpu::host_caxpby(a, x, b, y, geom, &norm2y);
}

// res = x - y, n2res = |res|^2 (:343-356)
template <typename FT, int V, int S, bool C>
void xmyNorm2Spinor(gpu::Spinor<FT, V, S, C> *res, const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y,
                    double &n2res, const Geometry<FT, V, S, C> &geom, int n_blas_simt, bool globalSum = true)
{
  (void)n_blas_simt;
  (void)globalSum;
  auto dx = geom.upload_spinor(x);
  auto dy = geom.upload_spinor(y);
  gpu::Field dr(geom.lattice(), QPHIX_GPU_SPINOR, Geometry<FT, V, S, C>::device_prec(), 0);
  gpu::check(qphix_gpu_blas_xmy_norm2(dx.get(), dy.get(), dr.get(), &n2res), "xmy_norm2");
  geom.download_spinor(dr, res);
}

// y = x - y, n2res = |y|^2 (:358-395)
template <typename FT, int V, int S, bool C>
void xmy2Norm2Spinor(const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y, double &n2res,
                     const Geometry<FT, V, S, C> &geom, int n_blas_simt, bool globalSum = true)
{
  (void)n_blas_simt;
  (void)globalSum;
  auto dx = geom.upload_spinor(x);
  auto dy = geom.upload_spinor(y);
  gpu::check(qphix_gpu_blas_xmy_norm2(dx.get(), dy.get(), dy.get(), &n2res), "xmy_norm2");
  geom.download_spinor(dy, y);
}

// results = <x, y> (re, im) (:518-569)
template <typename FT, int V, int S, bool C>
void innerProduct(double results[2], const gpu::Spinor<FT, V, S, C> *x, const gpu::Spinor<FT, V, S, C> *y,
                  const Geometry<FT, V, S, C> &geom, int n_blas_simt, bool globalSum = true)
{
  (void)n_blas_simt;
  (void)globalSum;
  auto dx = geom.upload_spinor(x);
  auto dy = geom.upload_spinor(y);
  gpu::check(qphix_gpu_blas_inner_product(dx.get(), dy.get(), results), "inner_product");
}

// results = <x, y> (re, im), |x|^2 (:571-625)
template <typename FT, int V, int S, bool C>
void innerProductNorm(double results[3], const gpu::Spinor<FT, V, S, C> *x, const gpu::Spinor<FT, V, S, C> *y,
                      const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  auto dx = geom.upload_spinor(x);
  auto dy = geom.upload_spinor(y);
  gpu::check(qphix_gpu_blas_inner_product_norm(dx.get(), dy.get(), results), "inner_product_norm");
}

// y = alpha x + y, alpha complex (:694-734)
template <typename FT, int V, int S, bool C>
void caxpySpinor(double alpha[2], const gpu::Spinor<FT, V, S, C> *x, gpu::Spinor<FT, V, S, C> *y,
                 const Geometry<FT, V, S, C> &geom, int n_blas_simt)
{
  (void)n_blas_simt;
  const double b[2] = {1.0, 0.0};
  gpu::host_caxpby(alpha, x, b, y, geom);
}

// spinor_out = scale_factor spinor_in between two Geometries (precisions and
// layouts) of one lattice (:848-909)
template <typename FTOut, int VOut, int SOut, bool CompressOut, typename FTIn, int VIn, bool CompressIn>
void convert(typename Geometry<FTOut, VOut, SOut, CompressOut>::FourSpinorBlock *spinor_out, double scale_factor,
             const typename Geometry<FTIn, VIn, SOut, CompressIn>::FourSpinorBlock *spinor_in,
             const Geometry<FTOut, VOut, SOut, CompressOut> &geom_out,
             const Geometry<FTIn, VIn, SOut, CompressIn> &geom_in, int n_blas_threads)
{
  (void)n_blas_threads;
  auto din = geom_in.upload_spinor(spinor_in);
  // on the input's lattice object (the conversion runs on one stream); the
  // download only needs the output Geometry's host layout
  gpu::Field dout(geom_in.lattice(), QPHIX_GPU_SPINOR, Geometry<FTOut, VOut, SOut, CompressOut>::device_prec(), 0);
  gpu::check(qphix_gpu_field_convert(dout.get(), din.get(), scale_factor), "convert");
  geom_out.download_spinor(dout, spinor_out);
}

}  // namespace QPhiX
