// Drop-in Geometry<FT, V, S, compress12> (reference: include/qphix/geometry.h:
// 115-441, layout types include/qphix_codegen/decl_common.h:9-62).
//
// Same template parameters, constructor signature, accessors and field
// allocators as QPhiX; the host arrays it hands out have QPhiX's blocked SoA
// layout (so packers written for QPhiX keep working), and the object also
// owns the device lattice on which every Dslash / operator / solver call of
// the drop-in headers runs.  V, S and the blocking parameters (By, Bz,
// NCores, Sy, Sz, MinCt) describe the host arrays only; the device uses its
// own coalesced layout.
#pragma once

#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>

#include "qphix/gpu_backend.h"

namespace QPhiX
{

typedef unsigned short half;  // IEEE binary16 bits, as in QPhiX

template <typename T, int V, int S, bool compressP>
struct Types {
  typedef T FourSpinorBlock[3][4][2][S];   // [colour][spin][re/im][soa]
  typedef T TwoSpinorBlock[3][2][2][V];
  typedef T SU3MatrixBlock[8][(compressP ? 2 : 3)][3][2][V];  // [2mu+dir][c][c2][re/im][vec]

  struct CloverBlock {
    T diag1[6][V];
    T off_diag1[15][2][V];
    T diag2[6][V];
    T off_diag2[15][2][V];
  };

  struct FullCloverBlock {
    T block1[6][6][2][V];
    T block2[6][6][2][V];
  };
};

template <typename T, int V, int S, bool compressP>
class Geometry
{
 public:
  typedef T FT;
  static constexpr int veclen = V;
  static constexpr int soalen = S;
  static constexpr bool compress12 = compressP;
  typedef typename Types<T, V, S, compressP>::FourSpinorBlock FourSpinorBlock;
  typedef typename Types<T, V, S, compressP>::TwoSpinorBlock TwoSpinorBlock;
  typedef typename Types<T, V, S, compressP>::SU3MatrixBlock SU3MatrixBlock;
  typedef typename Types<T, V, S, compressP>::CloverBlock CloverBlock;
  typedef typename Types<T, V, S, compressP>::FullCloverBlock FullCloverBlock;

  Geometry(const int latt_size[], int By_, int Bz_, int NCores_, int Sy_, int Sz_, int PadXY_, int PadXYZ_,
           int MinCt_, bool const verbose = false)
      : By(By_), Bz(Bz_), num_cores(NCores_), Sy(Sy_), Sz(Sz_), PadXY(PadXY_), PadXYZ(PadXYZ_), MinCt(MinCt_)
  {
    (void)verbose;
    Nx_ = latt_size[0];
    Ny_ = latt_size[1];
    Nz_ = latt_size[2];
    Nt_ = latt_size[3];
    Nxh_ = Nx_ / 2;
    if (Ny_ % By_ != 0 || Nz_ % Bz_ != 0)
      throw std::domain_error("Local lattice size Ny must be divisible by blocking length By. Same for Nz and Bz.");
    if (V % S != 0) throw std::domain_error("soalen must divide veclen");
    nvecs_ = Nxh_ / S + (Nxh_ % S ? 1 : 0);
    ngy_ = V / S;
    Pxy = nvecs_ * Ny_ + PadXY;
    Pxyz = Pxy * Nz_ + PadXYZ;
    spinor_bytes = (size_t)(Pxyz * Nt_ + 1) * sizeof(FourSpinorBlock);
    gauge_bytes = (size_t)((Pxyz * Nt_ * S) / V) * sizeof(SU3MatrixBlock);
    clover_bytes = (size_t)((Pxyz * Nt_ * S) / V) * sizeof(CloverBlock);
    full_clover_bytes = (size_t)((Pxyz * Nt_ * S) / V) * sizeof(FullCloverBlock);
    gpu::check(qphix_gpu_lattice_create(latt_size, &lat_), "qphix_gpu_lattice_create");
  }

  ~Geometry()
  {
    if (lat_) qphix_gpu_lattice_destroy(lat_);
  }
  Geometry(const Geometry &) = delete;
  Geometry &operator=(const Geometry &) = delete;

  int Nxh() const { return Nxh_; }
  int Nx() const { return Nx_; }
  int Ny() const { return Ny_; }
  int Nz() const { return Nz_; }
  int Nt() const { return Nt_; }
  int nVecs() const { return nvecs_; }
  int nGY() const { return ngy_; }
  int getBy() const { return By; }
  int getBz() const { return Bz; }
  int getSy() const { return Sy; }
  int getSz() const { return Sz; }
  int getPadXY() const { return PadXY; }
  int getPadXYZ() const { return PadXYZ; }
  int getPxy() const { return Pxy; }
  int getPxyz() const { return Pxyz; }
  int getNSIMT() const { return Sy * Sz; }
  int getNumThreads() const { return num_cores * Sy * Sz; }
  int getNumCores() const { return num_cores; }
  int getMinCt() const { return MinCt; }
  int getVolCB() const { return Nxh_ * Ny_ * Nz_ * Nt_; }

  // zero-filled; spinors keep QPhiX's one leading pad block (ptr + 1)
  FourSpinorBlock *allocCBFourSpinor() { return static_cast<FourSpinorBlock *>(alloc(spinor_bytes)) + 1; }
  SU3MatrixBlock *allocCBGauge() { return static_cast<SU3MatrixBlock *>(alloc(gauge_bytes)); }
  CloverBlock *allocCBClov() { return static_cast<CloverBlock *>(alloc(clover_bytes)); }
  FullCloverBlock *allocCBFullClov() { return static_cast<FullCloverBlock *>(alloc(full_clover_bytes)); }

  void free(FourSpinorBlock *p)
  {
    if (p) std::free(p - 1);
  }
  void free(SU3MatrixBlock *p)
  {
    ++gpu::host_field_epoch();
    std::free(p);
  }
  void free(CloverBlock *p)
  {
    ++gpu::host_field_epoch();
    std::free(p);
  }
  void free(FullCloverBlock *p)
  {
    ++gpu::host_field_epoch();
    std::free(p);
  }

  // ---- device side (not part of QPhiX's interface) --------------------------
  qphix_gpu_lattice lattice() const { return lat_; }
  qphix_gpu_host_layout host_layout() const
  {
    qphix_gpu_host_layout l;
    l.kind = QPHIX_GPU_HOST_QPHIX;
    l.ft = gpu::HostType<T>::code;
    l.veclen = V;
    l.soalen = S;
    l.compress12 = compressP ? 1 : 0;
    l.pad_xy = PadXY;
    l.pad_xyz = PadXYZ;
    return l;
  }
  static constexpr int device_prec() { return gpu::HostType<T>::prec; }

  gpu::Field upload_spinor(const FourSpinorBlock *h, int nrhs = 1) const
  {
    gpu::Field f(lat_, QPHIX_GPU_SPINOR, device_prec(), 0, nrhs);
    auto l = host_layout();
    gpu::check(qphix_gpu_field_upload(f.get(), h, &l, -1, -1), "spinor upload");
    return f;
  }
  void download_spinor(const gpu::Field &f, FourSpinorBlock *h) const
  {
    auto l = host_layout();
    gpu::check(qphix_gpu_field_download(f.get(), h, &l, -1), "spinor download");
  }
  // a two-flavour spinor (up, down host arrays) as the device field of two
  // right-hand sides, and back
  gpu::Field upload_flavours(const FourSpinorBlock *const h[2]) const
  {
    gpu::Field f(lat_, QPHIX_GPU_SPINOR, device_prec(), 0, 2);
    auto l = host_layout();
    for (int fl = 0; fl < 2; fl++) gpu::check(qphix_gpu_field_upload(f.get(), h[fl], &l, -1, fl), "spinor upload");
    return f;
  }
  void download_flavours(const gpu::Field &f, FourSpinorBlock *const h[2]) const
  {
    auto l = host_layout();
    for (int fl = 0; fl < 2; fl++) gpu::check(qphix_gpu_field_download(f.get(), h[fl], &l, fl), "spinor download");
  }
  // one gauge field from the two checkerboard arrays QPhiX packs
  gpu::Field upload_gauge(const SU3MatrixBlock *u0, const SU3MatrixBlock *u1) const
  {
    gpu::Field f(lat_, QPHIX_GPU_GAUGE, device_prec(), compressP ? 12 : 18);
    auto l = host_layout();
    gpu::check(qphix_gpu_field_upload(f.get(), u0, &l, 0, -1), "gauge upload (cb 0)");
    gpu::check(qphix_gpu_field_upload(f.get(), u1, &l, 1, -1), "gauge upload (cb 1)");
    return f;
  }
  gpu::Field upload_clover(const CloverBlock *c) const
  {
    gpu::Field f(lat_, QPHIX_GPU_CLOVER, device_prec(), 0);
    auto l = host_layout();
    gpu::check(qphix_gpu_field_upload(f.get(), c, &l, -1, -1), "clover upload");
    return f;
  }
  gpu::Field upload_full_clover(const FullCloverBlock *c) const
  {
    gpu::Field f(lat_, QPHIX_GPU_FULLCLOVER, device_prec(), 0);
    auto l = host_layout();
    gpu::check(qphix_gpu_field_upload(f.get(), c, &l, -1, -1), "full clover upload");
    return f;
  }

 private:
  void *alloc(size_t bytes)
  {
    size_t n = (bytes + 127) / 128 * 128;
    void *p = nullptr;
    if (posix_memalign(&p, 128, n) != 0 || !p) throw std::bad_alloc();
    std::memset(p, 0, n);
    return p;
  }

  int Nx_, Ny_, Nz_, Nt_, Nxh_, nvecs_, ngy_;
  int By, Bz, num_cores, Sy, Sz, PadXY, PadXYZ, MinCt;
  int Pxy, Pxyz;
  size_t spinor_bytes, gauge_bytes, clover_bytes, full_clover_bytes;
  qphix_gpu_lattice lat_ = nullptr;
};

}  // namespace QPhiX
