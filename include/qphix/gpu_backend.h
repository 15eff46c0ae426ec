// Shared plumbing of the QPhiX drop-in headers: status-code checking, RAII
// handles and the host-layout descriptor of a Geometry's arrays.  The headers
// in this directory keep QPhiX's class templates (same names, constructor
// signatures, member functions and host array layouts) and run every
// operation on the GPU through the C ABI in qphix_b200.h.
#pragma once

#include <atomic>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../qphix_b200.h"

namespace QPhiX
{
namespace gpu
{

// QPhiX aborts on misuse; the drop-in throws instead (the library itself
// never aborts).
inline void check(int rc, const char *what)
{
  if (rc != QPHIX_GPU_OK && rc != QPHIX_GPU_ENOTCONV && rc != QPHIX_GPU_EBREAKDOWN) {
    throw std::runtime_error(std::string(what) + ": " + qphix_gpu_last_error());
  }
}

template <typename FT>
struct HostType;
template <>
struct HostType<double> {
  static constexpr int code = QPHIX_GPU_HOST_F64;
  static constexpr int prec = QPHIX_GPU_F64;
};
template <>
struct HostType<float> {
  static constexpr int code = QPHIX_GPU_HOST_F32;
  static constexpr int prec = QPHIX_GPU_F32;
};
template <>
struct HostType<unsigned short> {  // QPhiX's `half` (IEEE binary16 bits)
  static constexpr int code = QPHIX_GPU_HOST_F16;
  static constexpr int prec = QPHIX_GPU_F16;
};

// owning device field handle
class Field
{
 public:
  Field() = default;
  Field(qphix_gpu_lattice lat, int kind, int prec, int recon, int nrhs = 1)
  {
    check(qphix_gpu_field_create(lat, kind, prec, recon, nrhs, &h_), "qphix_gpu_field_create");
  }
  Field(const Field &) = delete;
  Field &operator=(const Field &) = delete;
  Field(Field &&o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  Field &operator=(Field &&o) noexcept
  {
    reset();
    h_ = o.h_;
    o.h_ = nullptr;
    return *this;
  }
  ~Field() { reset(); }
  void reset()
  {
    if (h_) qphix_gpu_field_destroy(h_);
    h_ = nullptr;
  }
  qphix_gpu_field get() const { return h_; }
  explicit operator bool() const { return h_ != nullptr; }

 private:
  qphix_gpu_field h_ = nullptr;
};

// Host gauge / clover arrays released through Geometry::free bump this
// counter, so a device copy cached under an array's address is never reused
// for a later allocation that lands at the same address.
inline std::atomic<unsigned long> &host_field_epoch()
{
  static std::atomic<unsigned long> epoch{0};
  return epoch;
}

// Device copies of the operator fields (gauge checkerboards, clover terms) a
// Dslash object was handed, kept across its calls while the host array's
// address and host_field_epoch() are unchanged: a caller that applies the
// Dslash in a loop uploads its links once.  A caller that rewrites such an
// array in place calls clear() (Dslash::invalidateFieldCache()).
class FieldCache
{
 public:
  template <typename Make>
  qphix_gpu_field get(const void *host, int tag, Make &&make)
  {
    const unsigned long ep = host_field_epoch().load();
    for (auto &e : entries_)
      if (e.host == host && e.tag == tag && e.epoch == ep) return e.f.get();
    std::vector<Entry> keep;  // drop copies of an older epoch
    for (auto &e : entries_)
      if (e.epoch == ep) keep.push_back(std::move(e));
    entries_ = std::move(keep);
    if (entries_.size() >= kMax) entries_.erase(entries_.begin());
    entries_.push_back(Entry{host, tag, ep, make()});
    return entries_.back().f.get();
  }
  void clear() { entries_.clear(); }

 private:
  static constexpr size_t kMax = 8;
  struct Entry {
    const void *host;
    int tag;
    unsigned long epoch;
    Field f;
  };
  std::vector<Entry> entries_;
};

class EoOp
{
 public:
  EoOp() = default;
  EoOp(const EoOp &) = delete;
  EoOp &operator=(const EoOp &) = delete;
  ~EoOp() { reset(); }
  void reset()
  {
    if (h_) qphix_gpu_eo_op_destroy(h_);
    h_ = nullptr;
  }
  void create(const qphix_gpu_op_params &p, qphix_gpu_field u, qphix_gpu_field clov, qphix_gpu_field invclov,
              qphix_gpu_field f0, qphix_gpu_field f1)
  {
    reset();
    check(qphix_gpu_eo_op_create(&p, u, clov, invclov, f0, f1, &h_), "qphix_gpu_eo_op_create");
  }
  qphix_gpu_eo_op get() const { return h_; }

 private:
  qphix_gpu_eo_op h_ = nullptr;
};

inline qphix_gpu_op_params make_params(int kind, double t_boundary, double aniso_s, double aniso_t,
                                       const bool *use_tbc, const double (*tbc_phases)[2], double mass = 0.0,
                                       double twisted_mass = 0.0, double rho = 0.0)
{
  qphix_gpu_op_params p;
  std::memset(&p, 0, sizeof(p));
  p.kind = kind;
  p.t_boundary = t_boundary;
  p.aniso_s = aniso_s;
  p.aniso_t = aniso_t;
  for (int d = 0; d < 4; d++) {
    p.tbc_phases[d][0] = 1.0;
    p.tbc_phases[d][1] = 0.0;
  }
  if (use_tbc && tbc_phases) {
    for (int d = 0; d < 4; d++) {
      p.use_tbc[d] = use_tbc[d] ? 1 : 0;
      p.tbc_phases[d][0] = tbc_phases[d][0];
      p.tbc_phases[d][1] = tbc_phases[d][1];
    }
  }
  p.mass = mass;
  p.twisted_mass = twisted_mass;
  p.prec_mass_rho = rho;
  return p;
}

}  // namespace gpu
}  // namespace QPhiX
