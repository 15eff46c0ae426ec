// Drop-in FullSpinor (reference: include/qphix/full_spinor.h): the two
// checkerboard spinors of a full-lattice field, allocated by Geometry.
#pragma once

#include "qphix/geometry.h"

namespace QPhiX
{

template <typename T, int V, int S, bool compress12>
class FullSpinor
{
 public:
  using CBSpinor = typename Geometry<T, V, S, compress12>::FourSpinorBlock;

  explicit FullSpinor(Geometry<T, V, S, compress12> &geom) : _geom(geom)
  {
    _data[0] = geom.allocCBFourSpinor();
    _data[1] = geom.allocCBFourSpinor();
  }
  ~FullSpinor()
  {
    _geom.free(_data[0]);
    _geom.free(_data[1]);
  }
  FullSpinor(const FullSpinor &) = delete;
  FullSpinor &operator=(const FullSpinor &) = delete;

  CBSpinor *getCBData(int cb) const { return _data[cb]; }
  Geometry<T, V, S, compress12> &getGeometry() { return _geom; }

 private:
  Geometry<T, V, S, compress12> &_geom;
  CBSpinor *_data[2];
};

}  // namespace QPhiX
