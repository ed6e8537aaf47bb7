/*
 * OrientedBox.h -- stand-in for N-BodyShop/utility's OrientedBox
 * (un-vendored).  TEST INFRASTRUCTURE.  An empty box has lesser = +max and
 * greater = -max; grow(box) takes component-wise min/max of the corners, so
 * growing by an empty box is a no-op; center() = (lesser + greater) / 2.
 */
#ifndef PT_SHIM_ORIENTEDBOX_H_
#define PT_SHIM_ORIENTEDBOX_H_

#include <limits>
#include "Vector3D.h"

template <typename T>
class OrientedBox {
 public:
  Vector3D<T> lesser_corner, greater_corner;
  OrientedBox()
      : lesser_corner(std::numeric_limits<T>::max()),
        greater_corner(-std::numeric_limits<T>::max()) {}
  OrientedBox(const Vector3D<T>& l, const Vector3D<T>& g) : lesser_corner(l), greater_corner(g) {}
  void reset() { *this = OrientedBox(); }
  OrientedBox& grow(const Vector3D<T>& p) {
    if (p.x < lesser_corner.x) lesser_corner.x = p.x;
    if (p.y < lesser_corner.y) lesser_corner.y = p.y;
    if (p.z < lesser_corner.z) lesser_corner.z = p.z;
    if (p.x > greater_corner.x) greater_corner.x = p.x;
    if (p.y > greater_corner.y) greater_corner.y = p.y;
    if (p.z > greater_corner.z) greater_corner.z = p.z;
    return *this;
  }
  OrientedBox& grow(const OrientedBox& b) {
    if (b.lesser_corner.x < lesser_corner.x) lesser_corner.x = b.lesser_corner.x;
    if (b.lesser_corner.y < lesser_corner.y) lesser_corner.y = b.lesser_corner.y;
    if (b.lesser_corner.z < lesser_corner.z) lesser_corner.z = b.lesser_corner.z;
    if (b.greater_corner.x > greater_corner.x) greater_corner.x = b.greater_corner.x;
    if (b.greater_corner.y > greater_corner.y) greater_corner.y = b.greater_corner.y;
    if (b.greater_corner.z > greater_corner.z) greater_corner.z = b.greater_corner.z;
    return *this;
  }
  Vector3D<T> size() const { return greater_corner - lesser_corner; }
  Vector3D<T> center() const { return (lesser_corner + greater_corner) / T(2); }
  T volume() const { Vector3D<T> s = size(); return s.x * s.y * s.z; }
};

template <typename T>
inline std::ostream& operator<<(std::ostream& os, const OrientedBox<T>& b) {
  return os << "[" << b.lesser_corner << ", " << b.greater_corner << "]";
}

#endif
