/*
 * Space.h -- stand-in for N-BodyShop/utility's Space (un-vendored; the
 * boundary convention is UNPINNED).  TEST INFRASTRUCTURE.  Chosen
 * convention, mirrored by the CUDA traversal:
 *   box/sphere:    dsq = sum over x,y,z of the squared gap outside the box
 *                  (accumulated x, then y, then z); intersect iff dsq <= rsq
 *   sphere/sphere: intersect iff |c1 - c2|^2 <= (r1 + r2)^2
 *   enclose(a, b): b lies inside a (closed box)
 */
#ifndef PT_SHIM_SPACE_H_
#define PT_SHIM_SPACE_H_
#include "OrientedBox.h"
#include "Sphere.h"

namespace Space {
template <typename T, typename T2>
inline bool intersect(const OrientedBox<T>& b, const Vector3D<T2>& c, double rsq) {
  double dsq = 0.0, d;
  if ((d = b.lesser_corner.x - c.x) > 0) dsq += d * d;
  else if ((d = c.x - b.greater_corner.x) > 0) dsq += d * d;
  if ((d = b.lesser_corner.y - c.y) > 0) dsq += d * d;
  else if ((d = c.y - b.greater_corner.y) > 0) dsq += d * d;
  if ((d = b.lesser_corner.z - c.z) > 0) dsq += d * d;
  else if ((d = c.z - b.greater_corner.z) > 0) dsq += d * d;
  return dsq <= rsq;
}
template <typename T, typename T2>
inline bool intersect(const OrientedBox<T>& b, const Sphere<T2>& s) {
  return intersect(b, s.origin, s.radius * s.radius);
}
template <typename T>
inline bool intersect(const Sphere<T>& a, const Sphere<T>& b) {
  T rs = a.radius + b.radius;
  return (a.origin - b.origin).lengthSquared() <= rs * rs;
}
template <typename T>
inline bool enclose(const OrientedBox<T>& a, const OrientedBox<T>& b) {
  return a.lesser_corner.x <= b.lesser_corner.x && a.lesser_corner.y <= b.lesser_corner.y &&
         a.lesser_corner.z <= b.lesser_corner.z && a.greater_corner.x >= b.greater_corner.x &&
         a.greater_corner.y >= b.greater_corner.y && a.greater_corner.z >= b.greater_corner.z;
}
}  // namespace Space
#endif
