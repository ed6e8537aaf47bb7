/* Sphere.h -- stand-in for N-BodyShop/utility's Sphere.  TEST INFRASTRUCTURE. */
#ifndef PT_SHIM_SPHERE_H_
#define PT_SHIM_SPHERE_H_
#include "Vector3D.h"
template <typename T>
class Sphere {
 public:
  Vector3D<T> origin;
  T radius;
  Sphere() : origin(0), radius(0) {}
  Sphere(const Vector3D<T>& o, T r) : origin(o), radius(r) {}
};
#endif
