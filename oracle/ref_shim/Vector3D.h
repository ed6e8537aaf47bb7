/*
 * Vector3D.h -- stand-in for N-BodyShop/utility's Vector3D (un-vendored).
 * TEST INFRASTRUCTURE.  Every operation is component-wise and evaluates in
 * the obvious order: lengthSquared = (x*x + y*y) + z*z, dot likewise,
 * v / s divides each component by s (no reciprocal), s * v multiplies each
 * component.  The CUDA kernels and the C restatement follow this order.
 */
#ifndef PT_SHIM_VECTOR3D_H_
#define PT_SHIM_VECTOR3D_H_

#include <cmath>
#include <ostream>
#include "charm_stub.h"

template <typename T>
class Vector3D {
 public:
  T x, y, z;
  Vector3D() : x(0), y(0), z(0) {}
  Vector3D(T v) : x(v), y(v), z(v) {}
  Vector3D(T a, T b, T c) : x(a), y(b), z(c) {}
  template <typename U>
  Vector3D(const Vector3D<U>& o) : x(o.x), y(o.y), z(o.z) {}

  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }

  T lengthSquared() const { return x * x + y * y + z * z; }
  T length() const { return std::sqrt(lengthSquared()); }

  Vector3D operator+(const Vector3D& o) const { return Vector3D(x + o.x, y + o.y, z + o.z); }
  Vector3D operator-(const Vector3D& o) const { return Vector3D(x - o.x, y - o.y, z - o.z); }
  Vector3D operator-() const { return Vector3D(-x, -y, -z); }
  Vector3D operator*(T s) const { return Vector3D(x * s, y * s, z * s); }
  Vector3D operator/(T s) const { return Vector3D(x / s, y / s, z / s); }
  Vector3D& operator+=(const Vector3D& o) { x += o.x; y += o.y; z += o.z; return *this; }
  Vector3D& operator-=(const Vector3D& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  Vector3D& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
  Vector3D& operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
};

template <typename T>
inline Vector3D<T> operator*(T s, const Vector3D<T>& v) { return Vector3D<T>(s * v.x, s * v.y, s * v.z); }

template <typename T>
inline T dot(const Vector3D<T>& a, const Vector3D<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

template <typename T>
inline std::ostream& operator<<(std::ostream& os, const Vector3D<T>& v) {
  return os << "(" << v.x << ", " << v.y << ", " << v.z << ")";
}

#endif
