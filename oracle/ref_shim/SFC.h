/*
 * SFC.h -- stand-in for N-BodyShop/utility's SFC (un-vendored; UNPINNED).
 * TEST INFRASTRUCTURE.  generateKey is the FP64 Morton convention of
 * oracle/pt_sfc.h (21 bits per dimension, x most significant).
 */
#ifndef PT_SHIM_SFC_H_
#define PT_SHIM_SFC_H_
#include <cstdint>
#include "Vector3D.h"
#include "OrientedBox.h"
#include "../pt_sfc.h"

namespace SFC {
typedef uint64_t Key;
template <typename T, typename T2>
inline Key generateKey(const Vector3D<T>& p, const OrientedBox<T2>& box) {
  const double lo[3] = {box.lesser_corner.x, box.lesser_corner.y, box.lesser_corner.z};
  const double hi[3] = {box.greater_corner.x, box.greater_corner.y, box.greater_corner.z};
  return pt_morton_key(p.x, p.y, p.z, lo, hi);
}
}  // namespace SFC
#endif
