/*
 * charm_stub.h -- minimal stand-ins for the Charm++ names that the
 * reference's gravity headers mention in declarations only (PUP::er,
 * CkVec, CkAssert, CkReduction).  TEST INFRASTRUCTURE: lets the oracle
 * compile the reference's own GravityVisitor.h / CentroidData.h /
 * MultipoleMoments.h / Node.h / Particle.{h,C} without Charm++.
 */
#ifndef PT_SHIM_CHARM_STUB_H_
#define PT_SHIM_CHARM_STUB_H_

#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <limits>
#include <functional>
#include <iostream>
#include <cinttypes>

#define CkAssert(x) assert(x)
#define CkAbort(msg) (std::fprintf(stderr, "%s\n", msg), std::abort())
#define CkPrintf(...) std::fprintf(stderr, __VA_ARGS__)

namespace PUP {
class er {
 public:
  bool isUnpacking() const { return false; }
  bool isPacking() const { return false; }
  template <typename T>
  void operator()(T*, int) {}
};
template <typename T>
inline void operator|(er&, T&) {}
}  // namespace PUP

template <typename T>
using CkVec = std::vector<T>;

class CkReductionMsg;
namespace CkReduction {
typedef int reducerType;
typedef CkReductionMsg* (*reducerFn)(int, CkReductionMsg**);
inline reducerType addReducer(reducerFn) { return 0; }
}  // namespace CkReduction

#endif
