// pt_fp64.cuh -- FP64 gravity kernels of the reference, for translation units
// compiled with -fmad=false (no contraction: every product and sum rounds
// exactly as the reference's -DUSE_DOUBLE_FP build evaluates it).
//
// The association order of every expression below is the reference's
// (examples/GravityVisitor.h, examples/MultipoleMoments.h); it decides
// bit-for-bit parity, so it is kept as is.
#pragma once

namespace pt {

// GravityVisitor::SPLINE, examples/GravityVisitor.h:87-120.
__device__ __forceinline__ void spline_f64(double r2, double twoh, double& a, double& b) {
  double r = sqrt(r2);
  if (r < twoh) {
    double dih = 2.0 / twoh;
    double u = r * dih;
    if (u < 1.0) {
      a = dih * (7.0 / 5.0 - 2.0 / 3.0 * u * u + 3.0 / 10.0 * u * u * u * u - 1.0 / 10.0 * u * u * u * u * u);
      b = dih * dih * dih * (4.0 / 3.0 - 6.0 / 5.0 * u * u + 1.0 / 2.0 * u * u * u);
    } else {
      double dir = 1.0 / r;
      a = -1.0 / 15.0 * dir +
          dih * (8.0 / 5.0 - 4.0 / 3.0 * u * u + u * u * u - 3.0 / 10.0 * u * u * u * u + 1.0 / 30.0 * u * u * u * u * u);
      b = -1.0 / 15.0 * dir * dir * dir + dih * dih * dih * (8.0 / 3.0 - 3.0 * u + 6.0 / 5.0 * u * u - 1.0 / 6.0 * u * u * u);
    }
  } else {
    a = 1.0 / r;
    b = a * a * a;
  }
}

// GravityVisitor::SPLINEQ, examples/GravityVisitor.h:37-80 (its softened
// branch groups terms exactly like this).
__device__ __forceinline__ void splineq_f64(double invr, double r2, double twoh, double& a, double& b, double& c,
                                            double& d) {
  double dir = invr;
  if (r2 < twoh * twoh) {
    double dih = 2.0 / twoh;
    double u = dih / dir;
    if (u < 1.0) {
      a = dih * (7.0) / 5.0 - 2.0 / 3.0 * u * u + 3.0 / 10.0 * u * u * u * u - 1.0 / 10.0 * u * u * u * u * u;
      b = dih * dih * dih * (4.0) / 3.0 - 6.0 / 5.0 * u * u + 1.0 / 2.0 * u * u * u;
      c = dih * dih * dih * dih * dih * (12.0) / 5.0 - 3.0 / 2.0 * u;
      d = 3.0 / 2.0 * dih * dih * dih * dih * dih * dih * dir;
    } else {
      a = -1.0 / 15.0 * dir + dih * (8.0 / 5.0) - 4.0 / 3.0 * u * u + u * u * u - 3.0 / 10.0 * u * u * u * u +
          1.0 / 30.0 * u * u * u * u * u;
      b = -1.0 / 15.0 * dir * dir * dir + dih * dih * dih * (8.0) / 3.0 - 3.0 * u + 6.0 / 5.0 * u * u -
          1.0 / 6.0 * u * u * u;
      c = -1.0 / 5.0 * dir * dir * dir * dir * dir + 3.0 * dih * dih * dih * dih * dir +
          dih * dih * dih * dih * dih * (-12.0) / 5.0 + 1.0 / 2.0 * u;
      d = -dir * dir * dir * dir * dir * dir * dir + 3.0 * dih * dih * dih * dih * dir * dir * dir -
          1.0 / 2.0 * dih * dih * dih * dih * dih * dih * dir;
    }
  } else {
    a = dir;
    b = a * a * a;
    c = 3.0 * b * a * a;
    d = 5.0 * c * a * a;
  }
}

}  // namespace pt
