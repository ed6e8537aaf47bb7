// pt_f32.cuh -- FP32 forms of the reference's softening kernels, shared by
// the mixed-precision traversals (k_mixed.cu, k_mixed2.cu).
#pragma once

namespace pt {

// SPLINE in FP32, softened branch (r < twoh): kept out of line so that the
// rarely taken polynomial does not raise register pressure in the hot loops.
static __device__ __noinline__ void spline_f32_soft(float r2, float rinv, float twoh, float& a, float& b) {
  float r = r2 * rinv;
  float dih = 2.0f / twoh;
  float u = r * dih;
  float u2 = u * u;
  if (u < 1.0f) {
    a = dih * (7.0f / 5.0f - 2.0f / 3.0f * u2 + 3.0f / 10.0f * u2 * u2 - 1.0f / 10.0f * u2 * u2 * u);
    b = dih * dih * dih * (4.0f / 3.0f - 6.0f / 5.0f * u2 + 1.0f / 2.0f * u2 * u);
  } else {
    a = -1.0f / 15.0f * rinv +
        dih * (8.0f / 5.0f - 4.0f / 3.0f * u2 + u2 * u - 3.0f / 10.0f * u2 * u2 + 1.0f / 30.0f * u2 * u2 * u);
    b = -1.0f / 15.0f * rinv * rinv * rinv +
        dih * dih * dih * (8.0f / 3.0f - 3.0f * u + 6.0f / 5.0f * u2 - 1.0f / 6.0f * u2 * u);
  }
}

// SPLINE in FP32 (r2 > 0): force term b, potential term a.
static __device__ __forceinline__ void spline_f32(float r2, float rinv, float twoh, float& a, float& b) {
  if (r2 < twoh * twoh) {
    spline_f32_soft(r2, rinv, twoh, a, b);
  } else {
    a = rinv;
    b = rinv * rinv * rinv;
  }
}

// SPLINEQ in FP32 with the reference's grouping (examples/GravityVisitor.h:37-80);
// only the softened branch is called (out of line, rarely taken).
static __device__ __noinline__ void splineq_f32(float dir, float r2, float twoh, float& a, float& b, float& c, float& d) {
  if (r2 < twoh * twoh) {
    float dih = 2.0f / twoh;
    float u = dih / dir;
    float u2 = u * u;
    float d2 = dih * dih, d3 = d2 * dih, d4 = d3 * dih, d5 = d4 * dih, d6 = d5 * dih;
    if (u < 1.0f) {
      a = dih * 7.0f / 5.0f - 2.0f / 3.0f * u2 + 3.0f / 10.0f * u2 * u2 - 1.0f / 10.0f * u2 * u2 * u;
      b = d3 * 4.0f / 3.0f - 6.0f / 5.0f * u2 + 1.0f / 2.0f * u2 * u;
      c = d5 * 12.0f / 5.0f - 3.0f / 2.0f * u;
      d = 3.0f / 2.0f * d6 * dir;
    } else {
      float r3 = dir * dir * dir;
      a = -1.0f / 15.0f * dir + dih * (8.0f / 5.0f) - 4.0f / 3.0f * u2 + u2 * u - 3.0f / 10.0f * u2 * u2 +
          1.0f / 30.0f * u2 * u2 * u;
      b = -1.0f / 15.0f * r3 + d3 * 8.0f / 3.0f - 3.0f * u + 6.0f / 5.0f * u2 - 1.0f / 6.0f * u2 * u;
      c = -1.0f / 5.0f * r3 * dir * dir + 3.0f * d4 * dir + d5 * (-12.0f) / 5.0f + 1.0f / 2.0f * u;
      d = -r3 * r3 * dir + 3.0f * d4 * r3 - 1.0f / 2.0f * d6 * dir;
    }
  } else {
    a = dir;
    b = a * a * a;
    c = 3.0f * b * a * a;
    d = 5.0f * c * a * a;
  }
}

}  // namespace pt
