/*
 * pt_sfc.h -- the space-filling-curve key convention shared by the oracle
 * (both the C restatement and the stand-in `SFC.h` that the reference's own
 * sources are compiled against) and mirrored bit-for-bit by the CUDA key
 * kernel.  TEST INFRASTRUCTURE: nothing in the product links this header.
 *
 * The reference calls `SFC::generateKey(position, universe.box)` at
 * src/Decomposition.C:60 and src/Particle.C:88, then ORs in the placeholder
 * bit 63 (src/Decomposition.C:62, src/Particle.C:89).  `generateKey` lives in
 * the un-vendored N-BodyShop/utility submodule (pinned commit unknown: the
 * mount has no git metadata), so the exact bit recipe is UNPINNED.  The
 * published algorithm is a Morton (Z-order) key with 21 bits per dimension
 * (src/common.h:29-31: KEY_BITS=64, BITS_PER_DIM=21) interleaved with x as
 * the most significant bit of every triple.  This file restates it in FP64:
 *
 *   t_d = (p_d - lesser_d) / (greater_d - lesser_d)       (IEEE FP64 divide)
 *   q_d = clamp(floor(t_d * 2^21), 0, 2^21 - 1)
 *   key = sum_b  x_b<<(3b+2) | y_b<<(3b+1) | z_b<<(3b)
 */
#ifndef PT_SFC_H_
#define PT_SFC_H_

#include <stdint.h>

#define PT_KEY_BITS_PER_DIM 21
#define PT_KEY_PLACEHOLDER (((uint64_t)1) << 63)

static inline uint64_t pt_spread21(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x001f00000000ffffull;
  v = (v | (v << 16)) & 0x001f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

static inline uint32_t pt_quantize21(double p, double lo, double hi) {
  double t = (p - lo) / (hi - lo);
  double s = t * 2097152.0;
  if (!(s >= 0.0)) return 0u; /* negative (and NaN, rejected earlier) */
  if (s >= 2097151.0) return 2097151u;
  return (uint32_t)s;
}

/* Morton key without the placeholder bit (bits 0..62). */
static inline uint64_t pt_morton_key(double x, double y, double z,
                                     const double lo[3], const double hi[3]) {
  uint64_t qx = pt_quantize21(x, lo[0], hi[0]);
  uint64_t qy = pt_quantize21(y, lo[1], hi[1]);
  uint64_t qz = pt_quantize21(z, lo[2], hi[2]);
  return (pt_spread21(qx) << 2) | (pt_spread21(qy) << 1) | pt_spread21(qz);
}

#endif /* PT_SFC_H_ */
