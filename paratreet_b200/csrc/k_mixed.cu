// k_mixed.cu -- K7 mixed-precision traversal.
//
// Same interactions as the FP64 form: the tree, the opening tests
// (GravityVisitor::open) and the softening-overlap tests
// (GravityVisitor::openSoftening) are evaluated in FP64 with the same
// expressions, so every bucket meets exactly the reference's set of leaf()
// and node() interactions.  Every P2P (GravityVisitor::leaf,
// examples/GravityVisitor.h:144-160) and P2C (GravityVisitor::node, :184-224)
// interaction is evaluated in FP32 on offsets relative to the target bucket's
// centre of mass:
//   targets   (x_i - cm_bucket)                      FP64 subtract -> FP32
//   sources   (x_j - cm_leaf) [FP32, once per pass] + (cm_leaf - cm_bucket)
//             [FP64 subtract per (leaf, bucket) -> FP32]
//   P2C       (x_i - cm_bucket) - (cm_node - cm_bucket) [FP64 -> FP32]
// Terms are summed in plain FP32 within one flush of the interaction buffers
// (<= 64 entries) and the flush partials are Kahan-added into per-target FP32
// accumulators.  Acceleration and the full potential are produced.
//
// B200 mapping (one warp per bucket, dynamic bucket queue in DFS order):
//  walk     lanes 8e..8e+7 classify the 8 children of up to 4 opened nodes at
//           once (32 FP64 tests per step); leaves and accepted nodes are
//           appended to shared-memory buffers with their FP32 offsets, opened
//           nodes to a per-warp LIFO.  The interaction order is not the
//           reference's (only the FP64 form keeps it).
//  eval     the bucket's n_t targets are replicated over G = floor(32 / n_t)
//           lane groups; group g takes every G-th source pair / node pair of
//           a 64-entry chunk staged in shared memory as interleaved pairs, so
//           a 10-particle bucket keeps 30 lanes busy and each lane evaluates
//           two interactions per packed FP32 instruction (f32x2 add / mul /
//           fma, two operations per issue slot).  Leaves whose nearest
//           particle pair is provably beyond the softening length take a
//           branch-free Newtonian loop (rsqrt on the SFU).  The flushes are
//           out-of-line functions (targets in, partial sums out by value) so
//           that their loops get the register budget the walk state would
//           otherwise hold.
//  reduce   per-lane Kahan sums -> FP64, sum over the G groups.
#include "pt_internal.cuh"
#include "pt_walk.cuh"
#include "pt_f32.cuh"

namespace pt {

constexpr int kMixWarps = 4;
constexpr int kMixStack = 640;  // opened nodes pending; <= 21 levels x 28 + 32
constexpr int kMixBuf = 64;     // buffered terminals per kind (a step adds <= 32)

struct Kahan {
  float s, c;
  __device__ __forceinline__ void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// Per-warp shared memory.
struct MixWarp {
  BucketGeom geom;          // the target bucket (FP64), read by the walk
  int32_t stack[kMixStack];
  float4 cbuf[kMixBuf];     // P2C: offset xyz, node index bits (mono: node | 1<<31)
  float4 pbuf[kMixBuf];     // P2P leaves: offset xyz, node index bits; far leaves
                            // fill from the front, near leaves from the back
  float kahan[8][32];       // per-lane compensated sums (s, c) of ax, ay, az, pot
  int32_t pre[kMixBuf + 1]; // prefix of leaf sizes during a P2P flush
  int32_t ps0[kMixBuf];     // first particle of each buffered leaf
  float4 px[32];            // staged source pairs: x_a, x_b, y_a, y_b (rel. bucket)
  float4 pz[32];            // z_a, z_b, m_a, m_b
  float4 pr[32];            // near leaves: reach2_a, reach2_b, soft_a, soft_b; beyond
                            // reach2 = (soft_j + max bucket softening)^2 a pair is unsoftened
  float4 qp[6][32];         // staged P2C node pairs (see flush_p2c)
};

__device__ __forceinline__ float4 pack_entry(float ox, float oy, float oz, int node, bool flag) {
  return make_float4(ox, oy, oz, __int_as_float(node | (flag ? (int)0x80000000 : 0)));
}
__device__ __forceinline__ int entry_node(float4 e) { return __float_as_int(e.w) & 0x7fffffff; }
__device__ __forceinline__ bool entry_flag(float4 e) { return (__float_as_int(e.w) & 0x80000000) != 0; }

struct MixCtx {
  int lane, t, grp, G, nt;
  float tx, ty, tz, ts;                 // this lane's target (rel. bucket cm)
  float pax, pay, paz, ppf;             // flush partials
  float (*kah)[32];                     // this warp's compensated sums in shared memory
  unsigned n_src, n_node;               // sources / nodes evaluated for this target chunk

  // Kahan-add the flush partials into the lane's compensated sums.
  __device__ __forceinline__ void commit() {
    const float v[4] = {pax, pay, paz, ppf};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      Kahan q{kah[2 * k][lane], kah[2 * k + 1][lane]};
      q.add(v[k]);
      kah[2 * k][lane] = q.s;
      kah[2 * k + 1][lane] = q.c;
    }
    pax = pay = paz = ppf = 0.f;
  }
};

// One source of a near leaf: Newtonian beyond the softening reach, the spline
// inside it, nothing for the particle itself (r2 == 0).  pp sums +m a.
__device__ __forceinline__ void near_pair(float m, float dx, float dy, float dz, float r2, float reach2,
                                          float ssoft, float ts, float& ax, float& ay, float& az, float& pp) {
  if (r2 > reach2) {
    const float rinv = rsqrtf(r2);
    const float mr = m * rinv;
    const float mr3 = mr * rinv * rinv;
    ax += dx * mr3;
    ay += dy * mr3;
    az += dz * mr3;
    pp += mr;
  } else if (r2 > 0.f) {
    const float rinv = rsqrtf(r2);
    float a, b;
    spline_f32(r2, rinv, ssoft + ts, a, b);
    const float bm = b * m;
    ax += dx * bm;
    ay += dy * bm;
    az += dz * bm;
    pp += m * a;
  }
}

// Evaluate all buffered P2P leaves of one kind (far: no pair can be softened).
// Sources are staged 64 per chunk as 32 interleaved pairs, px = (x_a, x_b,
// y_a, y_b), pz = (z_a, z_b, m_a, m_b): each half of a 128-bit shared load is
// an aligned register pair, so a lane evaluates two sources against its
// target with the packed FP32 instructions (two FP32 operations per issue).
// Missing sources of the last pair have zero mass at a far position.
struct FlushIn {
  float tx, ty, tz, ts;
  int lane, grp, G;
};
template <bool kFar>
__device__ __noinline__ float4 flush_p2p_nl(MixWarp& w, const float4* __restrict__ buf, int nleaves,
                                            const WalkRec* __restrict__ walk, const float4* __restrict__ srcf,
                                            const float* __restrict__ softf, const FlushIn x, int& total_out) {
  // prefix of leaf sizes (nleaves <= 64: two entries per lane)
  int s0a = 0, s0b = 0, na = 0, nb = 0;
  if (x.lane < nleaves) { const WalkRec& r = walk[entry_node(buf[x.lane])]; s0a = r.pstart; na = r.pcount; }
  if (x.lane + 32 < nleaves) { const WalkRec& r = walk[entry_node(buf[x.lane + 32])]; s0b = r.pstart; nb = r.pcount; }
  int inca = na, incb = nb;
  for (int o = 1; o < 32; o <<= 1) {
    int ya = __shfl_up_sync(kFull, inca, o), yb = __shfl_up_sync(kFull, incb, o);
    if (x.lane >= o) { inca += ya; incb += yb; }
  }
  const int tota = __shfl_sync(kFull, inca, 31);
  const int total = tota + __shfl_sync(kFull, incb, 31);
  __syncwarp();
  if (x.lane < nleaves) { w.pre[x.lane] = inca - na; w.ps0[x.lane] = s0a; }
  if (x.lane + 32 < nleaves) { w.pre[x.lane + 32] = tota + incb - nb; w.ps0[x.lane + 32] = s0b; }
  if (x.lane == 0) w.pre[nleaves] = total;
  __syncwarp();
  const float kPadPos = 1.0e10f;
  int base_leaf = 0;  // leaf holding the next chunk's first source
  float4 ra, rb, oa, ob;
  float sa = 0.f, sb = 0.f;
  auto fetch = [&](int cs) {
    const int q0 = cs + 2 * x.lane;
    int lo = base_leaf;  // last leaf with pre <= q: a chunk spans few leaves
    while (lo + 1 < nleaves && w.pre[lo + 1] <= q0) lo++;
    int lo1 = lo;
    while (lo1 + 1 < nleaves && w.pre[lo1 + 1] <= q0 + 1) lo1++;
    base_leaf = __shfl_sync(kFull, lo1, 31);
    ra = rb = make_float4(kPadPos, kPadPos, kPadPos, 0.f);
    oa = ob = make_float4(0.f, 0.f, 0.f, 0.f);
    sa = sb = 0.f;
    if (q0 < total) {
      oa = buf[lo];
      const int j = w.ps0[lo] + (q0 - w.pre[lo]);
      ra = srcf[j];
      if (!kFar) sa = softf[j];
    }
    if (q0 + 1 < total) {
      ob = buf[lo1];
      const int j = w.ps0[lo1] + (q0 + 1 - w.pre[lo1]);
      rb = srcf[j];
      if (!kFar) sb = softf[j];
    }
  };
  fetch(0);
  const float2 ntx = make_float2(-x.tx, -x.tx), nty = make_float2(-x.ty, -x.ty), ntz = make_float2(-x.tz, -x.tz);
  float2 ax2 = make_float2(0.f, 0.f), ay2 = ax2, az2 = ax2, pp2 = ax2;  // pp2 sums +m/r
  for (int cs = 0; cs < total; cs += 64) {
    w.px[x.lane] = make_float4(ra.x + oa.x, rb.x + ob.x, ra.y + oa.y, rb.y + ob.y);
    w.pz[x.lane] = make_float4(ra.z + oa.z, rb.z + ob.z, ra.w, rb.w);
    if (!kFar) {
      const float gs = (float)w.geom.soft_max;
      const float qa = sa + gs, qb = sb + gs;
      // a padded source (zero mass) takes the Newtonian branch
      w.pr[x.lane] = make_float4(ra.w != 0.f ? qa * qa : -1.f, rb.w != 0.f ? qb * qb : -1.f, sa, sb);
    }
    __syncwarp();
    if (cs + 64 < total) fetch(cs + 64);
    const int np = (min(64, total - cs) + 1) >> 1;
    if (x.grp < x.G) {
      for (int k = x.grp; k < np; k += x.G) {
        const float4 X = w.px[k], Z = w.pz[k];
        const float2 dx = __fadd2_rn(make_float2(X.x, X.y), ntx);
        const float2 dy = __fadd2_rn(make_float2(X.z, X.w), nty);
        const float2 dz = __fadd2_rn(make_float2(Z.x, Z.y), ntz);
        float2 r2 = __fmul2_rn(dx, dx);
        r2 = __ffma2_rn(dy, dy, r2);
        r2 = __ffma2_rn(dz, dz, r2);
        bool fast = true;
        float4 R;
        if (!kFar) {
          R = w.pr[k];
          fast = (r2.x > R.x) && (r2.y > R.y);
        }
        if (fast) {
          const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
          const float2 mr = __fmul2_rn(make_float2(Z.z, Z.w), ri);
          const float2 mr3 = __fmul2_rn(mr, __fmul2_rn(ri, ri));
          ax2 = __ffma2_rn(dx, mr3, ax2);
          ay2 = __ffma2_rn(dy, mr3, ay2);
          az2 = __ffma2_rn(dz, mr3, az2);
          pp2 = __fadd2_rn(pp2, mr);
        } else {
          near_pair(Z.z, dx.x, dy.x, dz.x, r2.x, R.x, R.z, x.ts, ax2.x, ay2.x, az2.x, pp2.x);
          near_pair(Z.w, dx.y, dy.y, dz.y, r2.y, R.y, R.w, x.ts, ax2.y, ay2.y, az2.y, pp2.y);
        }
      }
    }
    __syncwarp();
  }
  total_out = total;
  return make_float4(ax2.x + ax2.y, ay2.x + ay2.y, az2.x + az2.y, -(pp2.x + pp2.y));
}
template <bool kFar>
__device__ __forceinline__ void flush_p2p(MixWarp& w, const float4* __restrict__ buf, int nleaves,
                                          const WalkRec* __restrict__ walk, const float4* __restrict__ srcf,
                                          const float* __restrict__ softf, MixCtx& x) {
  int total = 0;
  const float4 v = flush_p2p_nl<kFar>(w, buf, nleaves, walk, srcf, softf,
                                      FlushIn{x.tx, x.ty, x.tz, x.ts, x.lane, x.grp, x.G}, total);
  x.pax += v.x; x.pay += v.y; x.paz += v.z; x.ppf += v.w;
  x.n_src += (unsigned)total;
  x.commit();
}

// One P2C term (quadrupole, examples/GravityVisitor.h:207-220, in FP32).
// A monopole entry (openSoftening held, addGravity :130-139) is staged with
// zero second moments and a NaN softening, which takes the unsoftened branch
// and reduces the expression to -M r / r^3 and -M / r.
__device__ __forceinline__ void p2c_term(const float4 A, const float4 B, const float4 Cc, float tx, float ty,
                                         float tz, float ts, float& ax, float& ay, float& az, float& pf) {
  const float rx = tx - A.x, ry = ty - A.y, rz = tz - A.z;
  const float r2 = rx * rx + ry * ry + rz * rz;
  const float dir = rsqrtf(r2);
  float a, b, c, d;
  const float twoh = Cc.z + ts;
  if (r2 < twoh * twoh) {
    splineq_f32(dir, r2, twoh, a, b, c, d);
  } else {
    a = dir;
    const float d2 = dir * dir;
    b = a * d2;
    c = 3.0f * b * d2;
    d = 5.0f * c * d2;
  }
  const float qx = B.x * rx + B.y * ry + B.z * rz;
  const float qy = B.y * rx + B.w * ry + Cc.x * rz;
  const float qz = B.z * rx + Cc.x * ry + Cc.y * rz;
  const float qir = 0.5f * (qx * rx + qy * ry + qz * rz);
  const float qir3 = b * A.w + d * qir - c * Cc.w;
  pf += -A.w * a - c * qir + b * Cc.w;
  ax += -qir3 * rx + c * qx;
  ay += -qir3 * ry + c * qy;
  az += -qir3 * rz + c * qz;
}

// Both terms of a staged node pair in scalar form (the rare softened case);
// out of line so that it adds no registers to the packed loop.
__device__ __noinline__ float4 p2c_pair_scalar(const MixWarp& w, int k, float tx, float ty, float tz, float ts) {
  const float4 P0 = w.qp[0][k], P1 = w.qp[1][k], P2 = w.qp[2][k], P3 = w.qp[3][k], P4 = w.qp[4][k],
               P5 = w.qp[5][k];
  float ax = 0.f, ay = 0.f, az = 0.f, pf = 0.f;
  p2c_term(make_float4(P0.x, P0.z, P1.x, P1.z), make_float4(P2.x, P2.z, P3.x, P3.z),
           make_float4(P4.x, P4.z, P5.x, P5.z), tx, ty, tz, ts, ax, ay, az, pf);
  p2c_term(make_float4(P0.y, P0.w, P1.y, P1.w), make_float4(P2.y, P2.w, P3.y, P3.w),
           make_float4(P4.y, P4.w, P5.y, P5.w), tx, ty, tz, ts, ax, ay, az, pf);
  return make_float4(ax, ay, az, pf);
}

// Evaluate all buffered P2C nodes.  Nodes are staged 64 per chunk as 32
// interleaved pairs (six float4: offsets, masses, the six second moments,
// softening and half trace, each as (node a, node b)) and a lane evaluates
// two nodes against its target with the packed FP32 instructions.  The
// offsets are o = cm_node - cm_bucket and the expression is written for
// r' = o - t = -r (q' = -q, so the acceleration reads qir3 r' - c q').
// A pair with a softened term falls back to the scalar p2c_term for both.
// Missing nodes of the last pair have zero mass and moments at a far offset.
__device__ __noinline__ float4 flush_p2c_nl(MixWarp& w, int nent, const QuadRecF* __restrict__ quadf, const FlushIn x) {
  const float qnan = __int_as_float(0x7fc00000);
  const float kPad = 1.0e10f;
  float4 a0, a1, b0, b1;  // next chunk: records of this lane's two nodes
  auto load_node = [&](int q, float4& r0, float4& r1) {
    r0 = make_float4(0.f, 0.f, 0.f, 0.f);
    r1 = r0;
    if (q < nent) {
      const float4* rec = reinterpret_cast<const float4*>(quadf + entry_node(w.cbuf[q]));
      r0 = rec[0];  // mass, soft, xx, xy
      r1 = rec[1];  // xz, yy, yz, zz
    }
  };
  auto fetch = [&](int cs) {
    load_node(cs + 2 * x.lane, a0, a1);
    load_node(cs + 2 * x.lane + 1, b0, b1);
  };
  fetch(0);
  const float2 ntx = make_float2(-x.tx, -x.tx), nty = make_float2(-x.ty, -x.ty), ntz = make_float2(-x.tz, -x.tz);
  const float2 three = make_float2(3.f, 3.f), five = make_float2(5.f, 5.f), half = make_float2(0.5f, 0.5f);
  float2 ax2 = make_float2(0.f, 0.f), ay2 = ax2, az2 = ax2, pf2 = ax2;
  for (int cs = 0; cs < nent; cs += 64) {
    // (ox, oy) (oz, M) (xx, xy) (xz, yy) (yz, zz) (soft, tr/2), each for nodes a and b
    {
      const int qa = cs + 2 * x.lane, qb = qa + 1;
      const float4 pad = make_float4(kPad, kPad, kPad, 0.f);
      const float4 ea = qa < nent ? w.cbuf[qa] : pad, eb = qb < nent ? w.cbuf[qb] : pad;
      if (qa < nent && entry_flag(ea)) {  // monopole: no second moments, NaN softening
        a0 = make_float4(a0.x, qnan, 0.f, 0.f);
        a1 = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (qb < nent && entry_flag(eb)) {
        b0 = make_float4(b0.x, qnan, 0.f, 0.f);
        b1 = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    w.qp[0][x.lane] = make_float4(ea.x, eb.x, ea.y, eb.y);
    w.qp[1][x.lane] = make_float4(ea.z, eb.z, a0.x, b0.x);
    w.qp[2][x.lane] = make_float4(a0.z, b0.z, a0.w, b0.w);
    w.qp[3][x.lane] = make_float4(a1.x, b1.x, a1.y, b1.y);
    w.qp[4][x.lane] = make_float4(a1.z, b1.z, a1.w, b1.w);
    w.qp[5][x.lane] = make_float4(a0.y, b0.y, 0.5f * (a0.z + a1.y + a1.w), 0.5f * (b0.z + b1.y + b1.w));
    }
    __syncwarp();
    if (cs + 64 < nent) fetch(cs + 64);
    const int np = (min(64, nent - cs) + 1) >> 1;
    if (x.grp < x.G) {
      for (int k = x.grp; k < np; k += x.G) {
        const float4 P0 = w.qp[0][k], P1 = w.qp[1][k];
        const float2 rx = __fadd2_rn(make_float2(P0.x, P0.y), ntx);  // r' = o - t
        const float2 ry = __fadd2_rn(make_float2(P0.z, P0.w), nty);
        const float2 rz = __fadd2_rn(make_float2(P1.x, P1.y), ntz);
        float2 r2 = __fmul2_rn(rx, rx);
        r2 = __ffma2_rn(ry, ry, r2);
        r2 = __ffma2_rn(rz, rz, r2);
        const float4 P5 = w.qp[5][k];
        const float twa = P5.x + x.ts, twb = P5.y + x.ts;
        const float4 P2 = w.qp[2][k], P3 = w.qp[3][k], P4 = w.qp[4][k];
        if (r2.x < twa * twa || r2.y < twb * twb) {  // softened: both terms in scalar form
          const float4 v = p2c_pair_scalar(w, k, x.tx, x.ty, x.tz, x.ts);
          ax2.x += v.x;
          ay2.x += v.y;
          az2.x += v.z;
          pf2.x += v.w;
          continue;
        }
        const float2 a = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
        const float2 d2 = __fmul2_rn(a, a);
        const float2 b = __fmul2_rn(a, d2);
        const float2 c = __fmul2_rn(__fmul2_rn(b, d2), three);
        const float2 d = __fmul2_rn(__fmul2_rn(c, d2), five);
        const float2 xx = make_float2(P2.x, P2.y), xy = make_float2(P2.z, P2.w);
        const float2 xz = make_float2(P3.x, P3.y), yy = make_float2(P3.z, P3.w);
        const float2 yz = make_float2(P4.x, P4.y), zz = make_float2(P4.z, P4.w);
        const float2 qx = __ffma2_rn(xz, rz, __ffma2_rn(xy, ry, __fmul2_rn(xx, rx)));
        const float2 qy = __ffma2_rn(yz, rz, __ffma2_rn(yy, ry, __fmul2_rn(xy, rx)));
        const float2 qz = __ffma2_rn(zz, rz, __ffma2_rn(yz, ry, __fmul2_rn(xz, rx)));
        const float2 qir = __fmul2_rn(half, __ffma2_rn(qz, rz, __ffma2_rn(qy, ry, __fmul2_rn(qx, rx))));
        const float2 M = make_float2(P1.z, P1.w), tr = make_float2(P5.z, P5.w);
        const float2 ctr = __fmul2_rn(c, tr);
        // qir3 = b M + d qir - c tr ; pot += b tr - M a - c qir
        const float2 qir3 = __fadd2_rn(__ffma2_rn(d, qir, __fmul2_rn(b, M)), make_float2(-ctr.x, -ctr.y));
        const float2 pt = __ffma2_rn(b, tr, make_float2(-(M.x * a.x), -(M.y * a.y)));
        pf2 = __fadd2_rn(pf2, __ffma2_rn(make_float2(-c.x, -c.y), qir, pt));
        const float2 nc = make_float2(-c.x, -c.y);
        ax2 = __ffma2_rn(nc, qx, __ffma2_rn(qir3, rx, ax2));
        ay2 = __ffma2_rn(nc, qy, __ffma2_rn(qir3, ry, ay2));
        az2 = __ffma2_rn(nc, qz, __ffma2_rn(qir3, rz, az2));
      }
    }
    __syncwarp();
  }
  return make_float4(ax2.x + ax2.y, ay2.x + ay2.y, az2.x + az2.y, pf2.x + pf2.y);
}
__device__ __forceinline__ void flush_p2c(MixWarp& w, int nent, const QuadRecF* __restrict__ quadf, MixCtx& x) {
  const float4 v = flush_p2c_nl(w, nent, quadf, FlushIn{x.tx, x.ty, x.tz, x.ts, x.lane, x.grp, x.G});
  x.pax += v.x; x.pay += v.y; x.paz += v.z; x.ppf += v.w;
  x.n_node += (unsigned)nent;
  x.commit();
}

// Append this lane's entry (if flag) to a warp buffer in lane order.
__device__ __forceinline__ int append(float4* buf, int n, bool flag, float4 v, int lane) {
  const unsigned m = __ballot_sync(kFull, flag);
  if (flag) buf[n + __popc(m & ((1u << lane) - 1u))] = v;
  return n + __popc(m);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kMixWarps * 32, kMinBlocks) traverse_mixed(TravParams P, const Mom* __restrict__ mom) {
  __shared__ MixWarp warps[kMixWarps];
  MixWarp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  unsigned long long c_pp = 0, c_pc = 0, c_open = 0;
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(P.work, 1u);
    bi = __shfl_sync(kFull, bi, 0);
    const int64_t b = P.b_begin + (int64_t)bi;
    if (b >= P.b_end) break;
    const int tnode = P.buckets[b];
    if (tnode < 0 || tnode >= P.nnodes) {
      if (lane == 0) atomicOr(P.status, kErrCapacity);
      continue;
    }
    __syncwarp();
    if (lane == 0) load_bucket_geom(mom, tnode, w.geom);
    __syncwarp();
    const BucketGeom& g = w.geom;
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    // more than 32 particles only in a depth-21 leaf of identical keys: its
    // targets are walked in chunks of 32 (decisions depend on the bucket only)
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      unsigned long long opens = 0;
      MixCtx x;
      x.lane = lane;
      x.nt = nt;
      x.t = lane % nt;
      x.grp = lane / nt;
      x.G = 32 / nt;
      x.tx = x.ty = x.tz = x.ts = 0.f;
      if (x.grp < x.G) {
        const int i = t0 + x.t;
        x.tx = (float)(P.p.x[i] - g.cm[0]);
        x.ty = (float)(P.p.y[i] - g.cm[1]);
        x.tz = (float)(P.p.z[i] - g.cm[2]);
        x.ts = (float)P.p.soft[i];
      }
      x.pax = x.pay = x.paz = x.ppf = 0.f;
      x.kah = w.kahan;
#pragma unroll
      for (int k = 0; k < 8; k++) w.kahan[k][lane] = 0.f;
      x.n_src = x.n_node = 0;

      int sp = 0, nc = 0, nfar = 0, nnear = 0;
      int nexp = 1;          // nodes expanded this step
      int pop = -1;          // stack slot of the first expanded node; -1 = the root step
      bool ok = true;
      while (true) {
        // lanes 8e..8e+7: children of expanded node e (the root step tests node 0)
        const int e = lane >> 3, c = lane & 7;
        int node = -1;
        if (pop < 0) {
          if (lane == 0) node = 0;
        } else if (e < nexp) {
          node = w.stack[pop + e] + c;  // the stack holds first children of opened nodes
        }
        int cls = kClsNone;
        WalkRec r;
        if (node >= 0) {
          if (node >= P.nnodes) {
            atomicOr(P.status, kErrCapacity);
          } else {
            r = P.walk[node];
            cls = classify_node(r, g, P.ox, P.oy, P.oz);
          }
        }
        opens += (unsigned long long)__popc(__ballot_sync(kFull, node >= 0 && node < P.nnodes &&
                                                                      r.type == kTypeInternal));
        float ofx = 0.f, ofy = 0.f, ofz = 0.f;
        bool far = false;
        if (cls == kClsP2P || cls == kClsQuad || cls == kClsMono) {
          const double cx = r.cm[0] + P.ox, cy = r.cm[1] + P.oy, cz = r.cm[2] + P.oz;
          ofx = (float)(cx - g.cm[0]);
          ofy = (float)(cy - g.cm[1]);
          ofz = (float)(cz - g.cm[2]);
          if (cls == kClsP2P) {
            const double reach = r.reach + r.soft_max + g.soft_max;
            far = box_dist2(g.lo, g.hi, cx, cy, cz) > reach * reach;
          }
        }
        const float4 ent = pack_entry(ofx, ofy, ofz, node, cls == kClsMono);
        nc = append(w.cbuf, nc, cls == kClsQuad || cls == kClsMono, ent, lane);
        nfar = append(w.pbuf, nfar, cls == kClsP2P && far, ent, lane);
        {  // near leaves grow down from the end of the shared buffer
          const bool nr = (cls == kClsP2P && !far);
          const unsigned m = __ballot_sync(kFull, nr);
          if (nr) w.pbuf[kMixBuf - 1 - nnear - __popc(m & ((1u << lane) - 1u))] = ent;
          nnear += __popc(m);
        }
        {
          const bool op = (cls == kClsOpen);
          const unsigned m = __ballot_sync(kFull, op);
          if (sp + __popc(m) > kMixStack) {
            ok = false;
            break;
          }
          if (op) w.stack[sp + __popc(m & ((1u << lane) - 1u))] = r.first_child;
          sp += __popc(m);
        }
        __syncwarp();
        // one flush site per kind (the walk's last step drains every buffer)
        const bool last = (sp == 0);
        if (nc >= 32 || (last && nc)) { flush_p2c(w, nc, P.quadf, x); nc = 0; }
        if (nfar + nnear >= 32 || last) {
          if (nfar) flush_p2p<true>(w, w.pbuf, nfar, P.walk, P.srcf, P.softf, x);
          if (nnear) flush_p2p<false>(w, w.pbuf + (kMixBuf - nnear), nnear, P.walk, P.srcf, P.softf, x);
          nfar = nnear = 0;
        }
        if (last) break;
        nexp = sp < 4 ? sp : 4;
        sp -= nexp;
        pop = sp;
        __syncwarp();
      }
      if (!ok) {
        if (lane == 0) atomicOr(P.status, kErrStack);
        break;
      }

      // sum the G lane groups of each target (staging area reused as FP64 scratch)
      double* red = reinterpret_cast<double*>(&w.qp[0][0]);
      __syncwarp();
#pragma unroll
      for (int k = 0; k < 4; k++) red[4 * lane + k] = (double)w.kahan[2 * k][lane] - (double)w.kahan[2 * k + 1][lane];
      __syncwarp();
      if (lane < nt) {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int gg = 0; gg < x.G; gg++)
          for (int k = 0; k < 4; k++) v[k] += red[4 * (gg * nt + lane) + k];
        const int i = t0 + lane;
        if (P.accumulate) {  // later replica walks add to the stored sums
          P.p.ax[i] += v[0];
          P.p.ay[i] += v[1];
          P.p.az[i] += v[2];
          P.p.potf[i] += v[3];
        } else {
          P.p.ax[i] = v[0];
          P.p.ay[i] = v[1];
          P.p.az[i] = v[2];
          P.p.pot[i] = 0.0;  // this fallback sums P2C and P2P potentials together: pot_full only
          P.p.potf[i] = v[3];
        }
      }
      __syncwarp();
      c_pp += (unsigned long long)x.n_src * (unsigned long long)nt;
      c_pc += (unsigned long long)x.n_node * (unsigned long long)nt;
      if (tc == 0) c_open += opens;
      if (P.bucket_work && lane == 0) {  // this chunk's interactions, added to the bucket's
        unsigned long long wk = (unsigned long long)(x.n_src + x.n_node) * (unsigned long long)nt;
        if (tc > 0 || P.accumulate) wk += P.bucket_work[b];
        P.bucket_work[b] = wk;
      }
    }
  }
  if (lane == 0) {
    atomicAdd(&P.counters[0], c_pp);
    atomicAdd(&P.counters[1], c_pc);
    atomicAdd(&P.counters[2], c_open);
  }
}

// Per-particle FP32 source record: position relative to its leaf's cm, mass.
__global__ void __launch_bounds__(128) prep_sources(const int32_t* __restrict__ buckets, int64_t nbuckets,
                                                    const WalkRec* __restrict__ walk, Particles p,
                                                    float4* __restrict__ srcf, float* __restrict__ softf) {
  int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (b >= nbuckets) return;
  const WalkRec w = walk[buckets[b]];
  for (int j = lane; j < w.pcount; j += 32) {
    int i = w.pstart + j;
    srcf[i] = make_float4((float)(p.x[i] - w.cm[0]), (float)(p.y[i] - w.cm[1]), (float)(p.z[i] - w.cm[2]),
                          (float)p.m[i]);
    softf[i] = (float)p.soft[i];
  }
}

void launch_prep_sources(const int32_t* buckets, int64_t nbuckets, const WalkRec* walk, Particles p, float4* srcf,
                         float* softf, cudaStream_t st) {
  if (nbuckets <= 0) return;
  int64_t threads = nbuckets * 32;
  note_launch();
  prep_sources<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(buckets, nbuckets, walk, p, srcf, softf);
}

// 5 CTAs per SM (96 registers: at 80 the walk state spills)
void launch_traverse_mixed(const TravParams& P, const Mom* mom, int grid, cudaStream_t st) {
  note_launch();
  traverse_mixed<5><<<grid, kMixWarps * 32, 0, st>>>(P, mom);
}

}  // namespace pt
