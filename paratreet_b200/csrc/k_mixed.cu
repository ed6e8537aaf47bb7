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
//  eval     the bucket's n_t targets are replicated over G = 32 / T lane
//           groups (T = next power of two >= n_t); group g takes every G-th
//           source / node of a 32-entry chunk staged in shared memory, so a
//           10-particle bucket keeps all 32 lanes busy.  Leaves whose nearest
//           particle pair is provably beyond the softening length take a
//           branch-free Newtonian loop (rsqrt on the SFU).
//  reduce   per-lane Kahan sums -> FP64, butterfly over the G groups.
#include "pt_internal.cuh"
#include "pt_walk.cuh"

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
  float4 src[32];           // staged sources: x, y, z (rel. bucket), m
  float ssoft[32];
  float sreach2[32];        // (soft_j + max bucket softening)^2: beyond it a pair is unsoftened
  float4 qa[32];            // staged P2C: offset xyz, mass
  float4 qb[32];            // xx, xy, xz, yy
  float4 qc[32];            // yz, zz, soft (< 0: monopole), trace/2
};

// SPLINE in FP32, softened branch (r < twoh): kept out of line so that the
// rarely taken polynomial does not raise register pressure in the hot loops.
__device__ __noinline__ void spline_f32_soft(float r2, float rinv, float twoh, float& a, float& b) {
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
__device__ __forceinline__ void spline_f32(float r2, float rinv, float twoh, float& a, float& b) {
  if (r2 < twoh * twoh) {
    spline_f32_soft(r2, rinv, twoh, a, b);
  } else {
    a = rinv;
    b = rinv * rinv * rinv;
  }
}

// SPLINEQ in FP32 with the reference's grouping (examples/GravityVisitor.h:37-80);
// only the softened branch is called (out of line, rarely taken).
__device__ __noinline__ void splineq_f32(float dir, float r2, float twoh, float& a, float& b, float& c, float& d) {
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

// Evaluate all buffered P2P leaves of one kind (far: no pair can be softened).
template <bool kFar>
__device__ __forceinline__ void flush_p2p(MixWarp& w, const float4* __restrict__ buf, int nleaves,
                                          const WalkRec* __restrict__ walk, const float4* __restrict__ srcf,
                                          const float* __restrict__ softf, MixCtx& x) {
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
  // Chunks of 32 sources; the loads of chunk k+1 are issued before chunk k is
  // evaluated so that their L2 latency overlaps the arithmetic.
  int base_leaf = 0;  // leaf holding the next chunk's first source
  float4 nraw = make_float4(0.f, 0.f, 0.f, 0.f), noff = nraw;
  float nsoft = 0.f;
  auto fetch = [&](int cs) {
    const int q = cs + x.lane;
    int lo = base_leaf;  // last leaf with pre <= q: a chunk spans few leaves
    while (lo + 1 < nleaves && w.pre[lo + 1] <= q) lo++;
    base_leaf = __shfl_sync(kFull, lo, 31);
    if (q < total) {
      noff = buf[lo];
      const int j = w.ps0[lo] + (q - w.pre[lo]);
      nraw = srcf[j];
      if (!kFar) nsoft = softf[j];
    }
  };
  fetch(0);
  for (int cs = 0; cs < total; cs += 32) {
    if (cs + x.lane < total) {
      w.src[x.lane] = make_float4(nraw.x + noff.x, nraw.y + noff.y, nraw.z + noff.z, nraw.w);
      if (!kFar) {
        w.ssoft[x.lane] = nsoft;
        const float rr = nsoft + (float)w.geom.soft_max;
        w.sreach2[x.lane] = rr * rr;
      }
    }
    __syncwarp();
    if (cs + 32 < total) fetch(cs + 32);
    const int cnt = min(32, total - cs);
    if (kFar && x.grp < x.G) {
      float bx = 0.f, by = 0.f, bz = 0.f, bp = 0.f;  // second chain
      int jj = x.grp;
      for (; jj + x.G < cnt; jj += 2 * x.G) {
        const float4 s = w.src[jj];
        const float4 u = w.src[jj + x.G];
        const float dx = s.x - x.tx, dy = s.y - x.ty, dz = s.z - x.tz;
        const float ex = u.x - x.tx, ey = u.y - x.ty, ez = u.z - x.tz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float q2 = ex * ex + ey * ey + ez * ez;
        const float rinv = rsqrtf(r2), qinv = rsqrtf(q2);
        const float mr = s.w * rinv, mq = u.w * qinv;
        const float mr3 = mr * rinv * rinv, mq3 = mq * qinv * qinv;
        x.pax += dx * mr3;
        x.pay += dy * mr3;
        x.paz += dz * mr3;
        x.ppf -= mr;
        bx += ex * mq3;
        by += ey * mq3;
        bz += ez * mq3;
        bp -= mq;
      }
      if (jj < cnt) {
        const float4 s = w.src[jj];
        const float dx = s.x - x.tx, dy = s.y - x.ty, dz = s.z - x.tz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float rinv = rsqrtf(r2);
        const float mr = s.w * rinv;
        const float mr3 = mr * rinv * rinv;
        x.pax += dx * mr3;
        x.pay += dy * mr3;
        x.paz += dz * mr3;
        x.ppf -= mr;
      }
      x.pax += bx;
      x.pay += by;
      x.paz += bz;
      x.ppf += bp;
    } else if (!kFar && x.grp < x.G) {
      for (int jj = x.grp; jj < cnt; jj += x.G) {
        const float4 s = w.src[jj];
        const float dx = s.x - x.tx, dy = s.y - x.ty, dz = s.z - x.tz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > w.sreach2[jj]) {  // r > soft_i + soft_j: Newtonian, and r > 0
          const float rinv = rsqrtf(r2);
          const float mr = s.w * rinv;
          const float mr3 = mr * rinv * rinv;
          x.pax += dx * mr3;
          x.pay += dy * mr3;
          x.paz += dz * mr3;
          x.ppf -= mr;
        } else if (r2 > 0.f) {
          const float rinv = rsqrtf(r2);
          float a, b;
          spline_f32(r2, rinv, w.ssoft[jj] + x.ts, a, b);
          const float bm = b * s.w;
          x.pax += dx * bm;
          x.pay += dy * bm;
          x.paz += dz * bm;
          x.ppf -= s.w * a;
        }
      }
    }
    __syncwarp();
  }
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

// Evaluate all buffered P2C nodes.
__device__ __forceinline__ void flush_p2c(MixWarp& w, int nent, const QuadRecF* __restrict__ quadf, MixCtx& x) {
  const float qnan = __int_as_float(0x7fc00000);
  float4 ne = make_float4(0.f, 0.f, 0.f, 0.f), nq0 = ne, nq1 = ne;  // next chunk's entry and record
  auto fetch = [&](int cs) {
    const int q = cs + x.lane;
    if (q < nent) {
      ne = w.cbuf[q];
      const float4* rec = reinterpret_cast<const float4*>(quadf + entry_node(ne));
      nq0 = rec[0];  // mass, soft, xx, xy
      nq1 = rec[1];  // xz, yy, yz, zz
    }
  };
  fetch(0);
  for (int cs = 0; cs < nent; cs += 32) {
    if (cs + x.lane < nent) {
      w.qa[x.lane] = make_float4(ne.x, ne.y, ne.z, nq0.x);
      if (entry_flag(ne)) {
        w.qb[x.lane] = make_float4(0.f, 0.f, 0.f, 0.f);
        w.qc[x.lane] = make_float4(0.f, 0.f, qnan, 0.f);
      } else {
        w.qb[x.lane] = make_float4(nq0.z, nq0.w, nq1.x, nq1.y);
        w.qc[x.lane] = make_float4(nq1.z, nq1.w, nq0.y, 0.5f * (nq0.z + nq1.y + nq1.w));
      }
    }
    __syncwarp();
    if (cs + 32 < nent) fetch(cs + 32);
    const int cnt = min(32, nent - cs);
    if (x.grp < x.G) {
      // one P2C term has enough independent work; a 2-way unroll measured slower
      for (int ee = x.grp; ee < cnt; ee += x.G)
        p2c_term(w.qa[ee], w.qb[ee], w.qc[ee], x.tx, x.ty, x.tz, x.ts, x.pax, x.pay, x.paz, x.ppf);
    }
    __syncwarp();
  }
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
    const unsigned long long work0 = c_pp + c_pc;
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
      double* red = reinterpret_cast<double*>(w.qa);
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
          P.p.pot[i] = 0.0;
          P.p.potf[i] = v[3];
        }
      }
      __syncwarp();
      c_pp += (unsigned long long)x.n_src * (unsigned long long)nt;
      c_pc += (unsigned long long)x.n_node * (unsigned long long)nt;
      if (tc == 0) c_open += opens;
    }
    if (P.bucket_work && lane == 0) {
      const unsigned long long wk = c_pp + c_pc - work0;
      P.bucket_work[b] = P.accumulate ? P.bucket_work[b] + wk : wk;
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

// variant: 0 = at most 6 CTAs/SM (80 registers), 1 = 5 CTAs/SM (no spills)
void launch_traverse_mixed(const TravParams& P, const Mom* mom, int grid, int variant, cudaStream_t st) {
  if (variant == 1) { note_launch(); traverse_mixed<5><<<grid, kMixWarps * 32, 0, st>>>(P, mom); }
  else { note_launch(); traverse_mixed<6><<<grid, kMixWarps * 32, 0, st>>>(P, mom); }
}

}  // namespace pt
