// k_mixed.cu -- K7 mixed-precision traversal.
//
// Same walk (and so the same interaction lists) as the FP64 form: the tree,
// the opening tests and the softening-overlap tests stay FP64.  Every P2P
// (GravityVisitor::leaf, examples/GravityVisitor.h:144-160) and quadrupole
// P2C (GravityVisitor::node, :184-224) interaction is evaluated in FP32 on
// offsets relative to the target bucket's centre of mass:
//   targets   (x_i - cm_bucket)                      FP64 subtract -> FP32
//   sources   (x_j - cm_leaf) [FP32, per step] + (cm_leaf - cm_bucket)
//             [FP64 subtract per (leaf, bucket) -> FP32]
//   P2C       (x_i - cm_bucket) - (cm_node - cm_bucket)[FP64 -> FP32]
// Each source leaf's <=32-term partial is summed in plain FP32 and then
// Kahan-added into the per-target FP32 accumulators; P2C terms are
// Kahan-added directly.  Acceleration and the full potential (P2P spline,
// P2C quadrupole, monopole) are produced.
#include "pt_internal.cuh"
#include "pt_walk.cuh"

namespace pt {

constexpr int kMixWarps = 4;

struct Kahan {
  float s, c;
  __device__ __forceinline__ void add(float v) {
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// SPLINE in FP32 (r2 > 0): force term b, potential term a.
__device__ __forceinline__ void spline_f32(float r2, float rinv, float twoh, float& a, float& b) {
  if (r2 < twoh * twoh) {
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
      b = -1.0f / 15.0f * rinv * rinv * rinv + dih * dih * dih * (8.0f / 3.0f - 3.0f * u + 6.0f / 5.0f * u2 - 1.0f / 6.0f * u2 * u);
    }
  } else {
    a = rinv;
    b = rinv * rinv * rinv;
  }
}

// SPLINEQ in FP32, as the reference evaluates it (examples/GravityVisitor.h:37-80).
__device__ __forceinline__ void splineq_f32(float dir, float r2, float twoh, float& a, float& b, float& c, float& d) {
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
      a = -1.0f / 15.0f * dir + dih * (8.0f / 5.0f) - 4.0f / 3.0f * u2 + u2 * u - 3.0f / 10.0f * u2 * u2 + 1.0f / 30.0f * u2 * u2 * u;
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

struct MixedEval {
  const WalkRec* walk;
  const QuadRec* quad;
  const QuadRecF* quadf;
  const float4* srcf;
  const float* softf;
  float4* stage;   // this warp's 32 staged sources (x, y, z rel. bucket; m)
  float* stages;   // their softening
  int lane, nt;
  float tx, ty, tz, ts;  // target rel. bucket cm
  Kahan ax, ay, az, pf;
  const BucketGeom* g;
  double ox, oy, oz;
  unsigned long long n_pp, n_pc;

  __device__ void p2p(int node) {
    const WalkRec w = walk[node];
    const int s0 = w.pstart, sn = w.pcount;
    const float offx = (float)((w.cm[0] + ox) - g->cm[0]);
    const float offy = (float)((w.cm[1] + oy) - g->cm[1]);
    const float offz = (float)((w.cm[2] + oz) - g->cm[2]);
    float pax = 0.f, pay = 0.f, paz = 0.f, ppf = 0.f;
    for (int base = 0; base < sn; base += 32) {
      int cnt = min(32, sn - base);
      __syncwarp();
      if (lane < cnt) {
        float4 s = srcf[s0 + base + lane];
        stage[lane] = make_float4(s.x + offx, s.y + offy, s.z + offz, s.w);
        stages[lane] = softf[s0 + base + lane];
      }
      __syncwarp();
      if (lane < nt) {
        for (int j = 0; j < cnt; j++) {
          float4 s = stage[j];
          float dx = s.x - tx, dy = s.y - ty, dz = s.z - tz;
          float r2 = dx * dx + dy * dy + dz * dz;
          if (r2 > 0.f) {
            float rinv = rsqrtf(r2);
            float a, b;
            spline_f32(r2, rinv, stages[j] + ts, a, b);
            float bm = b * s.w;
            pax += dx * bm;
            pay += dy * bm;
            paz += dz * bm;
            ppf -= s.w * a;
          }
        }
      }
    }
    ax.add(pax);
    ay.add(pay);
    az.add(paz);
    pf.add(ppf);
    n_pp += (unsigned long long)sn * (unsigned long long)nt;
  }

  __device__ void p2c(int node) {
    const WalkRec w = walk[node];
    n_pc += (unsigned long long)nt;
    if (w.count == 0) return;
    const double cx = w.cm[0] + ox, cy = w.cm[1] + oy, cz = w.cm[2] + oz;
    const float offx = (float)(cx - g->cm[0]), offy = (float)(cy - g->cm[1]), offz = (float)(cz - g->cm[2]);
    const QuadRecF q = quadf[node];
    const double qsoft = quad[node].soft;
    if (open_softening_exact(cx, cy, cz, qsoft, g->cm[0], g->cm[1], g->cm[2], g->soft, g->lo, g->hi)) {
      if (lane < nt) {
        float dx = offx - tx, dy = offy - ty, dz = offz - tz;
        float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > 0.f) {
          float rinv = rsqrtf(r2);
          float f = q.mass * rinv * rinv * rinv;
          ax.add(dx * f);
          ay.add(dy * f);
          az.add(dz * f);
          pf.add(-q.mass * rinv);
        }
      }
      return;
    }
    if (lane < nt) {
      float rx = tx - offx, ry = ty - offy, rz = tz - offz;
      float r2 = rx * rx + ry * ry + rz * rz;
      float dir = rsqrtf(r2);
      float a, b, c, d;
      splineq_f32(dir, r2, q.soft + ts, a, b, c, d);
      float qx = q.xx * rx + q.xy * ry + q.xz * rz;
      float qy = q.xy * rx + q.yy * ry + q.yz * rz;
      float qz = q.xz * rx + q.yz * ry + q.zz * rz;
      float qir = 0.5f * (qx * rx + qy * ry + qz * rz);
      float tr = 0.5f * (q.xx + q.yy + q.zz);
      float qir3 = b * q.mass + d * qir - c * tr;
      pf.add(-q.mass * a - c * qir + b * tr);
      ax.add(-qir3 * rx + c * qx);
      ay.add(-qir3 * ry + c * qy);
      az.add(-qir3 * rz + c * qz);
    }
  }
};

__global__ void __launch_bounds__(kMixWarps * 32) traverse_mixed(TravParams P, const Mom* __restrict__ mom) {
  __shared__ WalkFrame stacks[kMixWarps][kWalkStack];
  __shared__ float4 stage[kMixWarps][32];
  __shared__ float stages[kMixWarps][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long c_pp = 0, c_pc = 0, c_open = 0;
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(P.work, 1u);
    bi = __shfl_sync(kFull, bi, 0);
    int64_t b = P.b_begin + (int64_t)bi;
    if (b >= P.b_end) break;
    const int tnode = P.buckets[b];
    BucketGeom g;
    {
      const Mom& q = mom[tnode];
      for (int d = 0; d < 3; d++) { g.lo[d] = q.lo[d]; g.hi[d] = q.hi[d]; g.cm[d] = q.cm[d]; }
      g.soft = q.soft;
    }
    const int t0 = P.walk[tnode].pstart, nt = P.walk[tnode].pcount;
    if (nt > 32) {
      if (lane == 0) atomicOr(P.status, kErrBucketTooBig);
      continue;
    }
    MixedEval ev;
    ev.walk = P.walk;
    ev.quad = P.quad;
    ev.quadf = P.quadf;
    ev.srcf = P.srcf;
    ev.softf = P.softf;
    ev.stage = stage[wid];
    ev.stages = stages[wid];
    ev.lane = lane;
    ev.nt = nt;
    ev.tx = ev.ty = ev.tz = ev.ts = 0.f;
    if (lane < nt) {
      ev.tx = (float)(P.p.x[t0 + lane] - g.cm[0]);
      ev.ty = (float)(P.p.y[t0 + lane] - g.cm[1]);
      ev.tz = (float)(P.p.z[t0 + lane] - g.cm[2]);
      ev.ts = (float)P.p.soft[t0 + lane];
    }
    ev.ax = Kahan{0.f, 0.f};
    ev.ay = Kahan{0.f, 0.f};
    ev.az = Kahan{0.f, 0.f};
    ev.pf = Kahan{0.f, 0.f};
    ev.g = &g;
    ev.ox = P.ox; ev.oy = P.oy; ev.oz = P.oz;
    ev.n_pp = 0; ev.n_pc = 0;
    if (!walk_bucket(P.walk, g, P.ox, P.oy, P.oz, stacks[wid], lane, ev, c_open) && lane == 0)
      atomicOr(P.status, kErrStack);
    if (lane < nt) {
      int i = t0 + lane;
      P.p.ax[i] = (double)ev.ax.s + (double)(-ev.ax.c);
      P.p.ay[i] = (double)ev.ay.s + (double)(-ev.ay.c);
      P.p.az[i] = (double)ev.az.s + (double)(-ev.az.c);
      P.p.pot[i] = 0.0;
      P.p.potf[i] = (double)ev.pf.s + (double)(-ev.pf.c);
    }
    c_pp += ev.n_pp;
    c_pc += ev.n_pc;
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
  prep_sources<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(buckets, nbuckets, walk, p, srcf, softf);
}

void launch_traverse_mixed(const TravParams& P, const Mom* mom, int grid, cudaStream_t st) {
  traverse_mixed<<<grid, kMixWarps * 32, 0, st>>>(P, mom);
}

}  // namespace pt
