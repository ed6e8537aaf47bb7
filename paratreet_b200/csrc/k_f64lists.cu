// k_f64lists.cu -- FP64 evaluation of the two-phase interaction lists
// (precision PT_FP64_LISTS).
//
// The comparator of the mixed form: the same walk_lists lists (so the same
// leaf() and node() interactions as the reference's traversal), evaluated
// with the same work layout as eval_p2c / eval_p2p (one warp per bucket, the
// bucket's targets replicated over G = floor(32 / n_t) lane groups, 32-entry
// chunks staged in shared memory), but in FP64 with the reference's
// expressions on absolute positions: GravityVisitor::leaf and ::node
// (examples/GravityVisitor.h:144-160, 184-224) with SPLINE / SPLINEQ
// (:37-120) where a pair may be softened, addGravity (:130-139) for monopole
// nodes.  Terms that cannot be softened (far leaves, unflagged nodes) use the
// hardware reciprocal square root instead of 1 / sqrt, and every target sums
// its terms in list order per lane group, then the groups in order, so the
// result differs from the ordered FP64 walk (traverse_f64) only in rounding.
// P2C stores (or, for replica walks after the first, adds) and P2P adds, as
// the mixed evaluators do.
#include "pt_fp64.cuh"
#include "pt_internal.cuh"
#include "pt_walk.cuh"

namespace pt {

constexpr int kE64Warps = 4;

struct Eval64Warp {
  double st[12][32];     // staged entries: P2C 12 rows (centre + offset 3, M, soft, 6 moments, class)
                         // P2P 5 rows (x, y, z + offset, m, soft); reused for the group sums
  int32_t lnode[32];     // P2P: leaves of the current block and kind
  int32_t lincl[32];     // P2P: inclusive prefix of their particle counts
};

struct E64Target {
  int t, grp, G, nt;
  double x, y, z, s;
};

__device__ __forceinline__ E64Target e64_target(const Particles& p, int t0, int nt, int lane) {
  E64Target x;
  x.nt = nt;
  x.t = lane % nt;
  x.grp = lane / nt;
  x.G = 32 / nt;
  x.x = x.y = x.z = x.s = 0.0;
  if (x.grp < x.G) {
    const int i = t0 + x.t;
    x.x = p.x[i];
    x.y = p.y[i];
    x.z = p.z[i];
    x.s = p.soft[i];
  }
  return x;
}

// Sum the G lane groups of each target in group order and store or add.
// p2c: pot gets the quadrupole node() terms, pot_full every term.
__device__ __forceinline__ void e64_finish(Eval64Warp& w, const double v[5], const E64Target& x, const TravParams& P,
                                           int t0, int lane, bool p2c, bool store) {
  double* red = &w.st[0][0];
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 5; k++) red[5 * lane + k] = v[k];
  __syncwarp();
  if (lane < x.nt) {
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int g = 0; g < x.G; g++)
      for (int k = 0; k < 5; k++) s[k] += red[5 * (g * x.nt + lane) + k];
    const int i = t0 + lane;
    if (store) {
      P.p.ax[i] = s[0];
      P.p.ay[i] = s[1];
      P.p.az[i] = s[2];
      P.p.pot[i] = p2c ? s[3] : 0.0;
      P.p.potf[i] = s[4];
    } else {
      P.p.ax[i] += s[0];
      P.p.ay[i] += s[1];
      P.p.az[i] += s[2];
      if (p2c) P.p.pot[i] += s[3];
      P.p.potf[i] += s[4];
    }
  }
  __syncwarp();
}

__device__ __forceinline__ bool e64_next_bucket(const TravParams& P, int lane, int64_t& b, int& tnode) {
  unsigned bi = 0;
  if (lane == 0) bi = atomicAdd(P.work, 1u);
  bi = __shfl_sync(kFull, bi, 0);
  b = P.b_begin + (int64_t)bi;
  if (b >= P.b_end) return false;
  tnode = P.buckets[b];
  return true;
}

// ------------------------------------------------------------------- P2C
__global__ void __launch_bounds__(kE64Warps * 32) eval_p2c_f64(TravParams P, ListParams L) {
  __shared__ Eval64Warp warps[kE64Warps];
  Eval64Warp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  int64_t b;
  int tnode;
  while (e64_next_bucket(P, lane, b, tnode)) {
    if (tnode < 0 || tnode >= P.nnodes) continue;
    const int64_t lb = b - P.b_begin;
    const int64_t start = L.pc_start[lb];
    const int count = L.pc_count[lb];
    if (count == 0 && P.accumulate) continue;  // nothing to add (the first walk stores, even zeros)
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const E64Target x = e64_target(P.p, t0, nt, lane);
      double ax = 0.0, ay = 0.0, az = 0.0, pq = 0.0, pf = 0.0;
      for (int cs = 0; cs < count; cs += 32) {
        const int n = min(32, count - cs);
        __syncwarp();
        if (lane < n) {
          const int e = L.pc_pool[start + cs + lane];
          const int node = e & 0x3fffffff;
          const WalkRec& r = P.walk[node];
          const QuadRec q = P.quad[node];
          // class: 0 quadrupole, 1 near quadrupole (SPLINEQ), 2 monopole (addGravity)
          const double cls = (e < 0) ? 2.0 : ((e & 0x40000000) ? 1.0 : 0.0);
          w.st[0][lane] = r.cm[0] + P.ox;
          w.st[1][lane] = r.cm[1] + P.oy;
          w.st[2][lane] = r.cm[2] + P.oz;
          w.st[3][lane] = q.mass;
          w.st[4][lane] = q.soft;
          w.st[5][lane] = q.xx;
          w.st[6][lane] = q.xy;
          w.st[7][lane] = q.xz;
          w.st[8][lane] = q.yy;
          w.st[9][lane] = q.yz;
          w.st[10][lane] = q.zz;
          w.st[11][lane] = (r.count == 0) ? -1.0 : cls;  // -1: an empty node (node() returns)
        }
        __syncwarp();
        if (x.grp < x.G) {
          for (int k = x.grp; k < n; k += x.G) {
            const double cls = w.st[11][k];
            if (cls < 0.0) continue;
            const double M = w.st[3][k];
            if (cls == 2.0) {  // addGravity, :130-139
              const double dx = w.st[0][k] - x.x, dy = w.st[1][k] - x.y, dz = w.st[2][k] - x.z;
              const double rsq = dx * dx + dy * dy + dz * dz;
              if (rsq != 0.0) {
                const double ri = rsqrt(rsq);
                const double f = M * ri * ri * ri;
                ax += dx * f;
                ay += dy * f;
                az += dz * f;
                pf += -M * ri;
              }
              continue;
            }
            const double rx = x.x - w.st[0][k], ry = x.y - w.st[1][k], rz = x.z - w.st[2][k];
            const double rsq = rx * rx + ry * ry + rz * rz;
            const double dir = rsqrt(rsq);
            double a, bb, c, d;
            if (cls == 1.0) {
              splineq_f64(dir, rsq, w.st[4][k] + x.s, a, bb, c, d);
            } else {
              a = dir;
              bb = a * a * a;
              c = 3.0 * bb * a * a;
              d = 5.0 * c * a * a;
            }
            const double xx = w.st[5][k], xy = w.st[6][k], xz = w.st[7][k];
            const double yy = w.st[8][k], yz = w.st[9][k], zz = w.st[10][k];
            const double qx = xx * rx + xy * ry + xz * rz;
            const double qy = xy * rx + yy * ry + yz * rz;
            const double qz = xz * rx + yz * ry + zz * rz;
            const double qir = 0.5 * (qx * rx + qy * ry + qz * rz);
            const double tr = 0.5 * (xx + yy + zz);
            const double qir3 = bb * M + d * qir - c * tr;
            const double pp = -M * a - c * qir + bb * tr;
            pq += pp;
            pf += pp;
            ax += -qir3 * rx + c * qx;
            ay += -qir3 * ry + c * qy;
            az += -qir3 * rz + c * qz;
          }
        }
      }
      const double v[5] = {ax, ay, az, pq, pf};
      e64_finish(w, v, x, P, t0, lane, true, P.accumulate == 0);
    }
  }
}

// ------------------------------------------------------------------- P2P
// Sources of the leaves w.lnode[0..nl) (inclusive count prefix w.lincl)
// against this lane's target, 32 sources per chunk (GravityVisitor::leaf,
// :144-160).  kFar: no pair of these leaves can be softened, and no source is
// the target itself.
template <bool kFar>
__device__ __forceinline__ void e64_p2p_leaves(Eval64Warp& w, int nl, const TravParams& P, const E64Target& x,
                                               int lane, double& ax, double& ay, double& az, double& pf) {
  const int total = w.lincl[nl - 1];
  for (int cs = 0; cs < total; cs += 32) {
    const int q = cs + lane;
    __syncwarp();
    if (q < total) {
      // leaf of stream position q: the first with inclusive prefix > q
      int lo = 0, hi = nl - 1;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (w.lincl[mid] > q) hi = mid;
        else lo = mid + 1;
      }
      const int node = w.lnode[lo];
      const int first = (lo == 0) ? 0 : w.lincl[lo - 1];
      const int j = P.walk[node].pstart + (q - first);
      w.st[0][lane] = P.p.x[j] + P.ox;
      w.st[1][lane] = P.p.y[j] + P.oy;
      w.st[2][lane] = P.p.z[j] + P.oz;
      w.st[3][lane] = P.p.m[j];
      w.st[4][lane] = P.p.soft[j];
    }
    __syncwarp();
    const int n = min(32, total - cs);
    if (x.grp < x.G) {
      for (int k = x.grp; k < n; k += x.G) {
        const double dx = w.st[0][k] - x.x, dy = w.st[1][k] - x.y, dz = w.st[2][k] - x.z;
        const double rsq = dx * dx + dy * dy + dz * dz;
        const double ms = w.st[3][k];
        if (kFar) {
          const double ri = rsqrt(rsq);
          const double mr = ms * ri;
          const double mr3 = mr * ri * ri;
          ax += dx * mr3;
          ay += dy * mr3;
          az += dz * mr3;
          pf += -mr;
        } else if (rsq != 0.0) {
          double a, bb;
          spline_f64(rsq, w.st[4][k] + x.s, a, bb);
          const double bm = bb * ms;
          ax += dx * bm;
          ay += dy * bm;
          az += dz * bm;
          pf += -ms * a;
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kE64Warps * 32) eval_p2p_f64(TravParams P, ListParams L,
                                                                  const Mom* __restrict__ mom) {
  __shared__ Eval64Warp warps[kE64Warps];
  Eval64Warp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  unsigned long long c_pp = 0;
  int64_t b;
  int tnode;
  while (e64_next_bucket(P, lane, b, tnode)) {
    if (tnode < 0 || tnode >= P.nnodes) continue;
    const int64_t lb = b - P.b_begin;
    const int64_t start = L.pp_start[lb];
    const int count = L.pp_count[lb];
    if (count == 0) continue;  // P2P only adds
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    BucketGeom g;
    load_bucket_geom(mom, tnode, g);
    unsigned long long nsrc = 0;
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const E64Target x = e64_target(P.p, t0, nt, lane);
      double ax = 0.0, ay = 0.0, az = 0.0, pf = 0.0;
      nsrc = 0;
      for (int blk = 0; blk < count; blk += 32) {
        const bool valid = blk + lane < count;
        int e = valid ? L.pp_pool[start + blk + lane] & 0x7fffffff : 0;
        const unsigned cnt = valid ? (unsigned)P.walk[e].pcount : 0u;
        nsrc += (unsigned long long)__reduce_add_sync(kFull, cnt);
        if (valid && p2p_leaf_near(P.walk, e, g.lo, g.hi, g.soft_max, P.ox, P.oy, P.oz)) e |= (int)0x80000000;
#pragma unroll
        for (int kind = 0; kind < 2; kind++) {  // far leaves, then near ones
          const bool sel = valid && ((e < 0) == (kind == 1));
          const unsigned m = __ballot_sync(kFull, sel);
          const int nl = __popc(m);
          int cnt = 0;
          if (sel) cnt = P.walk[e & 0x7fffffff].pcount;
          // inclusive prefix of the selected leaves' counts, in selection order
          const int pos = __popc(m & ((1u << lane) - 1u));
          int inc = cnt;
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, inc, o);
            if (lane >= o) inc += y;
          }
          __syncwarp();
          if (sel) {
            w.lnode[pos] = e & 0x7fffffff;
            w.lincl[pos] = inc;
          }
          __syncwarp();
          if (nl) {
            if (kind == 0) e64_p2p_leaves<true>(w, nl, P, x, lane, ax, ay, az, pf);
            else e64_p2p_leaves<false>(w, nl, P, x, lane, ax, ay, az, pf);
          }
        }
      }
      const double v[5] = {ax, ay, az, 0.0, pf};
      e64_finish(w, v, x, P, t0, lane, false, false);
    }
    // P2P pairs as the reference counts them (src/Traverser.h:27)
    c_pp += nsrc * (unsigned long long)ntot;
    if (P.bucket_work && lane == 0) P.bucket_work[b] += nsrc * (unsigned long long)ntot;
  }
  if (lane == 0) atomicAdd(&P.counters[0], c_pp);
}

void launch_eval_lists_f64(const TravParams& P, const ListParams& L, const Mom* mom, int grid, cudaStream_t st,
                           unsigned* work2) {
  TravParams Q = P;
  Q.work = work2;
  note_launch();
  eval_p2c_f64<<<grid, kE64Warps * 32, 0, st>>>(P, L);
  note_launch();
  eval_p2p_f64<<<grid, kE64Warps * 32, 0, st>>>(Q, L, mom);
}

}  // namespace pt
