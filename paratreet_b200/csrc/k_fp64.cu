// k_fp64.cu -- FP64 kernels (this file is compiled with -fmad=false).
//
//  K6 upward pass
//     leaf_moments     CentroidData(particles, n, depth),
//                      examples/CentroidData.h:41-59, accumulating
//                      MultipoleMoments::operator+=(Particle) in particle order
//                      (examples/MultipoleMoments.h:274-353, non-HEXADECAPOLE)
//     upward_level     Subtree::populateTree (src/Subtree.h:352-384): every
//                      parent combines its children with CentroidData::
//                      operator+= (examples/CentroidData.h:61-73,
//                      examples/MultipoleMoments.h:204-271, :458-469) in the
//                      order the reference's FIFO delivers them.  That order is
//                      reproduced without a queue: leaves hold FIFO rank
//                      (0, leaf DFS rank), empty leaves (0, n_leaves + rank),
//                      and a parent's rank is (1 + chain, t) of its
//                      latest-ranked child -- parents enter the FIFO in the
//                      order their last child leaves it.
//     finalize         per-node traversal records (WalkRec, QuadRec).
//  K7 traverse_f64     warp-per-bucket walk (pt_walk.cuh) with the FP64
//                      GravityVisitor leaf / node evaluators -- bit-identical
//                      to the reference built -DUSE_DOUBLE_FP.
//  K8 kick_perturb     Particle::kick + Particle::perturb
//                      (src/Particle.C:7-21) fused, and the leapfrog variant.
//  K9 direct_sum       FP64 spline direct sum (force-error yardstick).
#include <cfloat>

#include "pt_fp64.cuh"
#include "pt_internal.cuh"
#include "pt_walk.cuh"

namespace pt {

__device__ __forceinline__ void mom_clear(Mom& q) {
  q.mass = 0.0; q.cm[0] = q.cm[1] = q.cm[2] = 0.0; q.soft = 0.0; q.radius = 0.0;
  q.xx = q.xy = q.xz = q.yy = q.yz = q.zz = 0.0;
  q.lo[0] = q.lo[1] = q.lo[2] = DBL_MAX;
  q.hi[0] = q.hi[1] = q.hi[2] = -DBL_MAX;
  q.reach = 0.0;
  q.soft_max = 0.0;
}

// MultipoleMoments::operator+=(Particle), examples/MultipoleMoments.h:274-353.
__device__ __forceinline__ void mom_add_particle(Mom& q, double px, double py, double pz, double pm, double ps) {
  double m1 = q.mass;
  q.mass += pm;
  if (q.mass == 0.0) {
    q.soft = 0.5 * (q.soft + ps);
    q.cm[0] = 0.5 * (q.cm[0] + px);
    q.cm[1] = 0.5 * (q.cm[1] + py);
    q.cm[2] = 0.5 * (q.cm[2] + pz);
    return;
  }
  q.soft = (m1 * q.soft + pm * ps) / q.mass;
  double c0 = q.cm[0], c1 = q.cm[1], c2 = q.cm[2];
  q.cm[0] = (m1 * q.cm[0] + pm * px) / q.mass;
  q.cm[1] = (m1 * q.cm[1] + pm * py) / q.mass;
  q.cm[2] = (m1 * q.cm[2] + pm * pz) / q.mass;
  double d0 = c0 - q.cm[0], d1 = c1 - q.cm[1], d2 = c2 - q.cm[2];
  q.xx += m1 * d0 * d0;
  q.yy += m1 * d1 * d1;
  q.zz += m1 * d2 * d2;
  q.xy += m1 * d0 * d1;
  q.xz += m1 * d0 * d2;
  q.yz += m1 * d1 * d2;
  d0 = px - q.cm[0];
  d1 = py - q.cm[1];
  d2 = pz - q.cm[2];
  q.xx += pm * d0 * d0;
  q.yy += pm * d1 * d1;
  q.zz += pm * d2 * d2;
  q.xy += pm * d0 * d1;
  q.xz += pm * d0 * d2;
  q.yz += pm * d1 * d2;
}

// CentroidData::operator+= with MultipoleMoments::operator+=(MultipoleMoments).
__device__ __forceinline__ void mom_combine(Mom& q, int& count, const Mom& c, int ccount) {
  for (int d = 0; d < 3; d++) {
    if (c.lo[d] < q.lo[d]) q.lo[d] = c.lo[d];
    if (c.hi[d] > q.hi[d]) q.hi[d] = c.hi[d];
  }
  double m1 = q.mass;
  q.mass += c.mass;
  if (q.mass == 0.0) {
    q.soft = 0.5 * (q.soft + c.soft);
    for (int d = 0; d < 3; d++) q.cm[d] = 0.5 * (q.cm[d] + c.cm[d]);
  } else if (m1 == 0.0) {
    q.mass = c.mass; q.soft = c.soft; q.radius = c.radius;
    q.cm[0] = c.cm[0]; q.cm[1] = c.cm[1]; q.cm[2] = c.cm[2];
    q.xx = c.xx; q.xy = c.xy; q.xz = c.xz; q.yy = c.yy; q.yz = c.yz; q.zz = c.zz;
  } else if (c.mass != 0.0) {
    q.soft = (m1 * q.soft + c.mass * c.soft) / q.mass;
    double c0 = q.cm[0], c1 = q.cm[1], c2 = q.cm[2];
    for (int d = 0; d < 3; d++) q.cm[d] = (m1 * q.cm[d] + c.mass * c.cm[d]) / q.mass;
    double d0 = c0 - q.cm[0], d1 = c1 - q.cm[1], d2 = c2 - q.cm[2];
    q.xx += m1 * d0 * d0;
    q.yy += m1 * d1 * d1;
    q.zz += m1 * d2 * d2;
    q.xy += m1 * d0 * d1;
    q.xz += m1 * d0 * d2;
    q.yz += m1 * d1 * d2;
    d0 = c.cm[0] - q.cm[0];
    d1 = c.cm[1] - q.cm[1];
    d2 = c.cm[2] - q.cm[2];
    q.xx += c.xx + c.mass * d0 * d0;
    q.yy += c.yy + c.mass * d1 * d1;
    q.zz += c.zz + c.mass * d2 * d2;
    q.xy += c.xy + c.mass * d0 * d1;
    q.xz += c.xz + c.mass * d0 * d2;
    q.yz += c.yz + c.mass * d1 * d2;
  }
  count += ccount;
  if (count > 1) {
    double e[3];
    for (int d = 0; d < 3; d++) {
      double a = q.cm[d] - q.lo[d], b = q.hi[d] - q.cm[d];
      e[d] = (a > b) ? a : b;
    }
    q.radius = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  } else {
    q.radius = 1.0;
  }
}

__global__ void __launch_bounds__(256) leaf_moments(Nodes nd, int64_t nnodes, Particles p) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nnodes) return;
  Mom q;
  mom_clear(q);
  int cnt = 0;
  if (nd.type[i] == kTypeLeaf) {
    int s0 = nd.pstart[i], sn = nd.pcount[i];
    for (int j = s0; j < s0 + sn; j++) {
      double px = p.x[j], py = p.y[j], pz = p.z[j];
      mom_add_particle(q, px, py, pz, p.m[j], p.soft[j]);
      if (px < q.lo[0]) q.lo[0] = px;
      if (py < q.lo[1]) q.lo[1] = py;
      if (pz < q.lo[2]) q.lo[2] = pz;
      if (px > q.hi[0]) q.hi[0] = px;
      if (py > q.hi[1]) q.hi[1] = py;
      if (pz > q.hi[2]) q.hi[2] = pz;
    }
    cnt = sn;
    if (cnt > 1) {
      double dx = q.hi[0] - q.lo[0], dy = q.hi[1] - q.lo[1], dz = q.hi[2] - q.lo[2];
      q.radius = 0.5 * sqrt(dx * dx + dy * dy + dz * dz);
    } else {
      q.radius = 1.0;
    }
    // not part of the reference's data: reach and max softening of the leaf,
    // used only to select the mixed form's unsoftened fast path
    double r2max = 0.0, smax = 0.0;
    for (int j = s0; j < s0 + sn; j++) {
      double dx = p.x[j] - q.cm[0], dy = p.y[j] - q.cm[1], dz = p.z[j] - q.cm[2];
      r2max = fmax(r2max, dx * dx + dy * dy + dz * dz);
      smax = fmax(smax, p.soft[j]);
    }
    q.reach = sqrt(r2max);
    q.soft_max = smax;
  }
  nd.mom[i] = q;
  nd.count[i] = cnt;
}

__global__ void __launch_bounds__(128) upward_level(Nodes nd, int64_t begin, int64_t count) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  int64_t i = begin + t;
  if (nd.type[i] != kTypeInternal) return;
  int c0 = nd.first_child[i];
  uint64_t f[8];
  int ord[8];
  for (int c = 0; c < 8; c++) {
    f[c] = nd.fifo[c0 + c];
    ord[c] = c;
  }
  // ascending FIFO rank (all distinct): insertion sort of 8
  for (int a = 1; a < 8; a++) {
    int k = ord[a];
    int b = a - 1;
    while (b >= 0 && f[ord[b]] > f[k]) {
      ord[b + 1] = ord[b];
      b--;
    }
    ord[b + 1] = k;
  }
  Mom q;
  mom_clear(q);
  int cnt = 0;
  for (int a = 0; a < 8; a++) {
    int c = c0 + ord[a];
    mom_combine(q, cnt, nd.mom[c], nd.count[c]);
  }
  uint64_t last = f[ord[7]];
  nd.fifo[i] = (((last >> 40) + 1ull) << 40) | (last & ((1ull << 40) - 1ull));
  nd.mom[i] = q;
  nd.count[i] = cnt;
}

__global__ void __launch_bounds__(256) finalize_records(Nodes nd, int64_t nnodes, double gfac, int want_f32) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nnodes) return;
  const Mom q = nd.mom[i];
  WalkRec w;
  w.cm[0] = q.cm[0]; w.cm[1] = q.cm[1]; w.cm[2] = q.cm[2];
  w.type = nd.type[i];
  if (w.type == kTypeLeaf) {
    w.reach = q.reach;
    w.soft_max = q.soft_max;
  } else {
    w.orsq = q.radius * q.radius * gfac;  // GravityVisitor::open, :164
    w.soft = q.soft;
  }
  w.first_child = nd.first_child[i];
  w.count = nd.count[i];
  w.pstart = nd.pstart[i];
  w.pcount = nd.pcount[i];
  w.pad = 0;
  nd.walk[i] = w;
  if (i >= 1) {
    nd.walks[walk_sib_index(i, 0)] = make_double2(w.cm[0], w.cm[1]);
    nd.walks[walk_sib_index(i, 1)] = make_double2(w.cm[2], w.orsq);
    nd.walks[walk_sib_index(i, 2)] = make_double2(w.soft, __hiloint2double((min(w.count, 1 << 27) << 3) | w.type, w.first_child));
  }
  QuadRec r;
  r.mass = q.mass; r.soft = q.soft;
  r.xx = q.xx; r.xy = q.xy; r.xz = q.xz; r.yy = q.yy; r.yz = q.yz; r.zz = q.zz;
  nd.quad[i] = r;
  if (want_f32) {
    QuadRecF rf;
    rf.mass = (float)q.mass; rf.soft = (float)q.soft;
    rf.xx = (float)q.xx; rf.xy = (float)q.xy; rf.xz = (float)q.xz;
    rf.yy = (float)q.yy; rf.yz = (float)q.yz; rf.zz = (float)q.zz;
    nd.quadf[i] = rf;
  }
}

// ---------------------------------------------------------------- traversal
constexpr int kTravWarps = 4;

struct F64Eval {
  const Particles* p;
  const WalkRec* walk;
  const QuadRec* quad;
  double* stage;  // this warp's [5][32] source staging
  int lane, nt;
  double xi, yi, zi, si;
  double ax, ay, az, pot, potf;
  double ox, oy, oz;
  const BucketGeom* g;
  unsigned long long n_pp, n_pc;
  int record;
  int64_t nlist, lbase;
  int32_t* lnode;
  int8_t* lkind;

  // GravityVisitor::leaf, examples/GravityVisitor.h:144-160
  __device__ void p2p(int node) {
    const int s0 = walk[node].pstart, sn = walk[node].pcount;
    double pax = 0.0, pay = 0.0, paz = 0.0, ppf = 0.0;
    for (int base = 0; base < sn; base += 32) {
      int cnt = min(32, sn - base);
      __syncwarp();
      if (lane < cnt) {
        int j = s0 + base + lane;
        stage[0 * 32 + lane] = p->x[j];
        stage[1 * 32 + lane] = p->y[j];
        stage[2 * 32 + lane] = p->z[j];
        stage[3 * 32 + lane] = p->m[j];
        stage[4 * 32 + lane] = p->soft[j];
      }
      __syncwarp();
      if (lane < nt) {
        for (int j = 0; j < cnt; j++) {
          double xs = stage[j], ys = stage[32 + j], zs = stage[64 + j], ms = stage[96 + j], ss = stage[128 + j];
          double dx = (xs + ox) - xi;
          double dy = (ys + oy) - yi;
          double dz = (zs + oz) - zi;
          double rsq = dx * dx + dy * dy + dz * dz;
          double twoh = ss + si;
          if (rsq != 0) {
            double a, b;
            spline_f64(rsq, twoh, a, b);
            double bm = b * ms;
            pax += dx * bm;
            pay += dy * bm;
            paz += dz * bm;
            ppf += -ms * a;
          }
        }
      }
    }
    ax += pax;
    ay += pay;
    az += paz;
    potf += ppf;
    n_pp += (unsigned long long)sn * (unsigned long long)nt;
    if (record) {
      if (lane == 0) { lnode[lbase + nlist] = node; lkind[lbase + nlist] = 0; }
      ++nlist;
    }
  }

  // GravityVisitor::node, examples/GravityVisitor.h:184-224 (non-HEXADECAPOLE);
  // mono = openSoftening held (decided in the walk), i.e. addGravity (:130-139)
  __device__ void p2c(int node, bool mono) {
    const WalkRec w = walk[node];
    const QuadRec q = quad[node];
    n_pc += (unsigned long long)nt;
    if (record) {
      if (lane == 0) { lnode[lbase + nlist] = node; lkind[lbase + nlist] = mono ? 2 : 1; }
      ++nlist;
    }
    if (w.count == 0) return;
    const double cx = w.cm[0] + ox, cy = w.cm[1] + oy, cz = w.cm[2] + oz;
    if (mono) {
      if (lane < nt) {  // addGravity, :130-139
        double dx = cx - xi, dy = cy - yi, dz = cz - zi;
        double rsq = dx * dx + dy * dy + dz * dz;
        if (rsq != 0) {
          double f = q.mass / (rsq * sqrt(rsq));
          ax += dx * f;
          ay += dy * f;
          az += dz * f;
          potf += -q.mass / sqrt(rsq);
        }
      }
      return;
    }
    if (lane < nt) {
      double rx = (xi - w.cm[0]) - ox;
      double ry = (yi - w.cm[1]) - oy;
      double rz = (zi - w.cm[2]) - oz;
      double rsq = rx * rx + ry * ry + rz * rz;
      double dir = 1.0 / sqrt(rsq);
      double twoh = q.soft + si;
      double a, b, c, d;
      splineq_f64(dir, rsq, twoh, a, b, c, d);
      double qx = q.xx * rx + q.xy * ry + q.xz * rz;
      double qy = q.xy * rx + q.yy * ry + q.yz * rz;
      double qz = q.xz * rx + q.yz * ry + q.zz * rz;
      double qir = 0.5 * (qx * rx + qy * ry + qz * rz);
      double tr = 0.5 * (q.xx + q.yy + q.zz);
      double qir3 = b * q.mass + d * qir - c * tr;
      double pp = -q.mass * a - c * qir + b * tr;
      pot += pp;
      potf += pp;
      ax += -qir3 * rx + c * qx;
      ay += -qir3 * ry + c * qy;
      az += -qir3 * rz + c * qz;
    }
  }
};

__global__ void __launch_bounds__(kTravWarps * 32) traverse_f64(TravParams P, const Mom* __restrict__ mom) {
  __shared__ WalkFrame stacks[kTravWarps][kWalkStack];
  __shared__ int32_t queues[kTravWarps][kBfsQueue];  // basic-down order only
  __shared__ double stage[kTravWarps][5 * 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long c_pp = 0, c_pc = 0, c_open = 0;
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(P.work, 1u);
    bi = __shfl_sync(kFull, bi, 0);
    int64_t b = P.b_begin + (int64_t)bi;
    if (b >= P.b_end) break;
    const int tnode = P.buckets[b];
    if (tnode < 0 || tnode >= P.nnodes) {
      if (lane == 0) atomicOr(P.status, kErrCapacity);
      continue;
    }
    BucketGeom g;
    load_bucket_geom(mom, tnode, g);
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    if (P.mode == 1) {  // count the interaction list only
      ListRecorder rec{lane, 1, 0, 0, nullptr, nullptr};
      if (!(P.bfs ? walk_bucket_bfs(P.walk, P.nnodes, g, P.ox, P.oy, P.oz, queues[wid], kBfsQueue, lane, rec,
                                    c_open, P.status)
                  : walk_bucket(P.walk, P.nnodes, g, P.ox, P.oy, P.oz, stacks[wid], lane, rec, c_open, P.status)) &&
          lane == 0)
        atomicOr(P.status, kErrStack);
      if (lane == 0) P.list_count[b - P.b_begin] = rec.n;
      continue;
    }
    // A bucket holds more than 32 particles only when more than `bucket`
    // particles share one 63-bit key (depth-21 leaf); its targets are then
    // walked in chunks of 32 (the decisions depend on the bucket only).
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      unsigned long long opens = 0;
      F64Eval ev;
      ev.p = &P.p;
      ev.walk = P.walk;
      ev.quad = P.quad;
      ev.stage = stage[wid];
      ev.lane = lane;
      ev.nt = nt;
      ev.xi = ev.yi = ev.zi = ev.si = 0.0;
      if (lane < nt) {
        ev.xi = P.p.x[t0 + lane];
        ev.yi = P.p.y[t0 + lane];
        ev.zi = P.p.z[t0 + lane];
        ev.si = P.p.soft[t0 + lane];
      }
      ev.ax = ev.ay = ev.az = ev.pot = ev.potf = 0.0;
      if (P.accumulate && lane < nt) {  // later replica walks continue each particle's sum
        ev.ax = P.p.ax[t0 + lane];
        ev.ay = P.p.ay[t0 + lane];
        ev.az = P.p.az[t0 + lane];
        ev.pot = P.p.pot[t0 + lane];
        ev.potf = P.p.potf[t0 + lane];
      }
      ev.ox = P.ox; ev.oy = P.oy; ev.oz = P.oz;
      ev.g = &g;
      ev.n_pp = 0; ev.n_pc = 0;
      ev.record = (P.mode == 2 && tc == 0);
      ev.nlist = 0;
      ev.lbase = ev.record ? P.list_off[b - P.b_begin] : 0;
      ev.lnode = P.list_node;
      ev.lkind = P.list_kind;
      if (!(P.bfs ? walk_bucket_bfs(P.walk, P.nnodes, g, P.ox, P.oy, P.oz, queues[wid], kBfsQueue, lane, ev,
                                    opens, P.status)
                  : walk_bucket(P.walk, P.nnodes, g, P.ox, P.oy, P.oz, stacks[wid], lane, ev, opens, P.status)) &&
          lane == 0)
        atomicOr(P.status, kErrStack);
      if (tc == 0) c_open += opens;
      if (lane < nt) {
        int i = t0 + lane;
        P.p.ax[i] = ev.ax;
        P.p.ay[i] = ev.ay;
        P.p.az[i] = ev.az;
        P.p.pot[i] = ev.pot;
        P.p.potf[i] = ev.potf;
      }
      c_pp += ev.n_pp;
      c_pc += ev.n_pc;
      if (P.bucket_work && lane == 0) {  // this chunk's interactions, added to the bucket's
        unsigned long long wk = ev.n_pp + ev.n_pc;
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

// Frozen-list replay: evaluates each bucket's recorded interaction list (in the
// recorded order, i.e. the walk's) with the FP64 evaluator, without walking.
// Used to differentiate the force pass for a fixed interaction list.
__global__ void __launch_bounds__(kTravWarps * 32) replay_f64(TravParams P) {
  __shared__ double stage[kTravWarps][5 * 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(P.work, 1u);
    bi = __shfl_sync(kFull, bi, 0);
    const int64_t b = P.b_begin + (int64_t)bi;
    if (b >= P.b_end) break;
    const int tnode = P.buckets[b];
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    const int64_t e0 = P.list_off[b - P.b_begin], e1 = P.list_off[b - P.b_begin + 1];
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      F64Eval ev;
      ev.p = &P.p;
      ev.walk = P.walk;
      ev.quad = P.quad;
      ev.stage = stage[wid];
      ev.lane = lane;
      ev.nt = nt;
      ev.xi = ev.yi = ev.zi = ev.si = 0.0;
      if (lane < nt) {
        ev.xi = P.p.x[t0 + lane];
        ev.yi = P.p.y[t0 + lane];
        ev.zi = P.p.z[t0 + lane];
        ev.si = P.p.soft[t0 + lane];
      }
      ev.ax = ev.ay = ev.az = ev.pot = ev.potf = 0.0;
      ev.ox = P.ox; ev.oy = P.oy; ev.oz = P.oz;
      ev.g = nullptr;
      ev.n_pp = 0; ev.n_pc = 0;
      ev.record = 0;
      ev.nlist = 0;
      ev.lbase = 0;
      ev.lnode = nullptr;
      ev.lkind = nullptr;
      for (int64_t e = e0; e < e1; e++) {
        const int node = P.list_node[e];
        const int kind = P.list_kind[e];
        if (node < 0 || node >= P.nnodes) {
          if (lane == 0) atomicOr(P.status, kErrCapacity);
          continue;
        }
        if (kind == 0) ev.p2p(node);
        else ev.p2c(node, kind == 2);
      }
      if (lane < nt) {
        const int i = t0 + lane;
        P.p.ax[i] = ev.ax;
        P.p.ay[i] = ev.ay;
        P.p.az[i] = ev.az;
        P.p.pot[i] = ev.pot;
        P.p.potf[i] = ev.potf;
      }
    }
  }
}

// ---------------------------------------------------------------- integrate
// src/Particle.C:7-9 (kick) then :11-21 (perturb) for the same dt.
__global__ void __launch_bounds__(256) kick_perturb(Particles p, int64_t n, double dt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double ax = p.ax[i], ay = p.ay[i], az = p.az[i];
    double vx = p.vx[i], vy = p.vy[i], vz = p.vz[i];
    vx += ax * dt / 2;
    vy += ay * dt / 2;
    vz += az * dt / 2;
    vx += (ax * dt / 2);
    vy += (ay * dt / 2);
    vz += (az * dt / 2);
    p.x[i] += (vx * dt);
    p.y[i] += (vy * dt);
    p.z[i] += (vz * dt);
    p.vx[i] = vx;
    p.vy[i] = vy;
    p.vz[i] = vz;
  }
}

// Leapfrog halves: kick (v += a dt/2) and drift (x += v dt).
__global__ void __launch_bounds__(256) kick_half(Particles p, int64_t n, double dt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    p.vx[i] += p.ax[i] * dt / 2;
    p.vy[i] += p.ay[i] * dt / 2;
    p.vz[i] += p.az[i] * dt / 2;
  }
}
__global__ void __launch_bounds__(256) drift(Particles p, int64_t n, double dt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    p.x[i] += (p.vx[i] * dt);
    p.y[i] += (p.vy[i] * dt);
    p.z[i] += (p.vz[i] * dt);
  }
}

// ---------------------------------------------------------------- direct sum
constexpr int kDirTile = 256;

__global__ void __launch_bounds__(kDirTile) direct_sum_f64(const double* __restrict__ x, const double* __restrict__ y,
                                                           const double* __restrict__ z, const double* __restrict__ m,
                                                           const double* __restrict__ soft, int64_t n,
                                                           const int32_t* __restrict__ tgt, int64_t nt, int nsplit,
                                                           double* __restrict__ part) {
  // grid: (target blocks, nsplit source slices); part[(slice * nt + t) * 4 + k]
  __shared__ double sx[kDirTile], sy[kDirTile], sz[kDirTile], sm[kDirTile], ss[kDirTile];
  int64_t t = blockIdx.x * (int64_t)kDirTile + threadIdx.x;
  bool ok = t < nt;
  int i = ok ? tgt[t] : 0;
  double xi = x[i], yi = y[i], zi = z[i], si = soft[i];
  double ax = 0.0, ay = 0.0, az = 0.0, pp = 0.0;
  int64_t per = (n + nsplit - 1) / nsplit;
  int64_t j0 = per * blockIdx.y, j1 = min(n, j0 + per);
  for (int64_t base = j0; base < j1; base += kDirTile) {
    __syncthreads();
    int64_t j = base + threadIdx.x;
    if (j < j1) { sx[threadIdx.x] = x[j]; sy[threadIdx.x] = y[j]; sz[threadIdx.x] = z[j]; sm[threadIdx.x] = m[j]; ss[threadIdx.x] = soft[j]; }
    __syncthreads();
    int cnt = (int)min((int64_t)kDirTile, j1 - base);
    for (int k = 0; k < cnt; k++) {
      double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
      double rsq = dx * dx + dy * dy + dz * dz;
      if (rsq != 0) {
        double a, b;
        spline_f64(rsq, ss[k] + si, a, b);
        double bm = b * sm[k];
        ax += dx * bm;
        ay += dy * bm;
        az += dz * bm;
        pp += -sm[k] * a;
      }
    }
  }
  if (ok) {
    double* o = part + ((int64_t)blockIdx.y * nt + t) * 4;
    o[0] = ax; o[1] = ay; o[2] = az; o[3] = pp;
  }
}

// ---------------------------------------------------------------- launchers
static inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

void launch_leaf_moments(Nodes nd, int64_t nnodes, Particles p, cudaStream_t st) {
  if (nnodes > 0) { note_launch(); leaf_moments<<<blocks_for(nnodes), 256, 0, st>>>(nd, nnodes, p); }
}
void launch_upward_level(Nodes nd, int64_t begin, int64_t count, cudaStream_t st) {
  if (count > 0) { note_launch(); upward_level<<<blocks_for(count, 128), 128, 0, st>>>(nd, begin, count); }
}
void launch_finalize(Nodes nd, int64_t nnodes, double gfac, int want_f32, cudaStream_t st) {
  if (nnodes > 0) { note_launch(); finalize_records<<<blocks_for(nnodes), 256, 0, st>>>(nd, nnodes, gfac, want_f32); }
}
void launch_traverse_f64(const TravParams& P, const Mom* mom, int grid, cudaStream_t st) {
  note_launch();
  traverse_f64<<<grid, kTravWarps * 32, 0, st>>>(P, mom);
}
void launch_replay_f64(const TravParams& P, int grid, cudaStream_t st) {
  note_launch();
  replay_f64<<<grid, kTravWarps * 32, 0, st>>>(P);
}
void launch_kick_perturb(Particles p, int64_t n, double dt, int grid, cudaStream_t st) {
  note_launch();
  kick_perturb<<<grid, 256, 0, st>>>(p, n, dt);
}
void launch_kick_half(Particles p, int64_t n, double dt, int grid, cudaStream_t st) {
  note_launch();
  kick_half<<<grid, 256, 0, st>>>(p, n, dt);
}
void launch_drift(Particles p, int64_t n, double dt, int grid, cudaStream_t st) {
  note_launch();
  drift<<<grid, 256, 0, st>>>(p, n, dt);
}
void launch_direct_sum(const double* x, const double* y, const double* z, const double* m, const double* soft,
                       int64_t n, const int32_t* tgt, int64_t nt, int nsplit, double* part, cudaStream_t st) {
  dim3 grid(blocks_for(nt, kDirTile), nsplit);
  note_launch();
  direct_sum_f64<<<grid, kDirTile, 0, st>>>(x, y, z, m, soft, n, tgt, nt, nsplit, part);
}

}  // namespace pt
