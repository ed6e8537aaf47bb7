// pt_walk.cuh -- the ordered warp-per-bucket tree walk of the FP64 traversal
// (and of interaction-list recording), plus the FP64-exact opening tests that
// every traversal shares.
//
// Semantics: TransposedDownTraverser::recurse (src/Traverser.h:154-217) for
// one target bucket is a pre-order depth-first walk from the root: a Leaf is
// handed to GravityVisitor::leaf (P2P, the bucket itself included), an
// Internal node is tested with GravityVisitor::open and either descended or
// handed to GravityVisitor::node (P2C), an EmptyLeaf is skipped.  Per target
// particle the interactions are applied in exactly that order.
//
// B200 mapping: one warp owns one bucket (lanes = target particles).  When a
// node is opened, lanes 0..7 classify its 8 contiguous children in parallel
// (64-byte WalkRec each, one coalesced 512-byte read) into P2P / P2C
// (quadrupole) / P2C (softened monopole, GravityVisitor::openSoftening) /
// open; four ballots give the per-child masks.  The terminal children before
// the first opened child are handed to the evaluator in child order, the
// remaining masks are pushed on a per-warp shared-memory frame stack, and the
// walk descends.  Every decision is warp-uniform.  The tests use
// __dadd_rn/__dmul_rn so that they evaluate identically (no FMA contraction)
// in every translation unit: all traversal forms see the same interactions.
#pragma once

#include "pt_internal.cuh"

namespace pt {

constexpr int kWalkStack = 32;
constexpr int kBfsQueue = 512;  // pending sibling frames of a breadth-first walk
constexpr unsigned kFull = 0xffffffffu;

// Child classes.
enum : int { kClsNone = 0, kClsP2P = 1, kClsQuad = 2, kClsOpen = 3, kClsMono = 4 };

struct WalkFrame {
  int32_t c0;     // index of child 0
  uint32_t bits;  // P2P (0-7) | P2C quadrupole (8-15) | P2C monopole (16-23) | open (24-31)
};

// Squared gap between a box and a point as Space::intersect of the
// reference's utility submodule accumulates it (stand-in convention: per axis
// d = lo - c if positive, else c - hi if positive, else nothing; summed x, y,
// z).  Written with selects: an axis without a gap adds 0 * 0, which leaves
// the (non-negative) sum unchanged, so the value is the branchy form's bit for
// bit.
__device__ __forceinline__ double box_gap2_exact(const double lo[3], const double hi[3], double cx, double cy,
                                                 double cz) {
  const double c[3] = {cx, cy, cz};
  double dsq = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double a = __dadd_rn(lo[k], -c[k]), b = __dadd_rn(c[k], -hi[k]);
    const double d = (a > 0) ? a : ((b > 0) ? b : 0.0);
    dsq = __dadd_rn(dsq, __dmul_rn(d, d));
  }
  return dsq;
}

// Space::intersect(box, centre, rsq): intersect iff the gap is <= rsq.  Used
// by GravityVisitor::open (:180) and ::openSoftening (:127).
__device__ __forceinline__ bool box_sphere_exact(const double lo[3], const double hi[3], double cx,
                                                 double cy, double cz, double rsq) {
  return box_gap2_exact(lo, hi, cx, cy, cz) <= rsq;
}

// Squared distance from a point to a box (0 inside); conservative helper.
__device__ __forceinline__ double box_dist2(const double lo[3], const double hi[3], double cx, double cy,
                                            double cz) {
  double dsq = 0.0, d;
  if ((d = lo[0] - cx) > 0) dsq += d * d; else if ((d = cx - hi[0]) > 0) dsq += d * d;
  if ((d = lo[1] - cy) > 0) dsq += d * d; else if ((d = cy - hi[1]) > 0) dsq += d * d;
  if ((d = lo[2] - cz) > 0) dsq += d * d; else if ((d = cz - hi[2]) > 0) dsq += d * d;
  return dsq;
}

// GravityVisitor::openSoftening (:122-128): the softening spheres overlap, or
// the target bucket's box meets the source sphere of radius 2*soft; gap2 is
// box_gap2_exact of the bucket box and the source centre (the same gap the
// opening test measured).
__device__ __forceinline__ bool open_softening_gap(double scx, double scy, double scz, double ssoft, double tcx,
                                                   double tcy, double tcz, double tsoft, double gap2) {
  double r1 = __dmul_rn(2.0, ssoft), r2 = __dmul_rn(2.0, tsoft);
  double dx = __dadd_rn(scx, -tcx), dy = __dadd_rn(scy, -tcy), dz = __dadd_rn(scz, -tcz);
  double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  double rs = __dadd_rn(r1, r2);
  if (d2 <= __dmul_rn(rs, rs)) return true;
  return gap2 <= __dmul_rn(r1, r1);
}

__device__ __forceinline__ bool open_softening_exact(double scx, double scy, double scz, double ssoft,
                                                     double tcx, double tcy, double tcz, double tsoft,
                                                     const double lo[3], const double hi[3]) {
  return open_softening_gap(scx, scy, scz, ssoft, tcx, tcy, tcz, tsoft, box_gap2_exact(lo, hi, scx, scy, scz));
}

// Whether a P2P leaf may hold a pair that GravityVisitor::leaf softens (or
// the target itself): the box gap between the target bucket's particle box
// and the leaf's centre (plus offset) is within the leaf's reach plus both
// sides' largest softening.  Conservative: a leaf for which it is false has
// every pair at r >= soft_i + soft_j > 0.  rec = the leaf's WalkRec.
__device__ __forceinline__ bool p2p_leaf_near(const WalkRec* __restrict__ walk, int leaf, const double lo[3],
                                              const double hi[3], double tsoft_max, double ox, double oy,
                                              double oz) {
  const double2* r = reinterpret_cast<const double2*>(walk + leaf);
  const double2 c01 = r[0], c2reach = r[1], smax = r[2];
  const double gap2 = box_gap2_exact(lo, hi, __dadd_rn(c01.x, ox), __dadd_rn(c01.y, oy), __dadd_rn(c2reach.x, oz));
  const double reach = c2reach.y + smax.x + tsoft_max;
  return !(gap2 > reach * reach);
}

struct BucketGeom {
  double lo[3], hi[3];  // target bucket's particle bbox (CentroidData::box)
  double cm[3];         // target bucket's centre of mass
  double soft;          // target bucket's mass-weighted softening
  double soft_max;      // max particle softening in the bucket
};

__device__ __forceinline__ void load_bucket_geom(const Mom* mom, int node, BucketGeom& g) {
  const Mom& q = mom[node];
  g.lo[0] = q.lo[0]; g.lo[1] = q.lo[1]; g.lo[2] = q.lo[2];
  g.hi[0] = q.hi[0]; g.hi[1] = q.hi[1]; g.hi[2] = q.hi[2];
  g.cm[0] = q.cm[0]; g.cm[1] = q.cm[1]; g.cm[2] = q.cm[2];
  g.soft = q.soft;
  g.soft_max = q.soft_max;
}

// Class of one node against the bucket (GravityVisitor::open / node).  The
// box gap of the node's centre (plus offset) serves both the opening test and
// openSoftening's second clause; it is returned in gap2 (-1 where it was not
// needed: leaves, empty nodes, nodes opened by their count).
// The same with the bucket box passed apart (lo, hi: e.g. held in registers).
__device__ __forceinline__ int classify_node_gap(const WalkRec& w, const double lo[3], const double hi[3],
                                                 const BucketGeom& g, double ox, double oy, double oz, double& gap2) {
  gap2 = -1.0;
  if (w.type == kTypeLeaf) return kClsP2P;
  if (w.type != kTypeInternal) return kClsNone;
  if (w.count <= kMinParticleNode) return kClsOpen;
  const double cx = __dadd_rn(w.cm[0], ox), cy = __dadd_rn(w.cm[1], oy), cz = __dadd_rn(w.cm[2], oz);
  gap2 = box_gap2_exact(lo, hi, cx, cy, cz);
  if (gap2 <= w.orsq) return kClsOpen;
  return open_softening_gap(cx, cy, cz, w.soft, g.cm[0], g.cm[1], g.cm[2], g.soft, gap2) ? kClsMono : kClsQuad;
}

// The same without a replica offset (the node's centre as it is).
__device__ __forceinline__ int classify_node_gap_nooff(const WalkRec& w, const double lo[3], const double hi[3],
                                                       const BucketGeom& g, double& gap2) {
  gap2 = -1.0;
  if (w.type == kTypeLeaf) return kClsP2P;
  if (w.type != kTypeInternal) return kClsNone;
  if (w.count <= kMinParticleNode) return kClsOpen;
  gap2 = box_gap2_exact(lo, hi, w.cm[0], w.cm[1], w.cm[2]);
  if (gap2 <= w.orsq) return kClsOpen;
  return open_softening_gap(w.cm[0], w.cm[1], w.cm[2], w.soft, g.cm[0], g.cm[1], g.cm[2], g.soft, gap2) ? kClsMono
                                                                                                       : kClsQuad;
}

__device__ __forceinline__ int classify_node_gap(const WalkRec& w, const BucketGeom& g, double ox, double oy,
                                                 double oz, double& gap2) {
  return classify_node_gap(w, g.lo, g.hi, g, ox, oy, oz, gap2);
}

__device__ __forceinline__ int classify_node(const WalkRec& w, const BucketGeom& g, double ox, double oy, double oz) {
  double gap2;
  return classify_node_gap(w, g, ox, oy, oz, gap2);
}

// Classify up to 8 nodes [c0, c0+nvalid) against the bucket; returns frame bits.
__device__ __forceinline__ uint32_t classify_children(const WalkRec* __restrict__ walk, int64_t nnodes, int c0,
                                                      int nvalid, const BucketGeom& g, double ox, double oy,
                                                      double oz, int lane, unsigned long long& n_open,
                                                      unsigned* status) {
  int code = kClsNone;
  bool internal = false;
  if (lane < nvalid) {
    int64_t idx = (int64_t)c0 + lane;
    if (c0 < 0 || idx >= nnodes) {
      atomicOr(status, kErrCapacity);
    } else {
      const WalkRec w = walk[idx];
      internal = (w.type == kTypeInternal);
      code = classify_node(w, g, ox, oy, oz);
    }
  }
  uint32_t pp = __ballot_sync(kFull, code == kClsP2P) & 0xffu;
  uint32_t pq = __ballot_sync(kFull, code == kClsQuad) & 0xffu;
  uint32_t pm = __ballot_sync(kFull, code == kClsMono) & 0xffu;
  uint32_t op = __ballot_sync(kFull, code == kClsOpen) & 0xffu;
  n_open += (unsigned long long)__popc(__ballot_sync(kFull, internal) & 0xffu);
  return pp | (pq << 8) | (pm << 16) | (op << 24);
}

// Walk the tree for one bucket; ev.p2p(node), ev.p2c(node, mono) are called in
// the reference's per-bucket order.  Returns false on stack overflow.
template <class Eval>
__device__ __forceinline__ bool walk_bucket(const WalkRec* __restrict__ walk, int64_t nnodes, const BucketGeom& g,
                                            double ox, double oy, double oz, WalkFrame* stack, int lane, Eval& ev,
                                            unsigned long long& n_open, unsigned* status) {
  int c0 = 0;  // the root, tested as a one-child frame
  uint32_t bits = classify_children(walk, nnodes, 0, 1, g, ox, oy, oz, lane, n_open, status);
  int sp = 0;
  while (true) {
    if (bits == 0) {
      if (sp == 0) break;
      --sp;
      WalkFrame f = stack[sp];
      c0 = f.c0;
      bits = f.bits;
      continue;
    }
    uint32_t pp = bits & 0xffu, pq = (bits >> 8) & 0xffu, pm = (bits >> 16) & 0xffu, op = bits >> 24;
    int fo = op ? (__ffs(op) - 1) : 8;
    uint32_t low = (1u << fo) - 1u;
    uint32_t run = (pp | pq | pm) & low;
    while (run) {
      int k = __ffs(run) - 1;
      run &= run - 1u;
      if ((pp >> k) & 1u) ev.p2p(c0 + k);
      else ev.p2c(c0 + k, ((pm >> k) & 1u) != 0);
    }
    pp &= ~low;
    pq &= ~low;
    pm &= ~low;
    if (fo < 8) {
      op &= ~(1u << fo);
      uint32_t rem = pp | (pq << 8) | (pm << 16) | (op << 24);
      if (rem) {
        if (sp >= kWalkStack) return false;
        __syncwarp();
        if (lane == 0) stack[sp] = WalkFrame{c0, rem};
        __syncwarp();
        ++sp;
      }
      int nc0 = walk[c0 + fo].first_child;
      c0 = nc0;
      bits = classify_children(walk, nnodes, nc0, 8, g, ox, oy, oz, lane, n_open, status);
    } else {
      bits = 0;
    }
  }
  return true;
}

// The same walk in BasicDownTraverser order (src/Traverser.h:296-330, the
// deque used first in, first out): breadth first per bucket.  Siblings stay
// consecutive in that order, so the unit of the queue is a frame -- the 8
// children of an opened node -- processed in child order, each opened child
// queuing its own frame at the back.  queue is a per-warp ring of qcap frames
// (first-child indices).  Returns false if the ring overflows.
template <class Eval>
__device__ __forceinline__ bool walk_bucket_bfs(const WalkRec* __restrict__ walk, int64_t nnodes,
                                                const BucketGeom& g, double ox, double oy, double oz,
                                                int32_t* queue, int qcap, int lane, Eval& ev,
                                                unsigned long long& n_open, unsigned* status) {
  int c0 = 0;  // the root, as a one-child frame
  uint32_t bits = classify_children(walk, nnodes, 0, 1, g, ox, oy, oz, lane, n_open, status);
  int head = 0, tail = 0;
  while (true) {
    const uint32_t pp = bits & 0xffu, pq = (bits >> 8) & 0xffu, pm = (bits >> 16) & 0xffu, op = bits >> 24;
    uint32_t all = pp | pq | pm | op;
    while (all) {
      const int k = __ffs(all) - 1;
      all &= all - 1u;
      if ((pp >> k) & 1u) {
        ev.p2p(c0 + k);
      } else if (((pq | pm) >> k) & 1u) {
        ev.p2c(c0 + k, ((pm >> k) & 1u) != 0);
      } else {
        if (tail - head >= qcap) return false;
        const int fc = walk[c0 + k].first_child;
        __syncwarp();
        if (lane == 0) queue[tail % qcap] = fc;
        __syncwarp();
        ++tail;
      }
    }
    if (head == tail) break;
    c0 = queue[head % qcap];
    ++head;
    bits = classify_children(walk, nnodes, c0, 8, g, ox, oy, oz, lane, n_open, status);
  }
  return true;
}

// Evaluator that only records / counts the interaction list of a bucket.
// Stored kinds: 0 leaf() P2P, 1 node() quadrupole, 2 node() softened monopole.
struct ListRecorder {
  int lane;
  int mode;  // 1 count, 2 record
  int64_t n;
  int64_t base;
  int32_t* node_out;
  int8_t* kind_out;
  __device__ void p2p(int node) {
    if (mode == 2 && lane == 0) { node_out[base + n] = node; kind_out[base + n] = 0; }
    ++n;
  }
  __device__ void p2c(int node, bool mono) {
    if (mode == 2 && lane == 0) { node_out[base + n] = node; kind_out[base + n] = mono ? 2 : 1; }
    ++n;
  }
};

}  // namespace pt
