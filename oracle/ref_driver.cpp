/*
 * ref_driver.cpp -- TEST INFRASTRUCTURE (oracle).  Never linked into the
 * product.
 *
 * Compiles the reference's OWN gravity sources from where they lie (see
 * oracle/Makefile): examples/GravityVisitor.h, examples/CentroidData.h,
 * examples/MultipoleMoments.h, src/Node.h, src/Particle.{h,C}, src/Utility.h,
 * src/common.h -- built with -DUSE_DOUBLE_FP and without -DHEXADECAPOLE
 * (the monopole+quadrupole branch) and with -ffp-contract=off.  Around them
 * this file restates the Charm++-bound driver pieces, each following the
 * cited reference lines:
 *
 *   universe          src/Driver.h:67-80 (remakeUniverse), bbox from
 *                     src/Reader.C:92 / src/Partition.h:368-378
 *   keys              src/Decomposition.C:58-64
 *   sort              src/Subtree.h:281 (std::sort; stable here, so that
 *                     equal keys keep input order -- the reference's tie
 *                     order is unspecified)
 *   node allocation   src/CacheManager.h:38-43 (FullNodePool::alloc)
 *   tree build        src/Subtree.h:263-267, :293-298, :314-349,
 *                     src/Modularization.C:60-65
 *   upward pass       src/Subtree.h:352-384 (FIFO order)
 *   traversal         src/Traverser.h:154-217 (TransposedDownTraverser::
 *                     recurse) over contiguous groups of buckets, one group
 *                     per Partition (src/Partition.h:129-134)
 *   step              src/Driver.h:183-251: forces -> kick -> perturb ->
 *                     new universe -> rekey; dt from examples/Gravity.C:63-67
 *   SPH density       examples/SPH.C:11-37 and :77-86: the reference's own
 *                     DensityVisitor (examples/DensityVisitor.h) driven by a
 *                     restated up-and-down walk per bucket
 *                     (src/Traverser.h:363-482), then DensityFn with the
 *                     reference's kernelM4 (examples/SPHUtils.h)
 *   periodic          examples/Gravity.C:19-50: EwaldInit on the root's data
 *                     (examples/Ewald.C, compiled in ref_ewald.cpp), the
 *                     (2n+1)^3 replica walks with GravityVisitor offsets, then
 *                     the reference's own LeafEwaldFn (examples/Ewald.h) per
 *                     leaf
 *
 * Deviation for degenerate input only: a node at depth 21 (all 63 key bits
 * used) is made a Leaf even when it holds more than `bucket` particles (the
 * reference would shift its key out of range).
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <queue>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "common.h"
#include "Particle.h"
#include "Utility.h"
#include "CentroidData.h"
#include "Node.h"
#include "GravityVisitor.h"
#include "EwaldData.h"

// Readonly globals of examples/Main.C that Ewald.{h,C} read.
Vector3D<Real> fPeriod(1.0, 1.0, 1.0);
int nReplicas = 0;

// ewaldProxy.ckLocalBranch() of the single-process run: the EwaldData that
// EwaldInit filled.
struct CProxy_EwaldData {
  EwaldData* local = nullptr;
  EwaldData* ckLocalBranch() const { return local; }
};
CProxy_EwaldData ewaldProxy;
template <typename D>
struct Partition;
#define PARATREET_REGISTER_PER_LEAF_FN(name, data, fn) static auto name = fn;
#include "Ewald.h"

// Stand-in for src/ThreadStateHolder.h (a Charm++ group): doSPHCalc hands it
// the reaction on the neighbour ("opposing effect"), summed per particle.
class ThreadStateHolder {
 public:
  std::vector<Vector3D<Real>> acc;
  std::vector<Real> work;
  void applyOpposingEffect(const Particle& b, Vector3D<Real> a, Real w) {
    acc[b.order] += a;
    work[b.order] += w;
  }
};
#include "DensityVisitor.h"
#include "PressureVisitor.h"
#include "SPHUtils.h"

namespace {

using RNode = Node<CentroidData>;
using RFull = FullNode<CentroidData, 8>;

constexpr int kLogBranch = 3;
constexpr int kMaxDepth = 21;

struct ListEntry {
  uint64_t key;
  int kind;  // 0 = leaf (P2P), 1 = node (P2C)
};

struct RefSim {
  // configuration
  int bucket = 16;
  double theta = 0.7;
  double dt_max = 0.01;
  int group = 64;
  int record_lists = 0;
  int threads = 1;
  int periodic = 0;
  double period = 1.0;
  int n_replicas = 0;
  int basic_down = 0;  // Partition::startBasicDown instead of startDown
  // state
  std::vector<Particle> particles;  // sorted by key after each build
  OrientedBox<Real> universe;
  std::deque<RFull> pool;
  std::vector<RNode*> leaves, empty_leaves;
  RNode* root = nullptr;
  // outputs of the last force evaluation
  std::vector<double> acc, pot;  // original order, 3N and N
  std::vector<uint64_t> keys;    // original order
  std::vector<std::vector<ListEntry>> lists;  // per bucket (DFS leaf order)
  unsigned long long n_pp = 0, n_pc = 0, n_open = 0;
  double last_dt = 0.0;
  double t_build = 0.0, t_traverse = 0.0;
};

Node<CentroidData>::Type getType(size_t n, size_t B, int depth) {
  if (n == 0) return RNode::Type::EmptyLeaf;
  if (n <= B || depth >= kMaxDepth) return RNode::Type::Leaf;
  return RNode::Type::Internal;
}

RNode* makeNode(RefSim& s, Key key, RNode::Type type, int depth, int n, Particle* p, RNode* parent) {
  if (type == RNode::Type::Leaf) {
    s.pool.emplace_back(key, type, depth, n, p, parent, 0, 0);
  } else {
    s.pool.emplace_back(key, type, depth, parent, 0, 0);
  }
  return &s.pool.back();
}

void handlePossibleLeaf(RefSim& s, RNode* node) {
  if (node->type == RNode::Type::EmptyLeaf) s.empty_leaves.push_back(node);
  else if (node->type == RNode::Type::Leaf) s.leaves.push_back(node);
}

void recursiveBuild(RefSim& s, RNode* node, Particle* np, size_t n) {
  Key child_key = node->key << kLogBranch;
  int start = 0;
  int finish = (int)n;
  std::function<bool(const Particle&, Key)> compGE = [](const Particle& a, Key b) { return a.key >= b; };
  for (int i = 0; i < node->n_children; i++) {
    int first_ge = finish;
    if (i < node->n_children - 1) {
      Key sib = Utility::removeLeadingZeros(child_key + 1, kLogBranch);
      first_ge = Utility::binarySearchComp(sib, np, start, finish, compGE);
    }
    int cn = first_ge - start;
    RNode* child = makeNode(s, child_key, getType(cn, s.bucket, node->depth + 1), node->depth + 1, cn,
                            np + start, node);
    node->exchangeChild(i, child);
    if (child->isLeaf()) handlePossibleLeaf(s, child);
    else recursiveBuild(s, child, np + start, cn);
    start = first_ge;
    child_key++;
  }
}

void populateTree(RefSim& s) {
  std::queue<RNode*> going_up;
  for (auto* l : s.leaves) going_up.push(l);
  for (auto* e : s.empty_leaves) going_up.push(e);
  while (!going_up.empty()) {
    RNode* node = going_up.front();
    going_up.pop();
    if (node == s.root) continue;  // tp_key == root key; no canopy above it
    RNode* parent = node->parent;
    parent->data += node->data;
    parent->wait_count--;
    if (parent->wait_count == 0) going_up.push(parent);
  }
}

void remakeUniverse(RefSim& s, const OrientedBox<Real>& box) {
  Vector3D<Real> bsize = box.size();
  Real mx = (bsize.x > bsize.y) ? bsize.x : bsize.y;
  mx = (mx > bsize.z) ? mx : bsize.z;
  Vector3D<Real> bcenter = box.center();
  const Real fEps = 1.0 + 1.91e-6;
  bsize = Vector3D<Real>(fEps * 0.5 * mx);
  s.universe = OrientedBox<Real>(bcenter - bsize, bcenter + bsize);
}

void assignKeys(RefSim& s) {
  for (auto& p : s.particles) {
    p.key = SFC::generateKey(p.position, s.universe);
    p.key |= (Key)1 << (KEY_BITS - 1);
  }
}

void buildTree(RefSim& s) {
  std::stable_sort(s.particles.begin(), s.particles.end());
  s.pool.clear();
  s.leaves.clear();
  s.empty_leaves.clear();
  size_t n = s.particles.size();
  Key root_key = 1;
  s.root = makeNode(s, root_key, getType(n, s.bucket, 0), Utility::getDepthFromKey(root_key, kLogBranch),
                    (int)n, s.particles.data(), nullptr);
  if (s.root->isLeaf()) handlePossibleLeaf(s, s.root);
  else recursiveBuild(s, s.root, s.particles.data(), n);
  populateTree(s);
}

// One Partition's worth of TransposedDownTraverser::recurse.
struct GroupTrav {
  RefSim& s;
  GravityVisitor v;
  size_t b0, nb;
  unsigned long long pp = 0, pc = 0, op = 0;
  GroupTrav(RefSim& sim, size_t b0_, size_t nb_, Vector3D<Real> offset = Vector3D<Real>(0, 0, 0))
      : s(sim), v(offset, sim.theta), b0(b0_), nb(nb_) {}

  void recurse(RNode* node, const std::vector<char>& active) {
    std::vector<char> next(nb, 0);
    bool cont = false;
    switch (node->type) {
      case RNode::Type::Leaf:
        for (size_t b = 0; b < nb; b++) {
          if (!active[b]) continue;
          RNode* tgt = s.leaves[b0 + b];
          v.leaf(*node, *tgt);
          pp += (unsigned long long)node->n_particles * tgt->n_particles;
          if (s.record_lists) s.lists[b0 + b].push_back({node->key, 0});
        }
        break;
      case RNode::Type::Internal:
        for (size_t b = 0; b < nb; b++) {
          if (!active[b]) continue;
          RNode* tgt = s.leaves[b0 + b];
          bool open = v.open(*node, *tgt);
          op++;
          next[b] = open;
          if (open) {
            cont = true;
          } else {
            v.node(*node, *tgt);
            pc += (unsigned long long)tgt->n_particles;
            if (s.record_lists) s.lists[b0 + b].push_back({node->key, 1});
          }
        }
        break;
      default:
        break;
    }
    if (cont) {
      for (int c = 0; c < node->n_children; c++) recurse(node->getChild(c), next);
    }
  }
};

// BasicDownTraverser::doTrav (src/Traverser.h:296-330) for one bucket: a
// deque, children pushed at the front, nodes taken from the back.
void basic_down_bucket(RefSim& s, size_t b, unsigned long long& pp, unsigned long long& pc,
                       unsigned long long& op) {
  GravityVisitor v(Vector3D<Real>(0, 0, 0), s.theta);
  RNode* bucket = s.leaves[b];
  std::deque<RNode*> nodes;
  nodes.push_front(s.root);
  while (!nodes.empty()) {
    RNode* node = nodes.back();
    nodes.pop_back();
    switch (node->type) {
      case RNode::Type::Leaf:
        v.leaf(*node, *bucket);
        pp += (unsigned long long)node->n_particles * bucket->n_particles;
        if (s.record_lists) s.lists[b].push_back({node->key, 0});
        break;
      case RNode::Type::Internal:
        op++;
        if (v.open(*node, *bucket)) {
          for (int idx = 0; idx < node->n_children; idx++) nodes.push_front(node->getChild(idx));
        } else {
          v.node(*node, *bucket);
          pc += (unsigned long long)bucket->n_particles;
          if (s.record_lists) s.lists[b].push_back({node->key, 1});
        }
        break;
      default:
        break;
    }
  }
}

void traverse(RefSim& s) {
  size_t nb = s.leaves.size();
  if (s.record_lists) {
    s.lists.assign(nb, {});
  }
  size_t ngroups = (nb + s.group - 1) / s.group;
  unsigned long long pp = 0, pc = 0, op = 0;
  EwaldData ewald;
  if (s.periodic) {  // examples/Gravity.C:19-26 (preTraversalFn)
    fPeriod = Vector3D<Real>(s.period, s.period, s.period);
    nReplicas = s.n_replicas;
    ewaldProxy.local = &ewald;
    ewald.EwaldInit(s.root->data, CkCallback());
  }
  if (s.basic_down && !s.periodic) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : pp, pc, op) num_threads(s.threads)
#endif
    for (long b = 0; b < (long)nb; b++) basic_down_bucket(s, (size_t)b, pp, pc, op);
    s.n_pp = pp;
    s.n_pc = pc;
    s.n_open = op;
    return;
  }
  const int nr = s.periodic ? s.n_replicas : 0;
  for (int X = -nr; X <= nr; X++)
    for (int Y = -nr; Y <= nr; Y++)
      for (int Z = -nr; Z <= nr; Z++) {
        Vector3D<Real> offset(X * s.period, Y * s.period, Z * s.period);
        if (!s.periodic) offset = Vector3D<Real>(0, 0, 0);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : pp, pc, op) num_threads(s.threads)
#endif
        for (long g = 0; g < (long)ngroups; g++) {
          size_t b0 = (size_t)g * s.group;
          size_t n = std::min((size_t)s.group, nb - b0);
          GroupTrav t(s, b0, n, offset);
          std::vector<char> all(n, 1);
          t.recurse(s.root, all);
          pp += t.pp;
          pc += t.pc;
          op += t.op;
        }
      }
  if (s.periodic) {  // examples/Gravity.C:45-48: callPerLeafFn(LeafEwaldFn)
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(s.threads)
#endif
    for (long b = 0; b < (long)nb; b++) LeafEwaldFn(*s.leaves[b], (Partition<CentroidData>*)nullptr);
    ewaldProxy.local = nullptr;
  }
  s.n_pp = pp;
  s.n_pc = pc;
  s.n_open = op;
}

double now() {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

// DualTraverser (src/Traverser.h:485-610) with the reference's GravityVisitor
// on a single subtree (local root = root): a stack of (source, target) pairs
// from (root, root); cell() asks whether to open the target
// (GravityVisitor::cell, examples/GravityVisitor.h:226-229); with
// TargetMustBeLeaf an internal target is handled by runInvertedTraversal.
struct DualTrav {
  RefSim& s;
  GravityVisitor v;
  unsigned long long pp = 0, pc = 0;
  explicit DualTrav(RefSim& sim) : s(sim), v(Vector3D<Real>(0, 0, 0), sim.theta) {}
  void inverted(RNode* source, RNode* target) {  // runInvertedTraversal
    std::vector<RNode*> st{target};
    while (!st.empty()) {
      RNode* node = st.back();
      st.pop_back();
      if (node->isLeaf()) {
        if (node->type == RNode::Type::Leaf) {
          v.leaf(*source, *node);  // an internal source carries no particles (n_particles = -1)
          if (source->n_particles > 0) pp += (unsigned long long)source->n_particles * node->n_particles;
        }
      } else if (v.open(*source, *node)) {
        for (int j = 0; j < node->n_children; j++) st.push_back(node->getChild(j));
      } else {
        v.node(*source, *node);
        pc += (unsigned long long)node->n_particles;
      }
    }
  }
  void run() {
    std::vector<std::pair<RNode*, RNode*>> st{{s.root, s.root}};
    while (!st.empty()) {
      RNode* node = st.back().first;
      RNode* pay = st.back().second;
      st.pop_back();
      if (pay->type == RNode::Type::EmptyLeaf) continue;
      if (node->type == RNode::Type::Leaf) {
        if (pay->isLeaf()) {
          v.leaf(*node, *pay);
          pp += (unsigned long long)node->n_particles * pay->n_particles;
        } else {
          inverted(node, pay);
        }
      } else if (node->type == RNode::Type::Internal) {
        if (pay->isLeaf()) {
          if (v.open(*node, *pay)) {
            for (int i = 0; i < node->n_children; i++) st.push_back({node->getChild(i), pay});
          } else {
            v.node(*node, *pay);
            pc += (unsigned long long)pay->n_particles;
          }
        } else if (!v.cell(*node, *pay)) {
          inverted(node, pay);  // TargetMustBeLeaf
        } else {
          for (int i = 0; i < node->n_children; i++) {
            if (pay->depth <= node->depth) {  // ForceEvenDepth
              for (int j = 0; j < pay->n_children; j++) st.push_back({node->getChild(i), pay->getChild(j)});
            } else {
              st.push_back({node->getChild(i), pay});
            }
          }
        }
      }
    }
  }
};

// One bucket's up-and-down walk (src/Traverser.h:363-482): its own leaf
// first, then, climbing to each ancestor, the ancestor's other children in
// child order, each subtree depth first with the visitor's open().
template <typename Visitor>
void upnd_bucket(Visitor& v, RNode* bucket) {
  auto down = [&](RNode* start) {
    std::vector<RNode*> st{start};
    while (!st.empty()) {
      RNode* node = st.back();
      st.pop_back();
      if (node->type == RNode::Type::Leaf) {
        v.leaf(*node, *bucket);
      } else if (node->type == RNode::Type::Internal) {
        if (v.open(*node, *bucket)) {
          for (int i = 0; i < node->n_children; i++) st.push_back(node->getChild(i));
        } else {
          v.node(*node, *bucket);
        }
      }
    }
  };
  down(bucket);
  RNode* top = bucket;
  while (top->parent) {
    RNode* par = top->parent;
    for (int j = 0; j < par->n_children; j++)
      if (par->getChild(j) != top) down(par->getChild(j));
    top = par;
  }
}

// examples/SPH.C:77-86 (startUpAndDown<DensityVisitor>) and DensityFn
// (SPH.C:11-37): k = 32 nearest neighbours (the particle itself included),
// then the M4-kernel density.  Outputs in caller order; nbr / nd2 hold each
// particle's neighbours sorted by (distance^2, caller index).
void sph_density(RefSim& s, double* density, double* ballsq, int* nbr, double* nd2, int kmax) {
  buildTree(s);
  const size_t nb = s.leaves.size();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(s.threads)
#endif
  for (long b = 0; b < (long)nb; b++) {
    DensityVisitor v;
    upnd_bucket(v, s.leaves[b]);
  }
  for (size_t b = 0; b < nb; b++) {
    auto& leaf = *s.leaves[b];
    for (int pi = 0; pi < leaf.n_particles; pi++) {
      const Particle& part = leaf.particles()[pi];
      auto& Q = leaf.data.pps[pi].neighbors;
      auto rsq = Q[0].fKey, fBall = std::sqrt(rsq);
      Real dens = 0.;
      auto ih2 = 4.0 / rsq;
      for (int i = 0; i < (int)Q.size(); i++) {
        auto& fDist2 = Q[i].fKey;
        auto r2 = fDist2 * ih2;
        auto rs = paratreet::kernelM4(r2);
        dens += rs * Q[i].pPtr->mass;
      }
      Real r_cubed = rsq * fBall;
      dens /= (0.125 * M_PI * r_cubed);
      density[part.order] = dens;
      ballsq[part.order] = rsq;
      auto copy_part = part;  // SPH.C:30-34
      copy_part.density = dens;
      leaf.changeParticle(pi, copy_part);
      leaf.data.pps[pi].sphBallSq = rsq;
      leaf.data.max_rad = std::max(leaf.data.max_rad, fBall);
      std::vector<std::pair<double, int>> q;
      for (auto& e : Q) q.push_back({e.fKey, e.pPtr->order});
      std::sort(q.begin(), q.end());
      for (int i = 0; i < kmax; i++) {
        nbr[(size_t)part.order * kmax + i] = i < (int)q.size() ? q[i].second : -1;
        nd2[(size_t)part.order * kmax + i] = i < (int)q.size() ? q[i].first : -1.0;
      }
      Q.clear();
    }
  }
}

// The pressure half of examples/SPH.C:traversalFn (:87-101): startDown with the
// reference's PressureVisitor (its gather of every neighbour within the ball),
// ForceFn (SPH.C:39-64: the divv corrector, then the reference's doSPHCalc per
// neighbour, examples/SPHUtils.h:64-133), and the opposing effects applied
// afterwards.  Needs sph_density first.  u: internal energy (caller order),
// used as u_predicted; velocity_predicted = velocity.  Outputs in caller order.
void sph_pressure_pass(RefSim& s);

void sph_pressure(RefSim& s, const double* u, double* ax, double* ay, double* az, double* pdv) {
  for (auto& p : s.particles) {
    p.u = p.u_predicted = u[p.order];
    p.velocity_predicted = p.velocity;
  }
  sph_pressure_pass(s);
  for (auto& p : s.particles) {
    ax[p.order] = p.acceleration.x;
    ay[p.order] = p.acceleration.y;
    az[p.order] = p.acceleration.z;
    pdv[p.order] = p.pressure_dVolume;
  }
}

// The pressure pass on the particles' own u_predicted and velocity_predicted:
// accelerations and PdV work start at zero and end with the opposing effects
// added (ThreadStateHolder::applyAccumulatedOpposingEffects).
void sph_pressure_pass(RefSim& s) {
  const size_t n = s.particles.size(), nb = s.leaves.size();
  for (auto& p : s.particles) {
    p.acceleration = Vector3D<Real>(0.0);
    p.pressure_dVolume = 0.0;
  }
  for (size_t b = 0; b < nb; b++) {  // transposed down traversal, pre-order per bucket
    PressureVisitor v;
    RNode* bucket = s.leaves[b];
    std::vector<RNode*> st{s.root};
    while (!st.empty()) {
      RNode* node = st.back();
      st.pop_back();
      if (node->type == RNode::Type::Leaf) {
        v.leaf(*node, *bucket);
      } else if (node->type == RNode::Type::Internal) {
        if (v.open(*node, *bucket)) {
          for (int i = node->n_children - 1; i >= 0; i--) st.push_back(node->getChild(i));
        } else {
          v.node(*node, *bucket);
        }
      }
    }
  }
  ThreadStateHolder tls;
  tls.acc.assign(n, Vector3D<Real>(0.0));
  tls.work.assign(n, 0.0);
  for (size_t b = 0; b < nb; b++) {  // ForceFn
    auto& leaf = *s.leaves[b];
    for (int pi = 0; pi < leaf.n_particles; pi++) {
      auto& part = leaf.particles()[pi];
      auto& Q = leaf.data.pps[pi].neighbors;
      auto rsq = leaf.data.pps[pi].sphBallSq, fBall = std::sqrt(rsq);
      auto ih2 = 4.0 / rsq;
      double divvi = 0, divvj = 0;
      for (int i = 0; i < (int)Q.size(); i++) {
        auto& fDist2 = Q[i].fKey;
        auto r2 = fDist2 * ih2;
        Real rs1 = paratreet::dkernelM4(r2);
        auto& q = *(Q[i].pPtr);
        rs1 *= fDist2 * q.mass;
        divvi += rs1;
        divvj += rs1 / q.density;
      }
      divvi /= part.density;
      auto corr = (divvj != 0.0 ? divvi / divvj : 1.0);
      for (int i = 0; i < (int)Q.size(); i++) paratreet::doSPHCalc(leaf, pi, fBall, &tls, *Q[i].pPtr, corr);
      Q.clear();
    }
  }
  for (auto& p : s.particles) {  // applyAccumulatedOpposingEffects
    p.acceleration.x = p.acceleration.x + tls.acc[p.order].x;
    p.acceleration.y = p.acceleration.y + tls.acc[p.order].y;
    p.acceleration.z = p.acceleration.z + tls.acc[p.order].z;
    p.pressure_dVolume = p.pressure_dVolume + tls.work[p.order];
  }
}

// nsteps iterations of the SPH example's Driver::run (src/Driver.h:183-251
// with examples/SPH.C:74-111): tree build and density pass, the pressure pass
// on the particles' u_predicted / velocity_predicted, then the reference's
// Particle::kick and Particle::perturb (src/Particle.C:7-21) with dt =
// max_timestep, the universe remade from the drifted positions and the keys
// reassigned.  SPH state in and out in caller order.
void sph_step(RefSim& s, int nsteps, double* u, double* u_pred, double* vpx, double* vpy, double* vpz) {
  const size_t n = s.particles.size();
  for (auto& p : s.particles) {
    p.u = u[p.order];
    p.u_predicted = u_pred[p.order];
    p.velocity_predicted = Vector3D<Real>(vpx[p.order], vpy[p.order], vpz[p.order]);
  }
  std::vector<double> d(n), b(n), nd2(n * 32);
  std::vector<int> nbr(n * 32);
  for (int it = 0; it < nsteps; it++) {
    sph_density(s, d.data(), b.data(), nbr.data(), nd2.data(), 32);
    sph_pressure_pass(s);
    const Real dt = s.dt_max;
    s.last_dt = dt;
    for (auto& p : s.particles) p.kick(dt);
    OrientedBox<Real> box;
    for (auto& p : s.particles) {
      p.perturb(dt);
      box.grow(p.position);
    }
    remakeUniverse(s, box);
    assignKeys(s);
  }
  for (auto& p : s.particles) {
    u[p.order] = p.u;
    u_pred[p.order] = p.u_predicted;
    vpx[p.order] = p.velocity_predicted.x;
    vpy[p.order] = p.velocity_predicted.y;
    vpz[p.order] = p.velocity_predicted.z;
  }
}

void forces(RefSim& s) {
  double t0 = now();
  buildTree(s);
  double t1 = now();
  for (auto& p : s.particles) {
    p.acceleration = Vector3D<Real>(0.0);
    p.potential = 0.0;
  }
  traverse(s);
  double t2 = now();
  s.t_build = t1 - t0;
  s.t_traverse = t2 - t1;
  size_t n = s.particles.size();
  s.acc.assign(3 * n, 0.0);
  s.pot.assign(n, 0.0);
  s.keys.assign(n, 0);
  for (auto& p : s.particles) {
    s.acc[3 * p.order + 0] = p.acceleration.x;
    s.acc[3 * p.order + 1] = p.acceleration.y;
    s.acc[3 * p.order + 2] = p.acceleration.z;
    s.pot[p.order] = p.potential;
    s.keys[p.order] = p.key;
  }
}

// examples/Gravity.C:63-67 with max velocity from src/Subtree.h:164-170.
double timestep(const RefSim& s) {
  Real vmax2 = 0.0;
  for (auto& p : s.particles) {
    if (p.velocity.lengthSquared() > vmax2) vmax2 = p.velocity.lengthSquared();
  }
  Real vmax = std::sqrt(vmax2);
  Real len = s.universe.greater_corner.x - s.universe.lesser_corner.x;
  Real t = len / vmax / std::cbrt((Real)s.particles.size());
  return std::min(t, (Real)s.dt_max);
}


// Bounded CPU sample of one force pass: the full tree build, then bucket
// groups in a fixed pseudo-random order on all threads until budget_s of
// traversal time is spent.  frac = share of the particles whose buckets were
// traversed.
void forces_sample(RefSim& s, double budget_s, double* t_build, double* t_trav, double* frac) {
  double t0 = now();
  buildTree(s);
  double t1 = now();
  for (auto& p : s.particles) {
    p.acceleration = Vector3D<Real>(0.0);
    p.potential = 0.0;
  }
  s.record_lists = 0;
  size_t nb = s.leaves.size();
  size_t ngroups = (nb + s.group - 1) / s.group;
  std::vector<size_t> order(ngroups);
  for (size_t g = 0; g < ngroups; g++) order[g] = g;
  uint64_t st = 0x9E3779B97F4A7C15ull;
  for (size_t g = ngroups; g > 1; g--) {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    std::swap(order[g - 1], order[st % g]);
  }
  std::atomic<size_t> next(0);
  std::atomic<long> done_particles(0);
  double tstart = now();
#ifdef _OPENMP
#pragma omp parallel num_threads(s.threads)
#endif
  {
    while (true) {
      if (now() - tstart > budget_s) break;
      size_t k = next.fetch_add(1);
      if (k >= ngroups) break;
      size_t g = order[k];
      size_t b0 = g * s.group;
      size_t n = std::min((size_t)s.group, nb - b0);
      GroupTrav t(s, b0, n);
      std::vector<char> all(n, 1);
      t.recurse(s.root, all);
      long cnt = 0;
      for (size_t b = 0; b < n; b++) cnt += s.leaves[b0 + b]->n_particles;
      done_particles += cnt;
    }
  }
  double t2 = now();
  *t_build = t1 - t0;
  *t_trav = t2 - tstart;
  *frac = (double)done_particles.load() / (double)std::max<size_t>(1, s.particles.size());
}

}  // namespace

extern "C" {

int ptref_forces_sample(void* h, double budget_s, double* t_build, double* t_trav, double* frac) {
  forces_sample(*(RefSim*)h, budget_s, t_build, t_trav, frac);
  return 0;
}


void* ptref_create(int n, const double* x, const double* y, const double* z, const double* vx,
                   const double* vy, const double* vz, const double* m, const double* soft, int bucket,
                   double theta, double dt_max, int group, int threads) {
  RefSim* s = new RefSim();
  s->bucket = bucket;
  s->theta = theta;
  s->dt_max = dt_max;
  s->group = group > 0 ? group : 64;
  s->threads = threads > 0 ? threads : 1;
  s->particles.resize(n);
  OrientedBox<Real> box;
  for (int i = 0; i < n; i++) {
    Particle& p = s->particles[i];
    p.order = i;
    p.mass = m[i];
    p.soft = soft[i];
    p.position = Vector3D<Real>(x[i], y[i], z[i]);
    p.velocity = Vector3D<Real>(vx[i], vy[i], vz[i]);
    p.velocity_predicted = p.velocity;
    p.potential = 0.0;
    p.u = 0.0;
    p.u_predicted = 0.0;
    p.type = Particle::Type::eDark;
    box.grow(p.position);
  }
  remakeUniverse(*s, box);
  assignKeys(*s);
  return s;
}

void ptref_destroy(void* h) { delete (RefSim*)h; }

void ptref_set_record_lists(void* h, int on) { ((RefSim*)h)->record_lists = on; }

/* nsteps == 0: one force evaluation.  Otherwise nsteps iterations of
 * src/Driver.h:183-251; outputs describe the LAST force evaluation, and the
 * particle state is the state after the last drift. */
int ptref_run(void* hp, int nsteps) {
  RefSim& s = *(RefSim*)hp;
  if (nsteps <= 0) {
    forces(s);
    return 0;
  }
  for (int it = 0; it < nsteps; it++) {
    forces(s);
    double dt = timestep(s);
    s.last_dt = dt;
    for (auto& p : s.particles) p.kick(dt);
    OrientedBox<Real> box;
    for (auto& p : s.particles) {
      p.perturb(dt);
      box.grow(p.position);
    }
    remakeUniverse(s, box);
    assignKeys(s);
  }
  return 0;
}

/* Subtree::startDual<GravityVisitor> on one subtree: accelerations (caller
 * order) and the P2P pairs / P2C evaluations it made. */
int ptref_dual(void* h, double* ax, double* ay, double* az, unsigned long long* pp_pc) {
  RefSim& s = *(RefSim*)h;
  buildTree(s);
  for (auto& p : s.particles) {
    p.acceleration = Vector3D<Real>(0.0);
    p.potential = 0.0;
  }
  DualTrav t(s);
  t.run();
  for (auto& p : s.particles) {
    ax[p.order] = p.acceleration.x;
    ay[p.order] = p.acceleration.y;
    az[p.order] = p.acceleration.z;
  }
  pp_pc[0] = t.pp;
  pp_pc[1] = t.pc;
  return 0;
}

/* 1: Partition::startBasicDown (breadth first per bucket), 0: startDown. */
void ptref_set_traversal(void* h, int basic_down) { ((RefSim*)h)->basic_down = basic_down; }

/* nsteps iterations of the SPH example; SPH state in/out in caller order. */
int ptref_sph_step(void* h, int nsteps, double* u, double* u_pred, double* vpx, double* vpy, double* vpz) {
  sph_step(*(RefSim*)h, nsteps, u, u_pred, vpx, vpy, vpz);
  return 0;
}

/* SPH pressure pass after ptref_sph_density (same particles). */
int ptref_sph_pressure(void* h, const double* u, double* ax, double* ay, double* az, double* pdv) {
  sph_pressure(*(RefSim*)h, u, ax, ay, az, pdv);
  return 0;
}

/* SPH density of the reference's SPH example (k = 32 neighbours). */
int ptref_sph_density(void* h, double* density, double* ballsq, int* nbr, double* nd2) {
  sph_density(*(RefSim*)h, density, ballsq, nbr, nd2, 32);
  return 0;
}

/* Periodic cube of side L with n replica shells walked by the tree and the
 * reference's Ewald correction (fEwCut 2.6, |h| <= 2.8) for the rest. */
void ptref_set_periodic(void* h, int periodic, double L, int n_replicas) {
  RefSim* s = (RefSim*)h;
  s->periodic = periodic;
  s->period = L;
  s->n_replicas = n_replicas;
}

void ptref_get_acc(void* h, double* ax, double* ay, double* az, double* pot) {
  RefSim& s = *(RefSim*)h;
  size_t n = s.particles.size();
  for (size_t i = 0; i < n; i++) {
    ax[i] = s.acc[3 * i];
    ay[i] = s.acc[3 * i + 1];
    az[i] = s.acc[3 * i + 2];
    pot[i] = s.pot[i];
  }
}

void ptref_get_keys(void* h, uint64_t* keys) {
  RefSim& s = *(RefSim*)h;
  std::memcpy(keys, s.keys.data(), s.keys.size() * sizeof(uint64_t));
}

void ptref_get_state(void* h, double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  RefSim& s = *(RefSim*)h;
  for (auto& p : s.particles) {
    x[p.order] = p.position.x;
    y[p.order] = p.position.y;
    z[p.order] = p.position.z;
    vx[p.order] = p.velocity.x;
    vy[p.order] = p.velocity.y;
    vz[p.order] = p.velocity.z;
  }
}

void ptref_get_universe(void* h, double* lo3, double* hi3) {
  RefSim& s = *(RefSim*)h;
  lo3[0] = s.universe.lesser_corner.x;
  lo3[1] = s.universe.lesser_corner.y;
  lo3[2] = s.universe.lesser_corner.z;
  hi3[0] = s.universe.greater_corner.x;
  hi3[1] = s.universe.greater_corner.y;
  hi3[2] = s.universe.greater_corner.z;
}

void ptref_get_counters(void* h, unsigned long long* out4, double* times2, double* last_dt) {
  RefSim& s = *(RefSim*)h;
  out4[0] = s.n_pp;
  out4[1] = s.n_pc;
  out4[2] = s.n_open;
  out4[3] = s.leaves.size();
  times2[0] = s.t_build;
  times2[1] = s.t_traverse;
  *last_dt = s.last_dt;
}

long ptref_num_nodes(void* h) { return (long)((RefSim*)h)->pool.size(); }

/* Node dump of the last build, in allocation (pre-order) order.
 * ints:    [type, depth, count(n_particles or data.count), n_children]
 * dbls:    [mass, cmx, cmy, cmz, soft, radius, xx, xy, xz, yy, yz, zz,
 *           lox, loy, loz, hix, hiy, hiz]  (18 per node) */
void ptref_get_nodes(void* h, uint64_t* keys, int* ints4, double* dbls18) {
  RefSim& s = *(RefSim*)h;
  size_t i = 0;
  for (auto& nd : s.pool) {
    keys[i] = nd.key;
    ints4[4 * i + 0] = (int)nd.type;
    ints4[4 * i + 1] = nd.depth;
    ints4[4 * i + 2] = nd.data.count;
    ints4[4 * i + 3] = nd.n_children;
    const auto& mm = nd.data.multipoles;
    double* d = dbls18 + 18 * i;
    d[0] = mm.totalMass;
    d[1] = mm.cm.x;
    d[2] = mm.cm.y;
    d[3] = mm.cm.z;
    d[4] = mm.soft;
    d[5] = mm.radius;
    d[6] = mm.xx;
    d[7] = mm.xy;
    d[8] = mm.xz;
    d[9] = mm.yy;
    d[10] = mm.yz;
    d[11] = mm.zz;
    d[12] = nd.data.box.lesser_corner.x;
    d[13] = nd.data.box.lesser_corner.y;
    d[14] = nd.data.box.lesser_corner.z;
    d[15] = nd.data.box.greater_corner.x;
    d[16] = nd.data.box.greater_corner.y;
    d[17] = nd.data.box.greater_corner.z;
    i++;
  }
}

long ptref_num_buckets(void* h) { return (long)((RefSim*)h)->leaves.size(); }

void ptref_get_bucket_keys(void* h, uint64_t* keys) {
  RefSim& s = *(RefSim*)h;
  for (size_t i = 0; i < s.leaves.size(); i++) keys[i] = s.leaves[i]->key;
}

/* Interaction lists (CSR over buckets in DFS order): offsets has
 * nbuckets+1 entries; entries hold node keys, kinds 0 = P2P leaf, 1 = P2C. */
long ptref_list_total(void* h) {
  RefSim& s = *(RefSim*)h;
  long t = 0;
  for (auto& l : s.lists) t += (long)l.size();
  return t;
}

void ptref_get_lists(void* h, long* offsets, uint64_t* keys, int* kinds) {
  RefSim& s = *(RefSim*)h;
  long o = 0;
  for (size_t b = 0; b < s.lists.size(); b++) {
    offsets[b] = o;
    for (auto& e : s.lists[b]) {
      keys[o] = e.key;
      kinds[o] = e.kind;
      o++;
    }
  }
  offsets[s.lists.size()] = o;
}

}  // extern "C"
