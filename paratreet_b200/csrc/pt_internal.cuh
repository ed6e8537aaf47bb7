// pt_internal.cuh -- device data layout and kernel entry points shared by the
// CUDA translation units of the B200 gravity path.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pt {

// Host-side count of this library's kernel launches (process-wide); every
// launch site calls note_launch() right before it launches.
void note_launch();
unsigned long long launches_so_far();


constexpr int kMaxDepth = 21;          // 63 key bits / 3 (src/common.h:29-31)
constexpr int kTypeLeaf = 1;           // Node<Data>::Type numbering, src/Node.h:82-95
constexpr int kTypeEmpty = 2;
constexpr int kTypeInternal = 6;
constexpr int kMinParticleNode = 6;    // examples/GravityVisitor.h:35

// Device status word bits (written by kernels, read by the host after a pass).
enum : unsigned {
  kErrNonFinite = 1u << 0,
  kErrStack = 1u << 1,
  kErrBucketTooBig = 1u << 2,
  kErrListOverflow = 1u << 3,
  kErrCapacity = 1u << 4,
  kErrAdjointSoftened = 1u << 5,
  kErrSort = 1u << 6,                 // radix sort look-back gave up waiting
  kErrPool = 1u << 7,                 // two-phase traversal: a list outgrew its region or pool (retried)
  kErrSphNonFinite = 1u << 8,         // SPH pressure: a term failed doSPHCalc's isfinite(acc)
};

// Particle state, structure of arrays, FP64, in key-sorted order after a build.
struct Particles {
  double *x, *y, *z, *vx, *vy, *vz, *m, *soft;
  int32_t* order;  // caller index of each sorted slot
  uint64_t* key;
  double *ax, *ay, *az, *pot, *potf;
};

// Per-node walk record: what one lane needs to classify one child.
struct __align__(16) WalkRec {
  double cm[3];         // MultipoleMoments::cm
  union {
    double orsq;        // Internal: radius^2 * gravity_factor (GravityVisitor::open, :164)
    double reach;       // Leaf: max |x_j - cm| over the leaf's particles
  };
  union {
    double soft;        // Internal: MultipoleMoments::soft (openSoftening, :124)
    double soft_max;    // Leaf: max particle softening in the leaf
  };
  int32_t first_child;  // first of 8 contiguous children, -1 for leaves
  int32_t type;         // kTypeLeaf / kTypeEmpty / kTypeInternal
  int32_t count;        // CentroidData::count
  int32_t pstart;       // first particle (sorted order)
  int32_t pcount;       // particles in the node's key range
  int32_t pad;
};

// Sibling blocks: the 8 children of an internal node are contiguous and start
// at 1 + 8k (the build allocates every level in groups of 8 after the root),
// so group k of nodes 1 + 8k .. 8 + 8k is stored as 3 rows of 8 x 16 bytes:
// row 0 (cm.x, cm.y), row 1 (cm.z, orsq | reach), row 2 (soft | soft_max,
// first_child and type | count << 3 as one 8-byte word).  Eight lanes that
// classify the children of one node read each row as one 128-byte line
// instead of eight 64-byte records.  Node 0 (the root) has no block.
__host__ __device__ __forceinline__ int64_t walk_sib_index(int64_t node, int row) {
  return ((node - 1) >> 3) * 24 + row * 8 + ((node - 1) & 7);
}
__host__ __device__ __forceinline__ int64_t walk_sib_size(int64_t nodes) { return ((nodes + 7) >> 3) * 24 + 24; }
static_assert(sizeof(WalkRec) == 64, "WalkRec is one 64-byte record");

// Per-node P2C record (FP64): mass, soft and the 6 second moments.
struct __align__(16) QuadRec {
  double mass, soft, xx, xy, xz, yy, yz, zz;
};
static_assert(sizeof(QuadRec) == 64, "QuadRec is one 64-byte record");

// Per-node P2C record for the mixed form (FP32): the same fields.
struct __align__(16) QuadRecF {
  float mass, soft, xx, xy, xz, yy, yz, zz;
};

// Full FP64 node moments (18 doubles), the layout pt_get_tree reports.
struct Mom {
  double mass, cm[3], soft, radius;
  double xx, xy, xz, yy, yz, zz;
  double lo[3], hi[3];
  double reach, soft_max;  // leaves only: max |x_j - cm|, max particle softening
};

// Node arrays (breadth-first order: level by level, children of one parent
// contiguous).
struct Nodes {
  uint64_t* key;
  int32_t* type;
  int32_t* depth;
  int32_t* pstart;
  int32_t* pcount;
  int32_t* parent;
  int32_t* first_child;
  int32_t* count;       // CentroidData::count
  Mom* mom;
  WalkRec* walk;
  double2* walks;       // sibling-block copy of walk's classification fields (walk_sib_index)
  QuadRec* quad;
  QuadRecF* quadf;
  uint64_t* fifo;       // upward-pass FIFO position key (depth-of-chain << 40 | rank)
  int32_t* nleaf_sub;   // Leaf nodes in subtree
  int32_t* nempty_sub;  // EmptyLeaf nodes in subtree
  int32_t* leaf_base;   // DFS rank base of Leaf nodes in subtree
  int32_t* empty_base;  // DFS rank base of EmptyLeaf nodes in subtree
};

struct TravParams {
  Particles p;
  const WalkRec* walk;
  const double2* walks;   // sibling blocks of walk (list walk)
  const QuadRec* quad;
  const QuadRecF* quadf;
  const float4* srcf;     // mixed: per-particle (x,y,z) relative to its leaf's cm, mass
  const float* softf;     // mixed: per-particle softening (FP32)
  const int32_t* buckets; // bucket b -> node index (DFS order)
  int64_t b_begin, b_end;
  double ox, oy, oz;      // GravityVisitor offset (periodic replicas; 0 otherwise)
  int64_t nnodes;
  int mode;               // 0 evaluate, 1 count lists only, 2 evaluate + record lists
  int accumulate;         // add to the stored accelerations (replica walks after the first)
  unsigned long long* bucket_work;  // per bucket (DFS index): P2P pairs + P2C evaluations; may be null
  int bfs;                // FP64 walk in BasicDownTraverser order (breadth first) instead of pre-order
  int64_t* list_count;    // mode 1: entries per bucket
  const int64_t* list_off;// mode 2: CSR offsets
  int32_t* list_node;     // mode 2: node index per entry
  int8_t* list_kind;      // mode 2: 0 P2P, 1 P2C
  unsigned long long* counters;  // n_pp, n_pc, n_open
  unsigned int* work;     // dynamic bucket counter
  unsigned int* status;
  unsigned long long* smq;  // per-SM bucket batches (list kernels; null: one bucket per grab)
};

// Interaction lists of the two-phase mixed traversal (k_mixed2.cu): two pools
// of node indices (bit 31 = monopole for P2C, near for P2P), per-warp regions
// reserved from the cursors, and per bucket (index b - b_begin) the start and
// length of its contiguous list in each pool.
struct ListParams {
  int32_t* pc_pool;
  int32_t* pp_pool;
  unsigned long long* cursor;  // [0] P2C pool, [1] P2P pool
  unsigned long long cap_pc, cap_pp;
  unsigned region, thresh;     // region size; least space left before a bucket starts
  int64_t* pc_start;
  int32_t* pc_count;
  int64_t* pp_start;
  int32_t* pp_count;
  unsigned* max_len;           // longest list of the pass
};

// Root cell of the periodic cube for the Ewald correction (k_ewald.cu):
// CentroidData of the root (mass, cm, quadrupole about cm) and the sums' cuts.
struct EwaldRoot {
  double cm[3], mass;
  double xx, xy, xz, yy, yz, zz;
  double L, rcut;
  int n_replicas, n_h;
};

// Inputs and outputs of the adjoint force pass (k_adjoint.cu).
struct AdjParams {
  Particles p;  // sorted positions, masses, softening
  const WalkRec* walk;
  const QuadRec* quad;
  const Mom* mom;
  const int32_t* parent;
  const int32_t* buckets;
  int64_t nbuckets, nnodes;
  const int64_t* list_off;
  const int32_t* list_node;
  const int8_t* list_kind;
  const double *cax, *cay, *caz;  // cotangent, sorted order
  double *gx, *gy, *gz, *gm;      // particle adjoints, sorted order (zeroed)
  double* nadj;                   // 10 per node: cm x/y/z, M, Qxx, Qyy, Qzz, Qxy, Qxz, Qyz (zeroed)
  unsigned* work;
  unsigned* status;
};

}  // namespace pt
