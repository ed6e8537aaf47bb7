// k_build.cu -- K5 octree build from sorted keys, breadth-first.
//
// Restates Subtree::recursiveBuild (src/Subtree.h:314-349) level by level:
// every Internal node (more than `bucket` particles, src/Subtree.h:263-267)
// gets exactly 8 children with keys key<<3 | c; child c's particle range ends
// at the first sorted key >= removeLeadingZeros(child_key + 1)
// (OctTree::findChildsLastParticle, src/Modularization.C:60-65 with
// src/Utility.h:33-50, :91-93, :127-130), the last child takes the rest.
// Children of a node are stored contiguously; level L+1 follows level L.
//
// Then, also level-synchronously: Leaf / EmptyLeaf counts per subtree
// (bottom-up) and DFS rank bases (top-down), which give the bucket list in
// DFS order (Subtree::leaves, src/Subtree.h:268-273) and the position of every
// leaf in the upward pass's FIFO (src/Subtree.h:352-361).
#include "pt_internal.cuh"

namespace pt {

__device__ __forceinline__ int node_type_for(int64_t n, int bucket, int depth) {
  if (n == 0) return kTypeEmpty;
  if (n <= bucket || depth >= kMaxDepth) return kTypeLeaf;
  return kTypeInternal;
}

__global__ void init_root(Nodes nd, int64_t n, int bucket) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    nd.key[0] = 1ull;
    nd.type[0] = node_type_for(n, bucket, 0);
    nd.depth[0] = 0;
    nd.pstart[0] = 0;
    nd.pcount[0] = (int32_t)n;
    nd.parent[0] = -1;
    nd.first_child[0] = -1;
    nd.leaf_base[0] = 0;
    nd.empty_base[0] = 0;
  }
}

__global__ void __launch_bounds__(256) flag_internal(const int32_t* __restrict__ type, int64_t begin, int64_t count,
                                                     uint32_t* __restrict__ flags) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < count) flags[t] = (type[begin + t] == kTypeInternal) ? 1u : 0u;
}

__device__ __forceinline__ int first_ge(const uint64_t* __restrict__ keys, int lo, int hi, uint64_t v) {
  while (lo < hi) {
    int mid = lo + ((hi - lo) >> 1);
    if (keys[mid] >= v) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

__global__ void __launch_bounds__(256) build_children(Nodes nd, const uint64_t* __restrict__ keys, int64_t begin,
                                                      int64_t count, const uint32_t* __restrict__ rank,
                                                      int64_t next_begin, int bucket, int64_t cap,
                                                      unsigned* status) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  int64_t i = begin + t;
  if (nd.type[i] != kTypeInternal) return;
  int64_t c0 = next_begin + 8 * (int64_t)rank[t];
  if (c0 < next_begin || c0 + 8 > cap) {  // never expected: the host sized the level
    atomicOr(status, kErrCapacity);
    nd.type[i] = kTypeLeaf;
    return;
  }
  nd.first_child[i] = (int32_t)c0;
  int depth = nd.depth[i] + 1;
  uint64_t ck = nd.key[i] << 3;
  int start = nd.pstart[i];
  int finish = start + nd.pcount[i];
  int shift = 63 - 3 * depth;  // removeLeadingZeros for a key of this depth
  for (int c = 0; c < 8; c++) {
    int fge = (c < 7) ? first_ge(keys, start, finish, (ck + 1) << shift) : finish;
    int64_t j = c0 + c;
    int cn = fge - start;
    nd.key[j] = ck;
    nd.type[j] = node_type_for(cn, bucket, depth);
    nd.depth[j] = depth;
    nd.pstart[j] = start;
    nd.pcount[j] = cn;
    nd.parent[j] = (int32_t)i;
    nd.first_child[j] = -1;
    start = fge;
    ck++;
  }
}

__global__ void __launch_bounds__(256) count_subtree(Nodes nd, int64_t begin, int64_t count) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  int64_t i = begin + t;
  int ty = nd.type[i];
  int nl = 0, ne = 0;
  if (ty == kTypeLeaf) nl = 1;
  else if (ty == kTypeEmpty) ne = 1;
  else {
    int c0 = nd.first_child[i];
    for (int c = 0; c < 8; c++) { nl += nd.nleaf_sub[c0 + c]; ne += nd.nempty_sub[c0 + c]; }
  }
  nd.nleaf_sub[i] = nl;
  nd.nempty_sub[i] = ne;
}

__global__ void __launch_bounds__(256) base_topdown(Nodes nd, int64_t begin, int64_t count) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  int64_t i = begin + t;
  if (nd.type[i] != kTypeInternal) return;
  int lb = nd.leaf_base[i], eb = nd.empty_base[i];
  int c0 = nd.first_child[i];
  for (int c = 0; c < 8; c++) {
    nd.leaf_base[c0 + c] = lb;
    nd.empty_base[c0 + c] = eb;
    lb += nd.nleaf_sub[c0 + c];
    eb += nd.nempty_sub[c0 + c];
  }
}

// buckets[leaf DFS rank] = node; FIFO position of leaves (0 << 40 | rank) and
// empty leaves (0 << 40 | n_leaves + rank).
__global__ void __launch_bounds__(256) assign_buckets(Nodes nd, int64_t nnodes, int32_t* __restrict__ buckets,
                                                      int nleaves) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nnodes) return;
  int ty = nd.type[i];
  if (ty == kTypeLeaf) {
    buckets[nd.leaf_base[i]] = (int32_t)i;
    nd.fifo[i] = (uint64_t)nd.leaf_base[i];
  } else if (ty == kTypeEmpty) {
    nd.fifo[i] = (uint64_t)(nleaves + nd.empty_base[i]);
  }
}

static inline unsigned blocks_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

void launch_init_root(Nodes nd, int64_t n, int bucket, cudaStream_t st) {
  note_launch();
  init_root<<<1, 32, 0, st>>>(nd, n, bucket);
}

void launch_flag_internal(const int32_t* type, int64_t begin, int64_t count, uint32_t* flags, cudaStream_t st) {
  if (count > 0) { note_launch(); flag_internal<<<blocks_for(count), 256, 0, st>>>(type, begin, count, flags); }
}

void launch_build_children(Nodes nd, const uint64_t* keys, int64_t begin, int64_t count, const uint32_t* rank,
                           int64_t next_begin, int bucket, int64_t cap, unsigned* status, cudaStream_t st) {
  if (count > 0) {
    note_launch();
    build_children<<<blocks_for(count), 256, 0, st>>>(nd, keys, begin, count, rank, next_begin, bucket, cap, status);
  }
}

void launch_count_subtree(Nodes nd, int64_t begin, int64_t count, cudaStream_t st) {
  if (count > 0) { note_launch(); count_subtree<<<blocks_for(count), 256, 0, st>>>(nd, begin, count); }
}

void launch_base_topdown(Nodes nd, int64_t begin, int64_t count, cudaStream_t st) {
  if (count > 0) { note_launch(); base_topdown<<<blocks_for(count), 256, 0, st>>>(nd, begin, count); }
}

void launch_assign_buckets(Nodes nd, int64_t nnodes, int32_t* buckets, int nleaves, cudaStream_t st) {
  if (nnodes > 0) { note_launch(); assign_buckets<<<blocks_for(nnodes), 256, 0, st>>>(nd, nnodes, buckets, nleaves); }
}

}  // namespace pt
