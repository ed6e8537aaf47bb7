// pt_api.cu -- the C ABI (include/pt_gravity.h): handle, device buffers and the
// per-pass orchestration of the kernels.
//
// One force pass (pt_compute_forces) runs, on the handle's stream:
//   K1 bbox + universe -> K2 keys -> K3 radix sort -> K4 permute
//   -> K5 level-synchronous octree build (+ bucket DFS order)
//   -> K6 leaf moments + upward pass + traversal records
//   -> K7 traversal (FP64 or mixed), optionally with interaction lists.
// The host reads back one 4-byte count per tree level (to size the next
// level) and the status word at the end; everything else stays on the device.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pt_gravity.h"
#include "pt_launch.h"

using namespace pt;

struct pt_handle {
  pt_config cfg{};
  std::string err;
  int sms = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;

  int64_t n = 0, cap_n = 0;
  Particles p{};
  double* tmp_d = nullptr;
  int32_t* tmp_i = nullptr;
  uint64_t* key_alt = nullptr;
  uint32_t *idx = nullptr, *idx_alt = nullptr;
  unsigned char* sort_scratch = nullptr;  // onesweep histograms, tile counters, look-back words
  uint32_t* scan_scratch = nullptr;
  size_t scan_scratch_elems = 0;
  uint32_t* d_total = nullptr;
  double* bbox_partial = nullptr;
  int bbox_blocks = 0;
  double* d_uni = nullptr;  // 12 doubles
  unsigned* d_status = nullptr;
  unsigned long long* d_counters = nullptr;  // 3
  unsigned* d_work = nullptr;
  unsigned long long* d_vmax2 = nullptr;
  float4* srcf = nullptr;
  float* softf = nullptr;
  int64_t cap_srcf = 0;

  Nodes nd{};
  int64_t node_cap = 0, nnodes = 0;
  uint32_t* flags = nullptr;
  std::vector<int64_t> lev;
  int32_t* buckets = nullptr;
  unsigned long long* bucket_work = nullptr;  // interactions per bucket of the last pass
  int64_t nbuckets = 0, cap_buckets = 0;

  int64_t* list_count = nullptr;
  int64_t* list_off = nullptr;
  int32_t* list_node = nullptr;
  int8_t* list_kind = nullptr;
  int64_t list_total = 0, list_cap = 0, list_nb = 0;  // list_nb = recorded buckets + 1
  int64_t list_off_cap = 0;                              // entries of list_count / list_off
  bool lists_valid = false;
  bool tp_lists_valid = false;  // the two-phase pools hold the last pass's lists of every bucket

  double* dsum = nullptr;  // direct-sum scratch (caller-order copies + partials)
  int64_t dsum_cap = 0;

  // two-phase mixed traversal: list pools and per-bucket list descriptors
  bool two_phase = true;  // PT_MIXED_FUSED=1 selects the fused walk + evaluate kernel
  int32_t *pool_pc = nullptr, *pool_pp = nullptr;
  unsigned long long cap_pc = 0, cap_pp = 0;    // allocated entries of each pool
  unsigned long long want_pc = 0, want_pp = 0;  // entries the next pass should have
  int64_t *l_pc_start = nullptr, *l_pp_start = nullptr;
  int32_t *l_pc_count = nullptr, *l_pp_count = nullptr;
  int64_t l_nb_cap = 0;
  unsigned long long* d_lcur = nullptr;  // [0] P2C cursor, [1] P2P cursor, [2] longest list
  unsigned* d_work3 = nullptr;           // bucket queues of the list kernels (walk, P2C, P2P)
  unsigned long long* d_smq = nullptr;   // their per-SM batches, 256 words per kernel
  unsigned l_region = 32768;  // entries per warp region of the list pools

  double* sph = nullptr;  // SPH density pass: density, ball^2 (2n), neighbours (k n int32 + k n double)
  int64_t sph_cap = 0, sph_nbr_cap = 0;
  int32_t* sph_nbr = nullptr;
  double* sph_nd2 = nullptr;
  double* sph_list_d = nullptr;  // neighbour-search scratch: per-warp lists
  int32_t* sph_list_i = nullptr;
  int64_t sph_list_cap = 0;
  double* sph_state = nullptr;  // SPH step: u, u_pred, v_pred (caller order, 5 N), sorted v_pred (3 N)
  int64_t sph_state_cap = 0;

  double4* d_htab = nullptr;  // Ewald reciprocal table (h vector, hCfac)
  int htab_cap = 0;
  double* ewd = nullptr;  // Ewald direct-sum scratch
  int64_t ewd_cap = 0;

  cudaEvent_t ev[7]{};
  long long sort_spin_limit = 1LL << 21;  // pt_set_sort_spin_limit
  pt_counters last{};
  double last_dt = 0.0;
  bool have_forces = false;     // a force pass ran since the particles were set
  bool forces_current = false;  // ... and the positions have not moved since
  bool trav_range_partial = false;

  double* adj = nullptr;  // adjoint scratch: cotangent (3N) and gradients (4N), sorted + caller order,
                          // then pt_adjoint's caller-order input and output (7N)
  int64_t adj_cap = 0;
  double* nadj = nullptr;  // 10 adjoint values per node
  int64_t nadj_cap = 0;
};

namespace pt {
namespace {

// Scratch owned by one call (freed on every return path).
struct DevBuf {
  double* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
std::atomic<unsigned long long> g_launches{0};
}
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace pt

namespace {

int fail(pt_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CK(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return fail(h, (e_ == cudaErrorMemoryAllocation) ? PT_E_NOMEM : PT_E_CUDA,               \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                         \
  } while (0)

#define CKR(expr)              \
  do {                         \
    int r_ = (expr);           \
    if (r_ != PT_OK) return r_; \
  } while (0)

template <typename T>
int dalloc(pt_handle* h, T** ptr, size_t count) {
  if (*ptr) {
    cudaFree(*ptr);
    *ptr = nullptr;
  }
  if (count == 0) count = 1;
  CK(cudaMalloc((void**)ptr, count * sizeof(T)));
  return PT_OK;
}

template <typename T>
void dfree(T*& ptr) {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
}

int grid_for(const pt_handle* h, int64_t n) {
  int64_t g = (n + 255) / 256;
  int64_t cap = (int64_t)h->sms * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

int ensure_particles(pt_handle* h, int64_t n) {
  if (n <= h->cap_n && h->p.x) return PT_OK;
  int64_t c = std::max<int64_t>(n, 1);
  double** dbl[] = {&h->p.x, &h->p.y, &h->p.z, &h->p.vx, &h->p.vy, &h->p.vz, &h->p.m, &h->p.soft,
                    &h->p.ax, &h->p.ay, &h->p.az, &h->p.pot, &h->p.potf, &h->tmp_d};
  for (auto pp : dbl) CKR(dalloc(h, pp, c));
  CKR(dalloc(h, &h->p.order, c));
  CKR(dalloc(h, &h->tmp_i, c));
  CKR(dalloc(h, &h->p.key, c));
  CKR(dalloc(h, &h->key_alt, c));
  CKR(dalloc(h, &h->idx, c));
  CKR(dalloc(h, &h->idx_alt, c));
  CKR(dalloc(h, &h->sort_scratch, sort_scratch_bytes(c)));
  size_t ss = scan_scratch_bytes(8 * c + 64);
  h->scan_scratch_elems = ss / sizeof(uint32_t) + 1;
  CKR(dalloc(h, &h->scan_scratch, h->scan_scratch_elems));
  h->cap_n = c;
  return PT_OK;
}

int grow_nodes(pt_handle* h, int64_t need) {
  if (need <= h->node_cap) return PT_OK;
  int64_t nc = std::max<int64_t>(need + need / 2, 1024);
  Nodes o = h->nd;
  Nodes nn{};
  int64_t keep = h->nnodes;
  // build arrays are copied, the rest are (re)computed after the build
  CKR(dalloc(h, &nn.key, nc));
  CKR(dalloc(h, &nn.type, nc));
  CKR(dalloc(h, &nn.depth, nc));
  CKR(dalloc(h, &nn.pstart, nc));
  CKR(dalloc(h, &nn.pcount, nc));
  CKR(dalloc(h, &nn.parent, nc));
  CKR(dalloc(h, &nn.first_child, nc));
  CKR(dalloc(h, &nn.count, nc));
  CKR(dalloc(h, &nn.mom, nc));
  CKR(dalloc(h, &nn.walk, nc));
  CKR(dalloc(h, &nn.walks, walk_sib_size(nc)));
  CKR(dalloc(h, &nn.quad, nc));
  CKR(dalloc(h, &nn.quadf, nc));
  CKR(dalloc(h, &nn.fifo, nc));
  CKR(dalloc(h, &nn.nleaf_sub, nc));
  CKR(dalloc(h, &nn.nempty_sub, nc));
  CKR(dalloc(h, &nn.leaf_base, nc));
  CKR(dalloc(h, &nn.empty_base, nc));
  if (keep > 0 && o.key) {
    cudaStream_t st = h->stream;
    CK(cudaMemcpyAsync(nn.key, o.key, keep * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.type, o.type, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.depth, o.depth, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.pstart, o.pstart, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.pcount, o.pcount, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.parent, o.parent, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.first_child, o.first_child, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.leaf_base, o.leaf_base, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(nn.empty_base, o.empty_base, keep * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
  }
  dfree(o.key); dfree(o.type); dfree(o.depth); dfree(o.pstart); dfree(o.pcount); dfree(o.parent);
  dfree(o.first_child); dfree(o.count); dfree(o.mom); dfree(o.walk); dfree(o.walks); dfree(o.quad); dfree(o.quadf);
  dfree(o.fifo); dfree(o.nleaf_sub); dfree(o.nempty_sub); dfree(o.leaf_base); dfree(o.empty_base);
  h->nd = nn;
  // flags holds the current level's child ranks while the build is running:
  // the new buffer must start with the old contents.
  uint32_t* nf = nullptr;
  CK(cudaMalloc((void**)&nf, nc * sizeof(uint32_t)));
  if (h->flags && h->node_cap > 0) {
    CK(cudaMemcpyAsync(nf, h->flags, h->node_cap * sizeof(uint32_t), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  dfree(h->flags);
  h->flags = nf;
  h->node_cap = nc;
  return PT_OK;
}

int read_status(pt_handle* h) {
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (st) {
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream));
    std::string m = "device status:";
    if (st & kErrNonFinite) m += " non-finite particle position;";
    if (st & kErrStack) m += " traversal stack overflow;";
    if (st & kErrBucketTooBig) m += " bucket larger than 32;";
    if (st & kErrListOverflow) m += " interaction list overflow;";
    if (st & kErrCapacity) m += " capacity exceeded;";
    if (st & kErrAdjointSoftened) m += " adjoint met a softened quadrupole term (not differentiated);";
    if (st & kErrSort) m += " radix sort look-back timed out;";
    if (st & kErrPool) m += " interaction-list pools exhausted;";
    if (st & kErrSphNonFinite) m += " SPH pressure term not finite (a ball of zero radius: N = 1 or coincident particles);";
    return fail(h, (st & kErrNonFinite) ? PT_E_NONFINITE : PT_E_DEVICE, m);
  }
  return PT_OK;
}

// K1..K4: universe, keys, sort, permute.
int keys_and_sort(pt_handle* h) {
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  const int g = grid_for(h, n);
  launch_bbox(h->p.x, h->p.y, h->p.z, n, h->bbox_partial, h->bbox_blocks, h->d_uni, h->d_status, st);
  launch_keys(h->p.x, h->p.y, h->p.z, n, h->d_uni, h->p.key, h->idx, g, st);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[1], st));
  if (radix_sort_pairs(h->p.key, h->idx, h->key_alt, h->idx_alt, n, h->sort_scratch, h->d_status, h->sms,
                       h->sort_spin_limit, st))
    return fail(h, PT_E_CUDA, "radix sort: could not set the shared-memory attribute");
  // a look-back that gave up leaves indices that are not a permutation: stop
  // before the gather, so the particle arrays keep their last consistent state
  CKR(read_status(h));
  double** fields[] = {&h->p.x, &h->p.y, &h->p.z, &h->p.vx, &h->p.vy, &h->p.vz, &h->p.m, &h->p.soft};
  for (auto f : fields) {
    gather_f64(*f, h->tmp_d, h->idx, n, g, st);
    std::swap(*f, h->tmp_d);
  }
  gather_i32(h->p.order, h->tmp_i, h->idx, n, g, st);
  std::swap(h->p.order, h->tmp_i);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[2], st));
  return PT_OK;
}

// K5: octree build, levels, bucket order.
int build_tree(pt_handle* h) {
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  if (h->node_cap < 1024) {
    h->nnodes = 0;
    CKR(grow_nodes(h, std::max<int64_t>(1024, n / 2 + 1024)));
  }
  h->nnodes = 1;
  launch_init_root(h->nd, n, h->cfg.bucket, st);
  h->lev.assign(1, 0);
  int64_t begin = 0, count = 1;
  while (true) {
    launch_flag_internal(h->nd.type, begin, count, h->flags, st);
    scan_exclusive(h->flags, h->flags, count, h->scan_scratch, h->d_total, st);
    uint32_t ni = 0;
    CK(cudaMemcpyAsync(&ni, h->d_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h->lev.push_back(begin + count);
    if (ni == 0) break;
    int64_t next = begin + count;
    int64_t need = next + 8 * (int64_t)ni;
    if (need > h->node_cap) {
      h->nnodes = next;
      CKR(grow_nodes(h, need));
    }
    launch_build_children(h->nd, h->p.key, begin, count, h->flags, next, h->cfg.bucket, h->node_cap, h->d_status, st);
    begin = next;
    count = 8 * (int64_t)ni;
    h->nnodes = need;
  }
  const int L = (int)h->lev.size() - 1;
  for (int l = L - 1; l >= 0; l--) launch_count_subtree(h->nd, h->lev[l], h->lev[l + 1] - h->lev[l], st);
  for (int l = 0; l < L; l++) launch_base_topdown(h->nd, h->lev[l], h->lev[l + 1] - h->lev[l], st);
  int32_t nl = 0;
  CK(cudaMemcpyAsync(&nl, h->nd.nleaf_sub, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  h->nbuckets = nl;
  if (nl > h->cap_buckets) {
    // an eighth of headroom: the bucket count drifts from pass to pass as the
    // particles move, and a cudaFree on every new maximum would stall the device
    const int64_t cap = (int64_t)nl + nl / 8 + 64;
    CKR(dalloc(h, &h->buckets, cap));
    CKR(dalloc(h, &h->bucket_work, cap));
    h->cap_buckets = cap;
  }
  launch_assign_buckets(h->nd, h->nnodes, h->buckets, nl, st);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[3], st));
  return PT_OK;
}

// K6: moments, upward pass, traversal records.
int upward(pt_handle* h) {
  cudaStream_t st = h->stream;
  launch_leaf_moments(h->nd, h->nnodes, h->p, st);
  const int L = (int)h->lev.size() - 1;
  for (int l = L - 1; l >= 0; l--) launch_upward_level(h->nd, h->lev[l], h->lev[l + 1] - h->lev[l], st);
  const double gfac = (4.0 / 3.0) / (h->cfg.theta * h->cfg.theta);  // GravityVisitor.h:14,18
  const int mixed = h->cfg.precision == PT_MIXED;
  launch_finalize(h->nd, h->nnodes, gfac, mixed, st);
  if (mixed) {
    if (h->cap_srcf < h->cap_n) {
      CKR(dalloc(h, &h->srcf, h->cap_n));
      CKR(dalloc(h, &h->softf, h->cap_n));
      h->cap_srcf = h->cap_n;
    }
    launch_prep_sources(h->buckets, h->nbuckets, h->nd.walk, h->p, h->srcf, h->softf, st);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev[4], st));
  return PT_OK;
}

// The Ewald correction of a periodic pass (examples/Gravity.C:45-48 calls
// LeafEwaldFn on every leaf after the replica walks).  The host builds the
// reciprocal table from the root's moments as EwaldData::EwaldInit does
// (examples/Ewald.C:80-163, QEVAL at (hx, hy, hz) with the odd gamma terms
// zeroed: hCfac = -g2 Qmir - g0 M, hSfac = 0), then one thread per particle of
// the buckets [b0, b1) adds the real-space and reciprocal sums.
int ewald_correction_pass(pt_handle* h, int64_t b0, int64_t b1) {
  cudaStream_t st = h->stream;
  Mom root;
  CK(cudaMemcpyAsync(&root, h->nd.mom, sizeof(Mom), cudaMemcpyDeviceToHost, st));
  int32_t pb[2] = {0, 0};
  int32_t pe[2] = {0, 0};
  if (b1 > b0) {
    int32_t nb0 = 0, nb1 = 0;
    CK(cudaMemcpyAsync(&nb0, h->buckets + b0, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&nb1, h->buckets + (b1 - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpyAsync(pb, &h->nd.walk[nb0].pstart, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(pe, &h->nd.walk[nb1].pstart, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  const double L = h->cfg.period;
  const double hcut = h->cfg.ewald_hcut;
  const int hReps = (int)std::ceil(hcut);
  const double alpha = 2.0 / L;
  const double k4 = M_PI * M_PI / (alpha * alpha * L * L);
  std::vector<double4> tab;
  for (int hx = -hReps; hx <= hReps; ++hx)
    for (int hy = -hReps; hy <= hReps; ++hy)
      for (int hz = -hReps; hz <= hReps; ++hz) {
        const int h2 = hx * hx + hy * hy + hz * hz;
        if (h2 == 0) continue;
        if (h2 > hcut * hcut) continue;
        const double g0 = std::exp(-k4 * h2) / (M_PI * h2 * L);
        const double g1 = 2 * M_PI / L * g0;
        const double g2 = -2 * M_PI / L * g1;
        const double Qmirx = (1.0 / 1.0) * (root.xz * hz + root.xy * hy + root.xx * hx);
        const double Qmiry = (1.0 / 1.0) * (root.yz * hz + root.xy * hx + root.yy * hy);
        const double Qmirz = (1.0 / 1.0) * (root.yz * hy + root.xz * hx + root.zz * hz);
        const double Qmir = (1.0 / 2.0) * (Qmirx * hx + Qmiry * hy + Qmirz * hz);
        double mfacc = 0.0;
        mfacc -= g2 * Qmir;
        mfacc -= g0 * root.mass;
        tab.push_back(make_double4(2 * M_PI / L * hx, 2 * M_PI / L * hy, 2 * M_PI / L * hz, mfacc));
      }
  if ((int)tab.size() > h->htab_cap) {
    CKR(dalloc(h, &h->d_htab, tab.size()));
    h->htab_cap = (int)tab.size();
  }
  if (!tab.empty())
    CK(cudaMemcpyAsync(h->d_htab, tab.data(), tab.size() * sizeof(double4), cudaMemcpyHostToDevice, st));
  EwaldRoot R{};
  R.cm[0] = root.cm[0];
  R.cm[1] = root.cm[1];
  R.cm[2] = root.cm[2];
  R.mass = root.mass;
  R.xx = root.xx;
  R.xy = root.xy;
  R.xz = root.xz;
  R.yy = root.yy;
  R.yz = root.yz;
  R.zz = root.zz;
  R.L = L;
  R.rcut = h->cfg.ewald_rcut;
  R.n_replicas = h->cfg.n_replicas;
  R.n_h = (int)tab.size();
  const int64_t i0 = pb[0], i1 = (b1 > b0) ? (int64_t)pe[0] + pe[1] : i0;
  launch_ewald_correction(h->p, i0, i1, R, h->d_htab, st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));  // the host table must outlive the copy
  return PT_OK;
}

// Two-phase mixed evaluation: walk_lists writes every bucket's interaction
// list to the pools, then eval_p2c and eval_p2p evaluate them.  Pools are
// sized from the previous pass with a quarter of headroom (a bucket whose list
// outgrows its warp's region moves it to a new region inside the walk); only
// a pass whose lists fill a pool is repeated (counters restored) with pools
// twice as large, which happens at most on the first passes of a handle.
int run_two_phase(pt_handle* h, TravParams& P) {
  cudaStream_t st = h->stream;
  const int64_t nb = P.b_end - P.b_begin;
  if (nb <= 0) return PT_OK;
  if (nb > h->l_nb_cap) {
    const int64_t cap = nb + nb / 8 + 64;  // headroom, as for the bucket arrays
    CKR(dalloc(h, &h->l_pc_start, cap));
    CKR(dalloc(h, &h->l_pp_start, cap));
    CKR(dalloc(h, &h->l_pc_count, cap));
    CKR(dalloc(h, &h->l_pp_count, cap));
    h->l_nb_cap = cap;
  }
  if (!h->d_lcur) CKR(dalloc(h, &h->d_lcur, 3));
  if (!h->d_work3) CKR(dalloc(h, &h->d_work3, 3));
  if (!h->d_smq) CKR(dalloc(h, &h->d_smq, 3 * 256));
  const int wgrid = (int)std::max<int64_t>(1, std::min<int64_t>(walk_lists_grid(h->sms), (nb + 3) / 4));
  unsigned long long c0[3];
  CK(cudaMemcpyAsync(c0, h->d_counters, sizeof(c0), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  ListParams L{};
  for (int attempt = 0;; attempt++) {
    const unsigned region = h->l_region;
    const unsigned long long slack = (unsigned long long)wgrid * 4 * region;
    const unsigned long long need_pc =
        std::max<unsigned long long>(h->want_pc ? h->want_pc + slack : 0, 1024ull * nb + slack);
    const unsigned long long need_pp =
        std::max<unsigned long long>(h->want_pp ? h->want_pp + slack : 0, 256ull * nb + slack);
    if (need_pc > h->cap_pc || need_pp > h->cap_pp) {
      // a quarter of headroom, so that the pass-to-pass variation of the
      // reserved regions does not free and map the multi-GB pools again
      // (which costs more than a whole pass); without room for it, the bare need
      dfree(h->pool_pc);
      dfree(h->pool_pp);
      h->cap_pc = h->cap_pp = 0;
      unsigned long long alloc_pc = need_pc + need_pc / 4, alloc_pp = need_pp + need_pp / 4;
      if (cudaMalloc((void**)&h->pool_pc, alloc_pc * sizeof(int32_t)) != cudaSuccess ||
          cudaMalloc((void**)&h->pool_pp, alloc_pp * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        dfree(h->pool_pc);
        dfree(h->pool_pp);
        alloc_pc = need_pc;
        alloc_pp = need_pp;
      }
      if ((!h->pool_pc && cudaMalloc((void**)&h->pool_pc, need_pc * sizeof(int32_t)) != cudaSuccess) ||
          (!h->pool_pp && cudaMalloc((void**)&h->pool_pp, need_pp * sizeof(int32_t)) != cudaSuccess)) {
        // no room for the lists: this handle evaluates with the fused kernel from now on
        cudaGetLastError();
        dfree(h->pool_pc);
        dfree(h->pool_pp);
        h->two_phase = false;
        CK(cudaMemcpyAsync(h->d_counters, c0, sizeof(c0), cudaMemcpyHostToDevice, st));
        if (h->cfg.precision == PT_FP64_LISTS) launch_traverse_f64(P, h->nd.mom, h->sms * 16, st);
        else launch_traverse_mixed(P, h->nd.mom, h->sms * 16, st);
        CK(cudaGetLastError());
        return PT_OK;
      }
      h->cap_pc = alloc_pc;
      h->cap_pp = alloc_pp;
    }
    L.pc_pool = h->pool_pc;
    L.pp_pool = h->pool_pp;
    L.cursor = h->d_lcur;
    L.cap_pc = h->cap_pc;
    L.cap_pp = h->cap_pp;
    L.region = region;
    L.thresh = region / 8;
    L.pc_start = h->l_pc_start;
    L.pc_count = h->l_pc_count;
    L.pp_start = h->l_pp_start;
    L.pp_count = h->l_pp_count;
    L.max_len = reinterpret_cast<unsigned*>(h->d_lcur + 2);
    CK(cudaMemsetAsync(h->d_lcur, 0, 3 * sizeof(unsigned long long), st));
    CK(cudaMemsetAsync(h->d_work3, 0, 3 * sizeof(unsigned), st));
    if (h->d_smq) CK(cudaMemsetAsync(h->d_smq, 0, 3 * 256 * sizeof(unsigned long long), st));
    TravParams A = P;
    A.work = h->d_work3;
    A.smq = h->d_smq;
    launch_walk_lists(A, L, h->nd.mom, wgrid, st);
    CK(cudaGetLastError());
    unsigned status = 0;
    unsigned long long cur[3];
    CK(cudaMemcpyAsync(&status, h->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(cur, h->d_lcur, sizeof(cur), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the cursors count reserved regions (also refused ones): at most the pool size is used
    const unsigned long long used_pc = std::min(cur[0], h->cap_pc), used_pp = std::min(cur[1], h->cap_pp);
    if (!(status & kErrPool)) {
      // next pass: room for this pass's lists and a quarter more
      h->want_pc = std::max<unsigned long long>(h->want_pc, used_pc + used_pc / 4);
      h->want_pp = std::max<unsigned long long>(h->want_pp, used_pp + used_pp / 4);
      break;
    }
    if (attempt >= 6) return fail(h, PT_E_NOMEM, "interaction lists outgrow their pools");
    // repeat the walk with larger pools (the cursors under-count the need: warps
    // stop reserving once their pool is full)
    status &= ~kErrPool;
    CK(cudaMemcpyAsync(h->d_status, &status, sizeof(unsigned), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->d_counters, c0, sizeof(c0), cudaMemcpyHostToDevice, st));
    h->want_pc = std::max(2 * h->cap_pc, cur[0] + cur[0] / 2);
    h->want_pp = std::max(2 * h->cap_pp, cur[1] + cur[1] / 2);
  }
  TravParams E = P;
  E.work = h->d_work3 + 1;
  E.smq = h->d_smq ? h->d_smq + 256 : nullptr;
  if (h->cfg.precision == PT_FP64_LISTS) launch_eval_lists_f64(E, L, h->nd.mom, h->sms * 16, st, h->d_work3 + 2);
  else launch_eval_lists(E, L, h->nd.mom, h->sms * 16, st, h->d_work3 + 2);
  CK(cudaGetLastError());
  h->tp_lists_valid = (P.b_begin == 0 && P.b_end == h->nbuckets && !h->cfg.periodic);
  return PT_OK;
}

int run_traversal(pt_handle* h, TravParams& P, int grid) {
  const bool lists_form = h->cfg.precision == PT_MIXED || h->cfg.precision == PT_FP64_LISTS;
  if (lists_form && P.mode == 0 && h->two_phase) return run_two_phase(h, P);
  if (h->cfg.precision == PT_MIXED && P.mode != 1)
    launch_traverse_mixed(P, h->nd.mom, grid, h->stream);
  else launch_traverse_f64(P, h->nd.mom, grid, h->stream);
  CK(cudaGetLastError());
  return PT_OK;
}

// CSR lists (list_off / list_node / list_kind, kinds 0 P2P, 1 quadrupole,
// 2 monopole) of every bucket from the two-phase pools of the pass just
// made: per bucket its P2P leaves, then its P2C nodes, in the two-phase
// walk's order.
int lists_from_pools(pt_handle* h) {
  cudaStream_t st = h->stream;
  const int64_t nb = h->nbuckets;
  if (nb + 1 > h->list_off_cap) {
    CKR(dalloc(h, &h->list_count, nb + 1));
    CKR(dalloc(h, &h->list_off, nb + 1));
    h->list_off_cap = nb + 1;
  }
  std::vector<int32_t> cpc(nb), cpp(nb);
  std::vector<int64_t> off(nb + 1);
  CK(cudaMemcpyAsync(cpc.data(), h->l_pc_count, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(cpp.data(), h->l_pp_count, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  off[0] = 0;
  for (int64_t i = 0; i < nb; i++) off[i + 1] = off[i] + cpc[i] + cpp[i];
  h->list_total = off[nb];
  if (h->list_total > h->list_cap) {
    CKR(dalloc(h, &h->list_node, h->list_total));
    CKR(dalloc(h, &h->list_kind, h->list_total));
    h->list_cap = h->list_total;
  }
  CK(cudaMemcpyAsync(h->list_off, off.data(), (nb + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  launch_pools_to_csr(h->pool_pc, h->pool_pp, h->l_pc_start, h->l_pc_count, h->l_pp_start, h->l_pp_count, nb,
                      h->list_off, h->list_node, h->list_kind, st);
  CK(cudaGetLastError());
  h->list_nb = nb + 1;
  h->lists_valid = true;
  return PT_OK;
}

int traverse(pt_handle* h, int64_t b0, int64_t b1) {
  cudaStream_t st = h->stream;
  b0 = std::max<int64_t>(0, std::min(b0, h->nbuckets));
  b1 = std::max<int64_t>(b0, std::min(b1, h->nbuckets));
  h->trav_range_partial = !(b0 == 0 && b1 == h->nbuckets);
  if (h->trav_range_partial) {
    double* arrs[] = {h->p.ax, h->p.ay, h->p.az, h->p.pot, h->p.potf};
    for (auto a : arrs) CK(cudaMemsetAsync(a, 0, h->n * sizeof(double), st));
  }
  TravParams P{};
  P.p = h->p;
  P.walk = h->nd.walk;
  P.walks = h->nd.walks;
  P.quad = h->nd.quad;
  P.quadf = h->nd.quadf;
  P.srcf = h->srcf;
  P.softf = h->softf;
  P.buckets = h->buckets;
  P.b_begin = b0;
  P.b_end = b1;
  P.ox = P.oy = P.oz = 0.0;
  P.bucket_work = h->bucket_work;
  P.bfs = (h->cfg.traversal == PT_BASIC_DOWN) ? 1 : 0;
  if (h->nbuckets > 0) CK(cudaMemsetAsync(h->bucket_work, 0, h->nbuckets * sizeof(unsigned long long), st));
  P.nnodes = h->nnodes;
  P.counters = h->d_counters;
  P.work = h->d_work;
  P.status = h->d_status;
  const int grid = h->sms * 16;
  CK(cudaMemsetAsync(h->d_counters, 0, 3 * sizeof(unsigned long long), st));
  const int64_t nb = b1 - b0;
  h->lists_valid = false;
  h->tp_lists_valid = false;
  // The two-phase forms record a full pass's lists from their own pools
  // (lists_from_pools, after the pass); the FP64 form records them in the
  // reference's walk order with a counting and a recording walk.
  const bool two_phase_record = h->cfg.record_lists && nb > 0 && h->two_phase && !h->cfg.periodic &&
                                b0 == 0 && b1 == h->nbuckets &&
                                (h->cfg.precision == PT_MIXED || h->cfg.precision == PT_FP64_LISTS);
  if (h->cfg.record_lists && nb > 0 && !two_phase_record) {
    if (nb + 1 > h->list_off_cap) {
      CKR(dalloc(h, &h->list_count, nb + 1));
      CKR(dalloc(h, &h->list_off, nb + 1));
      h->list_off_cap = nb + 1;
    }
    h->list_nb = nb + 1;
    P.mode = 1;
    P.list_count = h->list_count;
    CK(cudaMemsetAsync(h->d_work, 0, sizeof(unsigned), st));
    CKR(run_traversal(h, P, grid));
    std::vector<int64_t> cnt(nb), off(nb + 1);
    CK(cudaMemcpyAsync(cnt.data(), h->list_count, nb * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    off[0] = 0;
    for (int64_t i = 0; i < nb; i++) off[i + 1] = off[i] + cnt[i];
    h->list_total = off[nb];
    if (h->list_total > h->list_cap) {
      CKR(dalloc(h, &h->list_node, h->list_total));
      CKR(dalloc(h, &h->list_kind, h->list_total));
      h->list_cap = h->list_total;
    }
    CK(cudaMemcpyAsync(h->list_off, off.data(), (nb + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(h->d_counters, 0, 3 * sizeof(unsigned long long), st));
    P.mode = 2;
    P.list_off = h->list_off;
    P.list_node = h->list_node;
    P.list_kind = h->list_kind;
    if (h->cfg.precision == PT_MIXED || h->cfg.precision == PT_FP64_LISTS) {
      // lists come from the FP64 walk (identical for every form); then the two-phase pass
      P.mode = 2;
      CK(cudaMemsetAsync(h->d_work, 0, sizeof(unsigned), st));
      launch_traverse_f64(P, h->nd.mom, grid, st);  // records lists (and FP64 forces)
      CK(cudaMemsetAsync(h->d_counters, 0, 3 * sizeof(unsigned long long), st));
      P.mode = 0;
    }
    h->lists_valid = true;
  } else {
    P.mode = 0;
  }
  CK(cudaEventRecord(h->ev[5], st));
  // examples/Gravity.C:32-46: one walk, or (2n+1)^3 replica walks with
  // GravityVisitor offsets (X, Y, Z) * L in that loop order; every walk after
  // the first continues each particle's sums
  const int nr = h->cfg.periodic ? h->cfg.n_replicas : 0;
  const double L = h->cfg.period;
  bool first = true;
  for (int X = -nr; X <= nr; X++)
    for (int Y = -nr; Y <= nr; Y++)
      for (int Z = -nr; Z <= nr; Z++) {
        P.ox = X * L;
        P.oy = Y * L;
        P.oz = Z * L;
        P.accumulate = first ? 0 : 1;
        first = false;
        CK(cudaMemsetAsync(h->d_work, 0, sizeof(unsigned), st));
        CKR(run_traversal(h, P, grid));
      }
  if (h->cfg.periodic) CKR(ewald_correction_pass(h, b0, b1));
  CK(cudaEventRecord(h->ev[6], st));
  if (two_phase_record && h->tp_lists_valid) CKR(lists_from_pools(h));
  return PT_OK;
}

int forces(pt_handle* h, int64_t b0, int64_t b1) {
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles: call pt_set_particles first");
  const unsigned long long launches0 = launches_so_far();
  cudaStream_t st = h->stream;
  CK(cudaEventRecord(h->ev[0], st));
  if (h->n == 0) {
    h->nnodes = 0;
    h->nbuckets = 0;
    h->have_forces = true;
    h->forces_current = true;
    return PT_OK;
  }
  CKR(keys_and_sort(h));
  CKR(build_tree(h));
  CKR(upward(h));
  CKR(traverse(h, b0, b1));
  CKR(read_status(h));
  unsigned long long c[3];
  CK(cudaMemcpyAsync(c, h->d_counters, sizeof(c), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  pt_counters& k = h->last;
  k.n_pp = c[0];
  k.n_pc = c[1];
  k.n_open = c[2];
  k.n_nodes = h->nnodes;
  k.n_buckets = h->nbuckets;
  k.depth = (int32_t)h->lev.size() - 2;
  k.launches = (int32_t)(launches_so_far() - launches0);
  CK(cudaEventElapsedTime(&k.ms_keys, h->ev[0], h->ev[1]));
  CK(cudaEventElapsedTime(&k.ms_sort, h->ev[1], h->ev[2]));
  CK(cudaEventElapsedTime(&k.ms_build, h->ev[2], h->ev[3]));
  CK(cudaEventElapsedTime(&k.ms_upward, h->ev[3], h->ev[4]));
  CK(cudaEventElapsedTime(&k.ms_traverse, h->ev[5], h->ev[6]));
  CK(cudaEventElapsedTime(&k.ms_total, h->ev[0], h->ev[6]));
  h->have_forces = true;
  h->forces_current = true;
  return PT_OK;
}

// examples/Gravity.C:63-67 with v_max from src/Subtree.h:164-170.
int timestep(pt_handle* h, double* dt) {
  cudaStream_t st = h->stream;
  CK(cudaMemsetAsync(h->d_vmax2, 0, sizeof(unsigned long long), st));
  launch_vmax2(h->p.vx, h->p.vy, h->p.vz, h->n, h->d_vmax2, grid_for(h, h->n), st);
  unsigned long long bits = 0;
  double uni[6];
  CK(cudaMemcpyAsync(&bits, h->d_vmax2, sizeof(bits), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(uni, h->d_uni, sizeof(uni), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  double v2;
  std::memcpy(&v2, &bits, sizeof(v2));
  double vmax = std::sqrt(v2);
  double len = uni[3] - uni[0];
  double t = len / vmax / std::cbrt((double)h->n);
  *dt = std::min(t, h->cfg.dt_max);
  return PT_OK;
}

int unpermute_f64(pt_handle* h, const double* dsrc, double* host_out) {
  if (!host_out) return PT_OK;
  launch_scatter_f64(dsrc, h->tmp_d, h->p.order, h->n, grid_for(h, h->n), h->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host_out, h->tmp_d, h->n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return PT_OK;
}

int set_particles_impl(pt_handle* h, int64_t n, const double* const src[8], cudaMemcpyKind kind) {
  if (n < 0 || n > (int64_t)INT32_MAX - 64) return fail(h, PT_E_ARG, "particle count out of range");
  for (int i = 0; i < 8 && n > 0; i++)
    if (!src[i]) return fail(h, PT_E_ARG, "null particle array");
  CKR(ensure_particles(h, n));
  h->n = n;
  double* dst[8] = {h->p.x, h->p.y, h->p.z, h->p.vx, h->p.vy, h->p.vz, h->p.m, h->p.soft};
  for (int i = 0; i < 8 && n > 0; i++)
    CK(cudaMemcpyAsync(dst[i], src[i], n * sizeof(double), kind, h->stream));
  launch_iota_i32(h->p.order, n, grid_for(h, n), h->stream);
  CK(cudaGetLastError());
  h->have_forces = false;
  h->forces_current = false;
  h->lists_valid = false;
  return PT_OK;
}

}  // namespace

extern "C" {

int pt_abi_version(void) { return PT_ABI_VERSION; }

int pt_config_default(pt_config* c) {
  if (!c) return PT_E_ARG;
  std::memset(c, 0, sizeof(*c));
  c->theta = 0.7;
  c->bucket = 16;
  c->precision = PT_FP64;
  c->integrator = PT_KKD;
  c->dt_max = 1e-5;
  c->device = 0;
  c->record_lists = 0;
  c->periodic = 0;
  c->n_replicas = 0;
  c->period = 1.0;
  c->ewald_rcut = 2.6;  // fEwCut, examples/Ewald.h:26
  c->ewald_hcut = 2.8;  // dEwhCut, examples/Ewald.C:86
  return PT_OK;
}

int pt_create(const pt_config* cfg, pt_handle** out) {
  if (!cfg || !out) return PT_E_ARG;
  *out = nullptr;
  if (!(cfg->theta > 0.0) || cfg->bucket < 1 || cfg->bucket > 32) return PT_E_ARG;
  if (cfg->precision != PT_FP64 && cfg->precision != PT_MIXED && cfg->precision != PT_FP64_LISTS) return PT_E_ARG;
  if (cfg->traversal != PT_TRANSPOSED_DOWN && cfg->traversal != PT_BASIC_DOWN) return PT_E_ARG;
  if (cfg->integrator != PT_KKD && cfg->integrator != PT_KDK) return PT_E_ARG;
  if (cfg->periodic && (!(cfg->period > 0.0) || cfg->n_replicas < 0 || cfg->n_replicas > 8 ||
                        !(cfg->ewald_rcut > 0.0) || cfg->ewald_rcut > 8.0 || !(cfg->ewald_hcut >= 0.0) ||
                        cfg->ewald_hcut > 16.0 || cfg->record_lists))
    return PT_E_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return PT_E_CUDA;
  if (cfg->device < 0 || cfg->device >= ndev) return PT_E_ARG;
  pt_handle* h = new pt_handle();
  h->cfg = *cfg;
  auto bail = [&](int code) {
    pt_destroy(h);
    return code;
  };
  if (cudaSetDevice(cfg->device) != cudaSuccess) return bail(PT_E_CUDA);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess) return bail(PT_E_CUDA);
  h->sms = prop.multiProcessorCount;
  if (const char* v = std::getenv("PT_MIXED_FUSED")) h->two_phase = std::atoi(v) == 0;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) return bail(PT_E_CUDA);
  h->stream = h->own_stream;
  for (auto& e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return bail(PT_E_CUDA);
  h->bbox_blocks = h->sms * 4;
  if (dalloc(h, &h->bbox_partial, 6 * (size_t)h->bbox_blocks) != PT_OK) return bail(PT_E_NOMEM);
  if (dalloc(h, &h->d_uni, 12) != PT_OK) return bail(PT_E_NOMEM);
  if (dalloc(h, &h->d_status, 1) != PT_OK) return bail(PT_E_NOMEM);
  if (dalloc(h, &h->d_counters, 3) != PT_OK) return bail(PT_E_NOMEM);
  if (dalloc(h, &h->d_work, 1) != PT_OK) return bail(PT_E_NOMEM);
  if (dalloc(h, &h->d_vmax2, 1) != PT_OK) return bail(PT_E_NOMEM);
  if (dalloc(h, &h->d_total, 4) != PT_OK) return bail(PT_E_NOMEM);
  if (cudaMemset(h->d_status, 0, sizeof(unsigned)) != cudaSuccess) return bail(PT_E_CUDA);
  *out = h;
  return PT_OK;
}

int pt_destroy(pt_handle* h) {
  if (!h) return PT_OK;
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  double** dbl[] = {&h->p.x, &h->p.y, &h->p.z, &h->p.vx, &h->p.vy, &h->p.vz, &h->p.m, &h->p.soft,
                    &h->p.ax, &h->p.ay, &h->p.az, &h->p.pot, &h->p.potf, &h->tmp_d};
  for (auto pp : dbl) dfree(*pp);
  dfree(h->p.order); dfree(h->tmp_i); dfree(h->p.key); dfree(h->key_alt); dfree(h->idx); dfree(h->idx_alt);
  dfree(h->sort_scratch); dfree(h->scan_scratch); dfree(h->d_total); dfree(h->bbox_partial); dfree(h->d_uni);
  dfree(h->d_status); dfree(h->d_counters); dfree(h->d_work); dfree(h->d_vmax2); dfree(h->srcf); dfree(h->softf);
  Nodes& o = h->nd;
  dfree(o.key); dfree(o.type); dfree(o.depth); dfree(o.pstart); dfree(o.pcount); dfree(o.parent);
  dfree(o.first_child); dfree(o.count); dfree(o.mom); dfree(o.walk); dfree(o.walks); dfree(o.quad); dfree(o.quadf);
  dfree(o.fifo); dfree(o.nleaf_sub); dfree(o.nempty_sub); dfree(o.leaf_base); dfree(o.empty_base);
  dfree(h->flags); dfree(h->buckets); dfree(h->bucket_work); dfree(h->list_count); dfree(h->list_off); dfree(h->list_node);
  dfree(h->list_kind); dfree(h->dsum); dfree(h->adj); dfree(h->nadj); dfree(h->d_htab); dfree(h->ewd); dfree(h->sph); dfree(h->sph_nbr); dfree(h->sph_nd2);
  dfree(h->sph_list_d); dfree(h->sph_list_i); dfree(h->sph_state);
  dfree(h->pool_pc); dfree(h->pool_pp); dfree(h->l_pc_start); dfree(h->l_pp_start); dfree(h->l_pc_count);
  dfree(h->l_pp_count); dfree(h->d_lcur); dfree(h->d_work3); dfree(h->d_smq);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return PT_OK;
}

const char* pt_last_error(const pt_handle* h) { return h ? h->err.c_str() : "null handle"; }

int pt_set_stream(pt_handle* h, void* stream) {
  if (!h) return PT_E_ARG;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return PT_OK;
}

int pt_set_theta(pt_handle* h, double theta) {
  if (!h || !(theta > 0.0)) return PT_E_ARG;
  h->cfg.theta = theta;
  return PT_OK;
}

int pt_set_precision(pt_handle* h, int precision) {
  if (!h || (precision != PT_FP64 && precision != PT_MIXED && precision != PT_FP64_LISTS)) return PT_E_ARG;
  h->cfg.precision = precision;
  return PT_OK;
}

int pt_set_sort_spin_limit(pt_handle* h, int64_t polls) {
  if (!h || polls < 0) return PT_E_ARG;
  h->sort_spin_limit = (long long)polls;
  return PT_OK;
}

int pt_set_list_region(pt_handle* h, int64_t entries) {
  if (!h || entries < 64 || entries > (1 << 30)) return PT_E_ARG;
  h->l_region = (unsigned)entries;
  return PT_OK;
}

int pt_set_particles(pt_handle* h, int64_t n, const double* x, const double* y, const double* z, const double* vx,
                     const double* vy, const double* vz, const double* m, const double* soft) {
  if (!h) return PT_E_ARG;
  cudaSetDevice(h->cfg.device);
  const double* src[8] = {x, y, z, vx, vy, vz, m, soft};
  CKR(set_particles_impl(h, n, src, cudaMemcpyHostToDevice));
  CK(cudaStreamSynchronize(h->stream));
  return PT_OK;
}

int pt_set_particles_device(pt_handle* h, int64_t n, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz, const double* m,
                            const double* soft) {
  if (!h) return PT_E_ARG;
  cudaSetDevice(h->cfg.device);
  const double* src[8] = {x, y, z, vx, vy, vz, m, soft};
  return set_particles_impl(h, n, src, cudaMemcpyDeviceToDevice);
}

int64_t pt_num_particles(const pt_handle* h) { return h ? h->n : -1; }

int pt_compute_forces(pt_handle* h) {
  if (!h) return PT_E_ARG;
  cudaSetDevice(h->cfg.device);
  return forces(h, 0, INT64_MAX);
}

int pt_compute_forces_range(pt_handle* h, int64_t b0, int64_t b1) {
  if (!h || b0 < 0 || b1 < b0) return PT_E_ARG;
  cudaSetDevice(h->cfg.device);
  return forces(h, b0, b1);
}

int pt_get_accel(pt_handle* h, double* ax, double* ay, double* az, double* pot, double* pot_full) {
  if (!h) return PT_E_ARG;
  if (!h->have_forces) return fail(h, PT_E_STATE, "no force pass yet");
  if (h->n == 0) return PT_OK;
  cudaSetDevice(h->cfg.device);
  const double* src[5] = {h->p.ax, h->p.ay, h->p.az, h->p.pot, h->p.potf};
  double* dst[5] = {ax, ay, az, pot, pot_full};
  for (int i = 0; i < 5; i++) {
    CKR(unpermute_f64(h, src[i], dst[i]));
    if (dst[i]) CK(cudaStreamSynchronize(h->stream));
  }
  return PT_OK;
}

int pt_device_accel(pt_handle* h, double** ax, double** ay, double** az, double** pot, double** pot_full,
                    const int32_t** order) {
  if (!h) return PT_E_ARG;
  if (ax) *ax = h->p.ax;
  if (ay) *ay = h->p.ay;
  if (az) *az = h->p.az;
  if (pot) *pot = h->p.pot;
  if (pot_full) *pot_full = h->p.potf;
  if (order) *order = h->p.order;
  return PT_OK;
}

// Density pass on a rebuilt tree; leaves density and ball^2 (sorted order) in
// h->sph and, with want_nbr, the neighbour lists in h->sph_nbr / h->sph_nd2.
// h->sph holds 7 N doubles: density, ball^2, and the pressure pass's u, ax,
// ay, az, PdV.
static int sph_density_device(pt_handle* h, bool want_nbr) {
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  const int k = sph_k();
  CKR(keys_and_sort(h));
  CKR(build_tree(h));
  CKR(upward(h));
  // the particle arrays were re-sorted: results of an earlier force pass no longer line up
  h->have_forces = false;
  h->forces_current = false;
  h->lists_valid = false;
  if (7 * n > h->sph_cap) {
    CKR(dalloc(h, &h->sph, 7 * n));
    h->sph_cap = 7 * n;
  }
  if (want_nbr && n * k > h->sph_nbr_cap) {
    CKR(dalloc(h, &h->sph_nbr, n * k));
    CKR(dalloc(h, &h->sph_nd2, n * k));
    h->sph_nbr_cap = n * k;
  }
  // per-warp candidate lists of the neighbour search: 32 targets x 32 entries
  const int kgrid = h->sms * 7;
  const int64_t slots = sph_knn_slots(kgrid);
  if (slots * 1024 > h->sph_list_cap) {
    CKR(dalloc(h, &h->sph_list_d, slots * 1024));
    CKR(dalloc(h, &h->sph_list_i, slots * 1024));
    h->sph_list_cap = slots * 1024;
  }
  CK(cudaMemsetAsync(h->d_work, 0, sizeof(unsigned), st));
  launch_sph_density(h->p, n, h->nd.mom, h->nd.walk, h->buckets, h->nbuckets, h->nnodes, h->sph, h->sph + n,
                     want_nbr ? h->sph_nbr : nullptr, want_nbr ? h->sph_nd2 : nullptr, h->sph_list_d,
                     h->sph_list_i, h->d_work, h->d_status, kgrid, st);
  CK(cudaGetLastError());
  return read_status(h);
}

int pt_sph_density(pt_handle* h, double* density, double* ball_sq, int32_t* nbr, double* nbr_d2) {
  if (!h || ((nbr == nullptr) != (nbr_d2 == nullptr))) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  const int k = sph_k();
  if (n == 0) return PT_OK;
  const bool want_nbr = nbr != nullptr;
  CKR(sph_density_device(h, want_nbr));
  CKR(unpermute_f64(h, h->sph, density));
  CK(cudaStreamSynchronize(st));
  CKR(unpermute_f64(h, h->sph + n, ball_sq));
  CK(cudaStreamSynchronize(st));
  if (want_nbr) {
    // neighbours of sorted particle i -> caller order, each list sorted by (d2, caller index)
    std::vector<int32_t> hn((size_t)n * k), order(n);
    std::vector<double> hd((size_t)n * k);
    CK(cudaMemcpyAsync(hn.data(), h->sph_nbr, hn.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hd.data(), h->sph_nd2, hd.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(order.data(), h->p.order, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<std::pair<double, int32_t>> row(k);
    for (int64_t i = 0; i < n; i++) {
      int m = 0;
      for (int e = 0; e < k; e++) {
        const int32_t j = hn[(size_t)i * k + e];
        if (j >= 0) row[m++] = {hd[(size_t)i * k + e], order[j]};
      }
      std::sort(row.begin(), row.begin() + m);
      const int64_t c = order[i];
      for (int e = 0; e < k; e++) {
        nbr[c * k + e] = e < m ? row[e].second : -1;
        nbr_d2[c * k + e] = e < m ? row[e].first : -1.0;
      }
    }
  }
  return PT_OK;
}

int pt_sph_pressure(pt_handle* h, const double* u, double* density, double* ax, double* ay, double* az,
                    double* pdv) {
  if (!h || !u) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  if (n == 0) return PT_OK;
  CKR(sph_density_device(h, true));
  double* us = h->sph + 2 * n;
  double* out = h->sph + 3 * n;  // ax, ay, az, PdV
  CK(cudaMemcpyAsync(h->tmp_d, u, n * sizeof(double), cudaMemcpyHostToDevice, st));
  launch_gather_by_order(h->tmp_d, us, h->p.order, n, grid_for(h, n), st);
  CK(cudaMemsetAsync(out, 0, 4 * n * sizeof(double), st));
  launch_sph_pressure(h->p, h->sph, h->sph + n, us, h->sph_nbr, h->sph_nd2, n, out, out + n, out + 2 * n,
                      out + 3 * n, h->d_status, h->sms * 16, st);
  CK(cudaGetLastError());
  CKR(read_status(h));
  double* dst[5] = {density, ax, ay, az, pdv};
  const double* src[5] = {h->sph, out, out + n, out + 2 * n, out + 3 * n};
  for (int i = 0; i < 5; i++) {
    CKR(unpermute_f64(h, src[i], dst[i]));
    CK(cudaStreamSynchronize(st));
  }
  return PT_OK;
}

// nsteps iterations of the SPH example: density pass, pressure pass with the
// predicted energies and velocities, then kick + perturb with the SPH updates.
// dt = max_timestep (examples/SPH.C getTimestep).  The caller-order state
// (u, u_pred, v_pred) stays on the device across the steps; the sorted copies
// the pressure pass reads are gathered by p.order after each re-sort.
int pt_sph_step(pt_handle* h, int nsteps, double* u, double* u_pred, double* vpx, double* vpy, double* vpz) {
  if (!h || nsteps < 0 || !u || !u_pred || !vpx || !vpy || !vpz) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  if (!(h->cfg.dt_max > 0.0)) return fail(h, PT_E_ARG, "dt_max must be positive");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  if (n == 0 || nsteps == 0) return PT_OK;
  if (8 * n > h->sph_state_cap) {
    CKR(dalloc(h, &h->sph_state, 8 * n));
    h->sph_state_cap = 8 * n;
  }
  double* cs = h->sph_state;  // caller order: u, u_pred, vpx, vpy, vpz
  double* vps = cs + 5 * n;   // sorted v_pred
  double* in[5] = {u, u_pred, vpx, vpy, vpz};
  for (int k = 0; k < 5; k++) CK(cudaMemcpyAsync(cs + k * n, in[k], n * sizeof(double), cudaMemcpyHostToDevice, st));
  const int g = grid_for(h, n);
  const double dt = h->cfg.dt_max;
  for (int s = 0; s < nsteps; s++) {
    CKR(sph_density_device(h, true));  // re-sorts the particles, builds the tree, density + neighbours
    double* us = h->sph + 2 * n;
    double* out = h->sph + 3 * n;  // ax, ay, az, PdV
    launch_gather_by_order(cs + n, us, h->p.order, n, g, st);
    for (int d = 0; d < 3; d++) launch_gather_by_order(cs + (2 + d) * n, vps + d * n, h->p.order, n, g, st);
    CK(cudaMemsetAsync(out, 0, 4 * n * sizeof(double), st));
    Particles q = h->p;  // the pressure pass reads velocity_predicted
    q.vx = vps;
    q.vy = vps + n;
    q.vz = vps + 2 * n;
    launch_sph_pressure(q, h->sph, h->sph + n, us, h->sph_nbr, h->sph_nd2, n, out, out + n, out + 2 * n,
                        out + 3 * n, h->d_status, h->sms * 16, st);
    CK(cudaGetLastError());
    CKR(read_status(h));  // a failed pressure pass leaves the particles as they were
    launch_sph_kick_perturb(h->p, out, out + n, out + 2 * n, out + 3 * n, cs, cs + n, cs + 2 * n, cs + 3 * n,
                            cs + 4 * n, n, dt, g, st);
    CK(cudaGetLastError());
    CKR(read_status(h));
    h->last_dt = dt;
  }
  double* outs[5] = {u, u_pred, vpx, vpy, vpz};
  for (int k = 0; k < 5; k++) CK(cudaMemcpyAsync(outs[k], cs + k * n, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return PT_OK;
}

int pt_get_bucket_work(pt_handle* h, uint64_t* work) {
  if (!h || !work) return PT_E_ARG;
  if (!h->have_forces) return fail(h, PT_E_STATE, "no force pass yet");
  if (h->nbuckets == 0) return PT_OK;
  cudaSetDevice(h->cfg.device);
  CK(cudaMemcpyAsync(work, h->bucket_work, h->nbuckets * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PT_OK;
}

int pt_advance(pt_handle* h, double* dt_out) {
  if (!h) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  if (!h->have_forces || !h->forces_current) return fail(h, PT_E_STATE, "no force pass at the current positions");
  cudaSetDevice(h->cfg.device);
  double dt = 0.0;
  if (h->n > 0) {
    CKR(timestep(h, &dt));
    launch_kick_perturb(h->p, h->n, dt, grid_for(h, h->n), h->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
  }
  h->last_dt = dt;
  h->forces_current = false;
  if (dt_out) *dt_out = dt;
  return PT_OK;
}

int pt_step(pt_handle* h, int nsteps) {
  if (!h || nsteps < 0) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  cudaSetDevice(h->cfg.device);
  const int g = grid_for(h, h->n);
  for (int s = 0; s < nsteps; s++) {
    if (h->cfg.integrator == PT_KKD) {
      CKR(forces(h, 0, INT64_MAX));
      double dt;
      CKR(timestep(h, &dt));
      h->last_dt = dt;
      launch_kick_perturb(h->p, h->n, dt, g, h->stream);
      CK(cudaGetLastError());
      h->forces_current = false;
    } else {
      if (!h->forces_current) CKR(forces(h, 0, INT64_MAX));
      double dt;
      CKR(timestep(h, &dt));
      h->last_dt = dt;
      launch_kick_half(h->p, h->n, dt, g, h->stream);
      launch_drift(h->p, h->n, dt, g, h->stream);
      CK(cudaGetLastError());
      CKR(forces(h, 0, INT64_MAX));
      launch_kick_half(h->p, h->n, dt, g, h->stream);
      CK(cudaGetLastError());
    }
  }
  CK(cudaStreamSynchronize(h->stream));
  return PT_OK;
}

int pt_get_state(pt_handle* h, double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  if (!h) return PT_E_ARG;
  if (h->n == 0) return PT_OK;
  cudaSetDevice(h->cfg.device);
  const double* src[6] = {h->p.x, h->p.y, h->p.z, h->p.vx, h->p.vy, h->p.vz};
  double* dst[6] = {x, y, z, vx, vy, vz};
  for (int i = 0; i < 6; i++) {
    CKR(unpermute_f64(h, src[i], dst[i]));
    if (dst[i]) CK(cudaStreamSynchronize(h->stream));
  }
  return PT_OK;
}

int pt_last_dt(const pt_handle* h, double* dt) {
  if (!h || !dt) return PT_E_ARG;
  *dt = h->last_dt;
  return PT_OK;
}

int pt_get_keys(pt_handle* h, uint64_t* keys) {
  if (!h || !keys) return PT_E_ARG;
  if (!h->have_forces) return fail(h, PT_E_STATE, "no force pass yet");
  if (h->n == 0) return PT_OK;
  cudaSetDevice(h->cfg.device);
  launch_scatter_u64(h->p.key, h->key_alt, h->p.order, h->n, grid_for(h, h->n), h->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(keys, h->key_alt, h->n * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PT_OK;
}

int pt_get_universe(pt_handle* h, double* lo3, double* hi3) {
  if (!h || !lo3 || !hi3) return PT_E_ARG;
  double u[6];
  CK(cudaMemcpyAsync(u, h->d_uni, sizeof(u), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int d = 0; d < 3; d++) {
    lo3[d] = u[d];
    hi3[d] = u[3 + d];
  }
  return PT_OK;
}

int pt_get_tree_size(pt_handle* h, int64_t* n_nodes, int64_t* n_buckets) {
  if (!h) return PT_E_ARG;
  if (n_nodes) *n_nodes = h->nnodes;
  if (n_buckets) *n_buckets = h->nbuckets;
  return PT_OK;
}

int pt_get_tree(pt_handle* h, uint64_t* keys, int32_t* ints4, double* dbls18) {
  if (!h) return PT_E_ARG;
  const int64_t nn = h->nnodes;
  if (nn == 0) return PT_OK;
  cudaStream_t st = h->stream;
  std::vector<int32_t> type(nn), depth(nn), count(nn);
  std::vector<Mom> mom(nn);
  if (keys) CK(cudaMemcpyAsync(keys, h->nd.key, nn * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(type.data(), h->nd.type, nn * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(depth.data(), h->nd.depth, nn * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(count.data(), h->nd.count, nn * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(mom.data(), h->nd.mom, nn * sizeof(Mom), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int64_t i = 0; i < nn; i++) {
    if (ints4) {
      ints4[4 * i + 0] = type[i];
      ints4[4 * i + 1] = depth[i];
      ints4[4 * i + 2] = count[i];
      ints4[4 * i + 3] = (type[i] == kTypeInternal) ? 8 : 0;
    }
    if (dbls18) {
      const Mom& q = mom[i];
      double* d = dbls18 + 18 * i;
      d[0] = q.mass; d[1] = q.cm[0]; d[2] = q.cm[1]; d[3] = q.cm[2]; d[4] = q.soft; d[5] = q.radius;
      d[6] = q.xx; d[7] = q.xy; d[8] = q.xz; d[9] = q.yy; d[10] = q.yz; d[11] = q.zz;
      d[12] = q.lo[0]; d[13] = q.lo[1]; d[14] = q.lo[2]; d[15] = q.hi[0]; d[16] = q.hi[1]; d[17] = q.hi[2];
    }
  }
  return PT_OK;
}

int pt_get_bucket_keys(pt_handle* h, uint64_t* keys) {
  if (!h || !keys) return PT_E_ARG;
  const int64_t nb = h->nbuckets;
  if (nb == 0) return PT_OK;
  std::vector<int32_t> b(nb);
  std::vector<uint64_t> nk(h->nnodes);
  CK(cudaMemcpyAsync(b.data(), h->buckets, nb * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(nk.data(), h->nd.key, h->nnodes * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int64_t i = 0; i < nb; i++) keys[i] = nk[b[i]];
  return PT_OK;
}

int pt_get_lists_size(pt_handle* h, int64_t* total) {
  if (!h || !total) return PT_E_ARG;
  if (!h->lists_valid) return fail(h, PT_E_STATE, "no interaction lists recorded (config.record_lists)");
  *total = h->list_total;
  return PT_OK;
}

int pt_get_lists(pt_handle* h, int64_t* offsets, uint64_t* keys, int32_t* kinds) {
  if (!h) return PT_E_ARG;
  if (!h->lists_valid) return fail(h, PT_E_STATE, "no interaction lists recorded (config.record_lists)");
  const int64_t nb = h->list_nb - 1, tot = h->list_total;
  std::vector<int64_t> off(nb + 1);
  std::vector<int32_t> node(tot);
  std::vector<int8_t> kind(tot);
  std::vector<uint64_t> nk(h->nnodes);
  cudaStream_t st = h->stream;
  CK(cudaMemcpyAsync(off.data(), h->list_off, (nb + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  if (tot) {
    CK(cudaMemcpyAsync(node.data(), h->list_node, tot * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(kind.data(), h->list_kind, tot * sizeof(int8_t), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaMemcpyAsync(nk.data(), h->nd.key, h->nnodes * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (offsets)
    for (int64_t i = 0; i <= nb; i++) offsets[i] = off[i];
  for (int64_t i = 0; i < tot; i++) {
    if (keys) keys[i] = nk[node[i]];
    if (kinds) kinds[i] = kind[i] ? 1 : 0;  // node() entries, softened or not, are kind 1
  }
  return PT_OK;
}

int pt_get_list_digests(pt_handle* h, int which, uint64_t* digest, int64_t* count) {
  if (!h || (which != 0 && which != 1)) return PT_E_ARG;
  const int64_t nb = h->nbuckets;
  if (which == 0 && !(h->lists_valid && !h->trav_range_partial && h->list_nb - 1 == nb))
    return fail(h, PT_E_STATE, "no interaction lists recorded for every bucket (config.record_lists)");
  if (which == 1 && !h->tp_lists_valid)
    return fail(h, PT_E_STATE, "the last pass was not a two-phase mixed pass over every bucket");
  if (nb == 0) return PT_OK;
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  DevBuf buf;
  CK(cudaMalloc((void**)&buf.p, 2 * nb * sizeof(double)));
  unsigned long long* d_dig = reinterpret_cast<unsigned long long*>(buf.p);
  int64_t* d_cnt = reinterpret_cast<int64_t*>(buf.p + nb);
  if (which == 0)
    launch_digest_recorded(h->list_off, h->list_node, h->list_kind, nb, d_dig, d_cnt, st);
  else
    launch_digest_two_phase(h->pool_pc, h->pool_pp, h->l_pc_start, h->l_pc_count, h->l_pp_start, h->l_pp_count, nb,
                            d_dig, d_cnt, st);
  CK(cudaGetLastError());
  if (digest) CK(cudaMemcpyAsync(digest, d_dig, nb * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  if (count) CK(cudaMemcpyAsync(count, d_cnt, nb * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return PT_OK;
}

int pt_get_counters(pt_handle* h, pt_counters* c) {
  if (!h || !c) return PT_E_ARG;
  *c = h->last;
  return PT_OK;
}

int pt_direct_sum(pt_handle* h, int64_t nt, const int32_t* targets, double* ax, double* ay, double* az,
                  double* pot) {
  if (!h || nt < 0 || (nt > 0 && !targets)) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  const int64_t n = h->n;
  if (nt == 0 || n == 0) return PT_OK;
  for (int64_t t = 0; t < nt; t++)
    if (targets[t] < 0 || targets[t] >= n) return fail(h, PT_E_ARG, "target index out of range");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int tb = (int)((nt + 255) / 256);
  int nsplit = std::max(1, std::min(256, (4 * h->sms + tb - 1) / tb));
  if (n < 4096) nsplit = 1;
  const int64_t need = 5 * n + 4 * nt * nsplit + nt;
  if (need > h->dsum_cap) {
    CKR(dalloc(h, &h->dsum, need));
    h->dsum_cap = need;
  }
  // caller-order copies of x, y, z, m, soft
  const double* src[5] = {h->p.x, h->p.y, h->p.z, h->p.m, h->p.soft};
  for (int k = 0; k < 5; k++) launch_scatter_f64(src[k], h->dsum + k * n, h->p.order, n, grid_for(h, n), st);
  int32_t* dt = reinterpret_cast<int32_t*>(h->dsum + 5 * n + 4 * nt * nsplit);
  CK(cudaMemcpyAsync(dt, targets, nt * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  double* part = h->dsum + 5 * n;
  launch_direct_sum(h->dsum, h->dsum + n, h->dsum + 2 * n, h->dsum + 3 * n, h->dsum + 4 * n, n, dt, nt, nsplit,
                    part, st);
  CK(cudaGetLastError());
  std::vector<double> hp((size_t)4 * nt * nsplit);
  CK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int64_t t = 0; t < nt; t++) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int sl = 0; sl < nsplit; sl++)
      for (int k = 0; k < 4; k++) s[k] += hp[((size_t)sl * nt + t) * 4 + k];
    if (ax) ax[t] = s[0];
    if (ay) ay[t] = s[1];
    if (az) az[t] = s[2];
    if (pot) pot[t] = s[3];
  }
  return PT_OK;
}

// FP64 periodic (Ewald) direct sum: alpha = 4/L, real-space images within
// 1.5 L (erfc(6) ~ 2e-17), reciprocal |h|^2 <= 64 (exp(-pi^2 64/16) ~ 7e-18),
// the spline kernel for the nearest image within soft_i + soft_j, and the
// background and self terms in the potential.
int pt_ewald_direct_sum(pt_handle* h, int64_t nt, const int32_t* targets, double* ax, double* ay, double* az,
                        double* pot) {
  if (!h || nt < 0 || (nt > 0 && !targets)) return PT_E_ARG;
  if (!h->p.x) return fail(h, PT_E_STATE, "no particles");
  if (!(h->cfg.period > 0.0)) return fail(h, PT_E_ARG, "period must be positive");
  const int64_t n = h->n;
  if (nt == 0 || n == 0) return PT_OK;
  for (int64_t t = 0; t < nt; t++)
    if (targets[t] < 0 || targets[t] >= n) return fail(h, PT_E_ARG, "target index out of range");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const double L = h->cfg.period, V = L * L * L;
  const double alpha = 4.0 / L, rcut = 1.5 * L;
  const int hmax = 8;
  std::vector<double4> kv;
  for (int hx = -hmax; hx <= hmax; hx++)
    for (int hy = -hmax; hy <= hmax; hy++)
      for (int hz = -hmax; hz <= hmax; hz++) {
        const int h2 = hx * hx + hy * hy + hz * hz;
        if (h2 == 0 || h2 > hmax * hmax) continue;
        const double kx = 2 * M_PI / L * hx, ky = 2 * M_PI / L * hy, kz = 2 * M_PI / L * hz;
        const double k2 = kx * kx + ky * ky + kz * kz;
        kv.push_back(make_double4(kx, ky, kz, 4 * M_PI / V * std::exp(-k2 / (4 * alpha * alpha)) / k2));
      }
  const int nk = (int)kv.size();
  kv.push_back(make_double4(0.0, 0.0, 0.0, 0.0));  // k = 0: total mass
  const int tb = (int)((nt + 127) / 128);
  int nsplit = std::max(1, std::min(256, (4 * h->sms + tb - 1) / tb));
  if (n < 4096) nsplit = 1;
  // doubles: caller-order x y z m soft (5n) | partials (4 nt nsplit) | recip out (4 nt) | S (2 nk + 2)
  //          | k vectors (4 (nk + 1), 32-byte aligned) | targets (int32, nt / 2 + 1 doubles)
  const int64_t off_part = 5 * n, off_rec = off_part + 4 * nt * nsplit, off_S = off_rec + 4 * nt;
  const int64_t off_kv = (off_S + 2 * (nk + 1) + 3) / 4 * 4;
  const int64_t off_tgt = off_kv + 4 * (nk + 1);
  const int64_t need = off_tgt + nt / 2 + 1;
  if (need > h->ewd_cap) {
    CKR(dalloc(h, &h->ewd, need));
    h->ewd_cap = need;
  }
  double* c = h->ewd;
  const double* src[5] = {h->p.x, h->p.y, h->p.z, h->p.m, h->p.soft};
  for (int k = 0; k < 5; k++) launch_scatter_f64(src[k], c + k * n, h->p.order, n, grid_for(h, n), st);
  double* part = c + off_part;
  double* rec = c + off_rec;
  double* S = c + off_S;
  double4* dkv = reinterpret_cast<double4*>(c + off_kv);
  int32_t* dt = reinterpret_cast<int32_t*>(c + off_tgt);
  CK(cudaMemcpyAsync(dkv, kv.data(), kv.size() * sizeof(double4), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dt, targets, nt * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  launch_ewald_structure(c, c + n, c + 2 * n, c + 3 * n, n, dkv, nk + 1, S, st);
  launch_ewald_real(c, c + n, c + 2 * n, c + 3 * n, c + 4 * n, n, dt, nt, nsplit, L, alpha, rcut, part, st);
  launch_ewald_recip(c, c + n, c + 2 * n, c + 3 * n, dt, nt, dkv, nk, S, alpha, V, rec, st);
  CK(cudaGetLastError());
  std::vector<double> hp((size_t)4 * nt * nsplit), hr((size_t)4 * nt);
  CK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(hr.data(), rec, hr.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int64_t t = 0; t < nt; t++) {
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
    for (int sl = 0; sl < nsplit; sl++)
      for (int k = 0; k < 4; k++) s4[k] += hp[((size_t)sl * nt + t) * 4 + k];
    for (int k = 0; k < 4; k++) s4[k] += hr[4 * t + k];
    if (ax) ax[t] = s4[0];
    if (ay) ay[t] = s4[1];
    if (az) az[t] = s4[2];
    if (pot) pot[t] = s4[3];
  }
  return PT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- differentiation
namespace {

int ensure_adjoint(pt_handle* h) {
  const int64_t need = 21 * std::max<int64_t>(h->n, 1);
  if (need > h->adj_cap) {
    CKR(dalloc(h, &h->adj, need));
    h->adj_cap = need;
  }
  const int64_t nneed = 10 * std::max<int64_t>(h->nnodes, 1);
  if (nneed > h->nadj_cap) {
    CKR(dalloc(h, &h->nadj, nneed));
    h->nadj_cap = nneed;
  }
  return PT_OK;
}

bool lists_cover_all(const pt_handle* h) {
  return h->lists_valid && !h->trav_range_partial && h->list_nb - 1 == h->nbuckets;
}

// Leaf moments, upward pass and traversal records on the existing topology.
int recompute_moments(pt_handle* h) {
  cudaStream_t st = h->stream;
  launch_leaf_moments(h->nd, h->nnodes, h->p, st);
  const int L = (int)h->lev.size() - 1;
  for (int l = L - 1; l >= 0; l--) launch_upward_level(h->nd, h->lev[l], h->lev[l + 1] - h->lev[l], st);
  const double gfac = (4.0 / 3.0) / (h->cfg.theta * h->cfg.theta);
  launch_finalize(h->nd, h->nnodes, gfac, h->cfg.precision == PT_MIXED, st);
  CK(cudaGetLastError());
  return PT_OK;
}

// Gradient of sum_i cot_i . a_i for the recorded lists.  cot: caller order,
// device; outputs: caller order, device (gx, gy, gz, gm; added into when
// accumulate is set).
int adjoint_device(pt_handle* h, const double* cx, const double* cy, const double* cz, double* gx, double* gy,
                   double* gz, double* gm, bool accumulate) {
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  const int g = grid_for(h, n);
  CKR(ensure_adjoint(h));
  double* cs = h->adj;       // 3N sorted cotangent
  double* gs = h->adj + 3 * n;  // 4N sorted gradient
  double* tmp = h->adj + 7 * n;  // 4N caller-order gradient
  launch_gather_by_order(cx, cs, h->p.order, n, g, st);
  launch_gather_by_order(cy, cs + n, h->p.order, n, g, st);
  launch_gather_by_order(cz, cs + 2 * n, h->p.order, n, g, st);
  CK(cudaMemsetAsync(gs, 0, 4 * n * sizeof(double), st));
  CK(cudaMemsetAsync(h->nadj, 0, 10 * h->nnodes * sizeof(double), st));
  CK(cudaMemsetAsync(h->d_work, 0, sizeof(unsigned), st));
  AdjParams A{};
  A.p = h->p;
  A.walk = h->nd.walk;
  A.quad = h->nd.quad;
  A.mom = h->nd.mom;
  A.parent = h->nd.parent;
  A.buckets = h->buckets;
  A.nbuckets = h->nbuckets;
  A.nnodes = h->nnodes;
  A.list_off = h->list_off;
  A.list_node = h->list_node;
  A.list_kind = h->list_kind;
  A.cax = cs;
  A.cay = cs + n;
  A.caz = cs + 2 * n;
  A.gx = gs;
  A.gy = gs + n;
  A.gz = gs + 2 * n;
  A.gm = gs + 3 * n;
  A.nadj = h->nadj;
  A.work = h->d_work;
  A.status = h->d_status;
  launch_adjoint(A, h->sms * 8, st);
  CK(cudaGetLastError());
  double* outs[4] = {gx, gy, gz, gm};
  for (int k = 0; k < 4; k++) {
    if (!outs[k]) continue;
    if (accumulate) {
      launch_scatter_f64(gs + k * n, tmp + k * n, h->p.order, n, g, st);
      launch_axpy1(n, 1.0, tmp + k * n, outs[k], g, st);
    } else {
      launch_scatter_f64(gs + k * n, outs[k], h->p.order, n, g, st);
    }
  }
  CK(cudaGetLastError());
  return read_status(h);
}

}  // namespace

extern "C" {

int pt_forces_frozen(pt_handle* h, const double* x, const double* y, const double* z, const double* m) {
  if (!h) return PT_E_ARG;
  if (!lists_cover_all(h)) return fail(h, PT_E_STATE, "needs a full force pass with config.record_lists");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  const int g = grid_for(h, n);
  CKR(ensure_adjoint(h));
  const double* src[4] = {x, y, z, m};
  double* dst[4] = {h->p.x, h->p.y, h->p.z, h->p.m};
  for (int k = 0; k < 4; k++) {
    if (!src[k]) continue;
    CK(cudaMemcpyAsync(h->adj, src[k], n * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_gather_by_order(h->adj, dst[k], h->p.order, n, g, st);
  }
  CKR(recompute_moments(h));
  TravParams P{};
  P.p = h->p;
  P.walk = h->nd.walk;
  P.walks = h->nd.walks;
  P.quad = h->nd.quad;
  P.buckets = h->buckets;
  P.b_begin = 0;
  P.b_end = h->nbuckets;
  P.nnodes = h->nnodes;
  P.list_off = h->list_off;
  P.list_node = h->list_node;
  P.list_kind = h->list_kind;
  P.status = h->d_status;
  P.work = h->d_work;
  CK(cudaMemsetAsync(h->d_work, 0, sizeof(unsigned), st));
  launch_replay_f64(P, h->sms * 16, st);
  CK(cudaGetLastError());
  return read_status(h);
}

int pt_adjoint(pt_handle* h, const double* cax, const double* cay, const double* caz, double* gx, double* gy,
               double* gz, double* gm) {
  if (!h || !cax || !cay || !caz) return PT_E_ARG;
  if (!lists_cover_all(h)) return fail(h, PT_E_STATE, "needs a full force pass with config.record_lists");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  if (n == 0) return PT_OK;
  CKR(ensure_adjoint(h));
  double* buf = h->adj + 14 * n;  // caller-order cotangent (3N) and gradients (4N), kept by the handle
  const double* hin[3] = {cax, cay, caz};
  for (int k = 0; k < 3; k++) {
    CK(cudaMemcpyAsync(buf + k * n, hin[k], n * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  int rc = adjoint_device(h, buf, buf + n, buf + 2 * n, buf + 3 * n, buf + 4 * n, buf + 5 * n, buf + 6 * n, false);
  if (rc == PT_OK) {
    double* hout[4] = {gx, gy, gz, gm};
    for (int k = 0; k < 4; k++)
      if (hout[k]) CK(cudaMemcpyAsync(hout[k], buf + (3 + k) * n, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------- K-step chain
namespace {

// Caller-order state -> particle arrays (order reset to identity).
int load_state(pt_handle* h, const double* X, const double* V, const double* M, const double* S) {
  const int64_t n = h->n;
  const double* src[8] = {X, X + n, X + 2 * n, V, V + n, V + 2 * n, M, S};
  return set_particles_impl(h, n, src, cudaMemcpyDeviceToDevice);
}

// Force pass with interaction lists; accelerations in caller order into A (3N).
int chain_forces(pt_handle* h, double* A) {
  const int saved = h->cfg.record_lists;
  h->cfg.record_lists = 1;
  const int rc = forces(h, 0, INT64_MAX);
  h->cfg.record_lists = saved;
  CKR(rc);
  const int64_t n = h->n;
  const int g = grid_for(h, n);
  launch_scatter_f64(h->p.ax, A, h->p.order, n, g, h->stream);
  launch_scatter_f64(h->p.ay, A + n, h->p.order, n, g, h->stream);
  launch_scatter_f64(h->p.az, A + 2 * n, h->p.order, n, g, h->stream);
  CK(cudaGetLastError());
  return PT_OK;
}

}  // namespace

extern "C" int pt_chain_grad(pt_handle* h, int nsteps, double dt, int ckpt_every, const double* yx, const double* yy,
                             const double* yz, double* loss, double* gx, double* gy, double* gz, double* gvx,
                             double* gvy, double* gvz, double* gm) {
  if (!h || nsteps < 1 || !(dt > 0.0) || !yx || !yy || !yz) return PT_E_ARG;
  if (!h->p.x || h->n == 0) return fail(h, PT_E_STATE, "no particles");
  cudaSetDevice(h->cfg.device);
  cudaStream_t st = h->stream;
  const int64_t n = h->n;
  const int g = grid_for(h, n);
  const int K = nsteps;
  int C = ckpt_every > 0 ? ckpt_every : std::max(1, (int)std::lround(std::sqrt((double)K)));
  if (C > K) C = K;
  const int nck = (K + C - 1) / C;
  // layout (doubles): X0 V0 M0 S0 | X V A | Y | xb vb mb pend | ckpt (nck x 6N) | seg ((C+1) x 3N)
  const int64_t off_X0 = 0, off_V0 = 3 * n, off_M0 = 6 * n, off_S0 = 7 * n, off_X = 8 * n, off_V = 11 * n,
                off_A = 14 * n, off_Y = 17 * n, off_xb = 20 * n, off_vb = 23 * n, off_mb = 26 * n, off_pd = 27 * n,
                off_ck = 30 * n, off_seg = off_ck + (int64_t)nck * 6 * n;
  const int64_t total = off_seg + (int64_t)(C + 1) * 3 * n;
  DevBuf buf;
  CK(cudaMalloc((void**)&buf.p, total * sizeof(double)));
  double* B = buf.p;
  double *X0 = B + off_X0, *V0 = B + off_V0, *M0 = B + off_M0, *S0 = B + off_S0, *X = B + off_X, *V = B + off_V,
         *A = B + off_A, *Y = B + off_Y, *xb = B + off_xb, *vb = B + off_vb, *mb = B + off_mb, *pd = B + off_pd,
         *ck = B + off_ck, *seg = B + off_seg;
  // initial state in caller order (the arrays may be key-sorted by an earlier pass)
  const double* cur[8] = {h->p.x, h->p.y, h->p.z, h->p.vx, h->p.vy, h->p.vz, h->p.m, h->p.soft};
  double* dst0[8] = {X0, X0 + n, X0 + 2 * n, V0, V0 + n, V0 + 2 * n, M0, S0};
  for (int k = 0; k < 8; k++) launch_scatter_f64(cur[k], dst0[k], h->p.order, n, g, st);
  const double* hy[3] = {yx, yy, yz};
  for (int k = 0; k < 3; k++) CK(cudaMemcpyAsync(Y + k * n, hy[k], n * sizeof(double), cudaMemcpyHostToDevice, st));
  auto copy3 = [&](double* d, const double* s) {
    return cudaMemcpyAsync(d, s, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  };
  // one KDK step from (X, V) with A = a(X) on entry; A = a(X') on exit
  auto kdk = [&]() -> int {
    launch_axpy3(n, 0.5 * dt, A, A + n, A + 2 * n, V, V + n, V + 2 * n, g, st);
    launch_axpy3(n, dt, V, V + n, V + 2 * n, X, X + n, X + 2 * n, g, st);
    CKR(load_state(h, X, V, M0, S0));
    CKR(chain_forces(h, A));
    launch_axpy3(n, 0.5 * dt, A, A + n, A + 2 * n, V, V + n, V + 2 * n, g, st);
    return PT_OK;
  };

  // forward, keeping (X, V) every C steps
  CK(copy3(X, X0));
  CK(copy3(V, V0));
  CKR(load_state(h, X, V, M0, S0));
  CKR(chain_forces(h, A));
  for (int s = 0; s < K; s++) {
    if (s % C == 0) {
      CK(copy3(ck + (int64_t)(s / C) * 6 * n, X));
      CK(copy3(ck + (int64_t)(s / C) * 6 * n + 3 * n, V));
    }
    CKR(kdk());
  }
  // loss = 0.5 sum |x_K - y|^2 and its gradient
  {
    std::vector<double> hx(3 * n);
    CK(cudaMemcpyAsync(hx.data(), X, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double L = 0.0;
    for (int k = 0; k < 3; k++)
      for (int64_t i = 0; i < n; i++) {
        const double d = hx[k * n + i] - hy[k][i];
        L += d * d;
      }
    if (loss) *loss = 0.5 * L;
  }
  CK(copy3(xb, X));
  launch_axpy3(n, -1.0, Y, Y + n, Y + 2 * n, xb, xb + n, xb + 2 * n, g, st);
  CK(cudaMemsetAsync(vb, 0, 3 * n * sizeof(double), st));
  CK(cudaMemsetAsync(mb, 0, n * sizeof(double), st));
  CK(cudaMemsetAsync(pd, 0, 3 * n * sizeof(double), st));

  // backward, segment by segment, recomputing each segment's positions
  for (int c = nck - 1; c >= 0; c--) {
    const int s0 = c * C, s1 = std::min(s0 + C, K);
    CK(copy3(X, ck + (int64_t)c * 6 * n));
    CK(copy3(V, ck + (int64_t)c * 6 * n + 3 * n));
    CK(copy3(seg, X));
    CKR(load_state(h, X, V, M0, S0));
    CKR(chain_forces(h, A));
    for (int s = s0; s < s1; s++) {
      CKR(kdk());
      CK(copy3(seg + (int64_t)(s + 1 - s0) * 3 * n, X));
    }
    for (int s = s1 - 1; s >= s0; s--) {
      // the point x_{s+1}: a(x_{s+1}) feeds v_{s+1} (and v_h of step s+1, already in pd)
      launch_axpy3(n, 0.5 * dt, vb, vb + n, vb + 2 * n, pd, pd + n, pd + 2 * n, g, st);
      if (s + 1 < K) {
        CKR(load_state(h, seg + (int64_t)(s + 1 - s0) * 3 * n, V, M0, S0));
        CKR(chain_forces(h, A));
        CKR(adjoint_device(h, pd, pd + n, pd + 2 * n, xb, xb + n, xb + 2 * n, mb, true));
      }
      // x_{s+1} = x_s + dt v_h ; v_h = v_s + dt/2 a(x_s)
      launch_axpy3(n, dt, xb, xb + n, xb + 2 * n, vb, vb + n, vb + 2 * n, g, st);
      CK(cudaMemsetAsync(pd, 0, 3 * n * sizeof(double), st));
      launch_axpy3(n, 0.5 * dt, vb, vb + n, vb + 2 * n, pd, pd + n, pd + 2 * n, g, st);
    }
  }
  // the point x_0
  CKR(load_state(h, X0, V0, M0, S0));
  CKR(chain_forces(h, A));
  CKR(adjoint_device(h, pd, pd + n, pd + 2 * n, xb, xb + n, xb + 2 * n, mb, true));
  double* hout[7] = {gx, gy, gz, gvx, gvy, gvz, gm};
  const double* dsrc[7] = {xb, xb + n, xb + 2 * n, vb, vb + n, vb + 2 * n, mb};
  for (int k = 0; k < 7; k++)
    if (hout[k]) CK(cudaMemcpyAsync(hout[k], dsrc[k], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  // leave the handle at the initial state (with its force pass)
  return PT_OK;
}
