// k_mixed2.cu -- K7 mixed-precision traversal in two phases.
//
// Phase A (walk_lists): one warp per bucket walks the tree exactly as the
// fused traversal does (FP64 opening and softening tests, GravityVisitor::
// open / openSoftening, so the same leaf() and node() interactions) and
// writes the bucket's interaction list to HBM: P2C node indices (bit 31 =
// monopole, addGravity; bit 30 = near: a target may lie inside the node's
// softening sphere) and P2P leaf indices.  Whether a P2P leaf may hold a
// softened pair, and how many source particles the leaves hold, are left to
// eval_p2p, which reads every leaf record anyway.  The walk reads the
// classification fields from the sibling blocks (walk_sib_index), so the
// eight lanes that classify one node's children load one 128-byte line per
// field row (with the 64-byte walk records the walk was bound by the L1 data
// pipe's wavefronts, not by arithmetic).  Each warp writes its terminals
// straight to regions it reserves
// from two global pools, so every bucket's list is contiguous; a bucket that
// outgrows what is left of its region moves its list so far to a new, larger
// region and goes on.  Only a full pool sets kErrPool (the host then repeats
// the walk with larger pools).
//
// Phase B (eval_p2c2 / eval_p2c, eval_p2p): one warp per bucket streams its
// list in chunks of 64 entries and evaluates them with the packed FP32
// instructions (two interactions per issue slot) on offsets relative to the
// bucket's centre of mass.  Each staged node or source meets two targets per
// packed instruction, so it is read from shared memory once for two (P2C)
// or four (P2P) evaluations.  The P2C evaluation stores (or, for replica
// walks after the first, adds) and eval_p2p adds.
#include "pt_internal.cuh"
#include "pt_walk.cuh"
#include "pt_f32.cuh"

namespace pt {


// Phase timers of a diagnostic build (PT_PROF=1): lane 0 adds the clock
// cycles since the previous mark to a per-warp slot in shared memory; the
// slots are summed into g_prof when the warp exits.
#ifndef PT_PROF
#define PT_PROF 0
#endif
#if PT_PROF
__device__ unsigned long long g_prof[32];
#define PROF_FIELDS unsigned prof[6]; unsigned tlast;
#define PROF_START(w) if (lane == 0) { for (int i_ = 0; i_ < 6; i_++) (w).prof[i_] = 0; (w).tlast = (unsigned)clock(); }
#define PROF_MARK(w, i) if (lane == 0) { const unsigned t_ = (unsigned)clock(); (w).prof[i] += t_ - (w).tlast; (w).tlast = t_; }
#define PROF_FLUSH(w, base) if (lane == 0) { for (int i_ = 0; i_ < 6; i_++) atomicAdd(&g_prof[(base) + i_], (unsigned long long)(w).prof[i_]); }
#else
#define PROF_FIELDS
#define PROF_START(w)
#define PROF_MARK(w, i)
#define PROF_FLUSH(w, base)
#endif

constexpr int kWlWarps = 4;
constexpr int kWlStack = 640;  // opened nodes pending (as the fused walk)
constexpr int kWlBuf = 64;

struct WalkWarp {
  BucketGeom geom;
  int32_t stack[kWlStack];
  PROF_FIELDS
};

// Per-warp region of one pool: [cur, end).
struct Region {
  unsigned long long cur, end;
};

// Reserve a new region when less than `thresh` entries are left (lane 0 calls
// the atomic; the result is broadcast).  Returns false if the pool is full.
__device__ __forceinline__ bool ensure_region(Region& r, unsigned long long* cursor, unsigned long long cap,
                                              unsigned region, unsigned thresh, int lane) {
  if (r.end - r.cur >= thresh) return true;
  unsigned long long s = 0;
  if (lane == 0) s = atomicAdd(cursor, (unsigned long long)region);
  s = __shfl_sync(kFull, s, 0);
  if (s + region > cap) {
    r.cur = r.end = cap;
    return false;
  }
  r.cur = s;
  r.end = s + region;
  return true;
}

#ifndef PT_SMQ_BATCH
#define PT_SMQ_BATCH 32
#endif
// The next bucket index of a warp (lane 0 grabs, all lanes receive it).  With
// smq, the warps of one SM take consecutive buckets from a batch of
// PT_SMQ_BATCH that the SM's queue holds, so the warps resident on an SM work
// on neighbouring buckets: their targets, results and most of their node
// records share cache lines.  (On the periodic 256^3 lattice pass, whose outer
// replica walks leave little work per bucket besides loading its targets and
// adding to its results, this measured 239.5 -> 214.4 ms; the Plummer pass at
// N = 2^24 is unchanged.)  A queue word is (batch start + 1) << 32 | next
// index; zero = no batch yet.
// The warp that draws index 0 of an empty queue, or the index one past the
// batch, takes a new batch from the global counter (keeping its first bucket);
// warps that draw past the batch meanwhile take single buckets.
__device__ __forceinline__ unsigned grab_bucket(unsigned* work, unsigned long long* smq, int lane) {
  unsigned bi = 0;
  if (lane == 0) {
    if (smq == nullptr) {
      bi = atomicAdd(work, 1u);
    } else {
      unsigned sm;
      asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
      unsigned long long* q = smq + (sm & 255u);
      const unsigned long long old = atomicAdd(q, 1ull);
      const unsigned hi = (unsigned)(old >> 32), idx = (unsigned)old;
      if (hi != 0u && idx < (unsigned)PT_SMQ_BATCH) {
        bi = hi - 1u + idx;
      } else if (hi == 0u ? idx == 0u : idx == (unsigned)PT_SMQ_BATCH) {
        bi = atomicAdd(work, (unsigned)PT_SMQ_BATCH);
        atomicExch(q, ((unsigned long long)(bi + 1u) << 32) | 1ull);
      } else {
        bi = atomicAdd(work, 1u);
      }
    }
  }
  return __shfl_sync(kFull, bi, 0);
}

// Room for n more entries of the bucket's list, which occupies [start,
// r.cur) of the warp's region: when they do not fit, the list so far moves to
// a new region of at least twice its new length.  False only if the pool is
// full.  Warp-uniform; the list's entries were written before the __syncwarp
// that ends each walk step.
__device__ __forceinline__ bool make_room(int n, Region& r, unsigned long long& start, int32_t* __restrict__ pool,
                                          unsigned long long* cursor, unsigned long long cap, unsigned region,
                                          int lane) {
  if (r.cur + (unsigned long long)n <= r.end) return true;
  const unsigned long long len = r.cur - start;
  const unsigned long long want = max((unsigned long long)region, 2ull * (len + (unsigned long long)n));
  unsigned long long s = 0;
  if (lane == 0) s = atomicAdd(cursor, want);
  s = __shfl_sync(kFull, s, 0);
  if (s + want > cap) {
    r.cur = r.end = cap;
    return false;
  }
  for (unsigned long long k = lane; k < len; k += 32) pool[s + k] = pool[start + k];
  start = s;
  r.cur = s + len;
  r.end = s + want;
  return true;
}

// CTAs per SM of the walk (72 registers); 6 and 8 measured slower at N = 2^24
#ifndef PT_WALK_MINB
#define PT_WALK_MINB 7
#endif
// kOffset: the replica offset (P.ox, P.oy, P.oz) may be non-zero (periodic
// walks); without it the walk skips three FP64 adds at the head of every
// classification's dependent chain (c + 0.0 == c, so the tests are unchanged).
template <bool kOffset>
__global__ void __launch_bounds__(kWlWarps * 32, PT_WALK_MINB) walk_lists(TravParams P, ListParams L,
                                                                         const Mom* __restrict__ mom) {
  __shared__ WalkWarp warps[kWlWarps];
  WalkWarp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  unsigned long long c_pc = 0, c_open = 0;
  unsigned max_len = 0;
  Region rpc{0, 0}, rpp{0, 0};
  bool pool_ok = true;
  const int nn32 = (int)min(P.nnodes, (int64_t)INT_MAX);  // node indices are 32-bit
  PROF_START(w);
  while (true) {
    const unsigned bi = grab_bucket(P.work, P.smq, lane);
    const int64_t b = P.b_begin + (int64_t)bi;
    if (b >= P.b_end) break;
    const int64_t lb = b - P.b_begin;
    const int tnode = P.buckets[b];
    if (tnode < 0 || tnode >= P.nnodes) {
      if (lane == 0) atomicOr(P.status, kErrCapacity);
      continue;
    }
    pool_ok = pool_ok && ensure_region(rpc, L.cursor + 0, L.cap_pc, L.region, L.thresh, lane) &&
              ensure_region(rpp, L.cursor + 1, L.cap_pp, L.region, L.thresh, lane);
    if (!pool_ok) {
      if (lane == 0) {
        atomicOr(P.status, kErrPool);
        L.pc_count[lb] = 0;
        L.pp_count[lb] = 0;
      }
      continue;
    }
    __syncwarp();
    if (lane == 0) load_bucket_geom(mom, tnode, w.geom);
    __syncwarp();
    // the bucket geometry in registers: every classification reads it
    const BucketGeom g = w.geom;
    const double blo[3] = {g.lo[0], g.lo[1], g.lo[2]}, bhi[3] = {g.hi[0], g.hi[1], g.hi[2]};
    const int ntot = P.walk[tnode].pcount;
    unsigned long long pc0 = rpc.cur, pp0 = rpp.cur;  // the bucket's lists start here (moved on overflow)
    // internal children classified (fits 32 bits per bucket): those accepted as
    // P2C nodes plus those opened, counted from the two ballots the step takes
    // anyway (one ballot fewer per step: 1.1 ms at N = 2^24)
    unsigned opens32 = 0;
    int sp = 0;
    int nexp = 1, pop = -1;
    bool ok = true, fits = true;
    PROF_MARK(w, 0);
    while (true) {
      const int e = lane >> 3, c = lane & 7;
      int node = -1;
      if (pop < 0) {
        if (lane == 0) node = 0;
      } else if (e < nexp) {
        node = w.stack[pop + e] + c;
      }
      int cls = kClsNone;
      double gap2 = -1.0;
      WalkRec r;
      if (node >= 0) {
        if (node >= nn32) {
          atomicOr(P.status, kErrCapacity);
        } else {
          if (node == 0) {
            r = P.walk[0];
          } else {  // the classification fields from the sibling blocks (3 lines per 8 lanes)
            const double2* sb = P.walks + walk_sib_index(node, 0);
            const double2 v0 = sb[0], v1 = sb[8], v2 = sb[16];
            r.cm[0] = v0.x;
            r.cm[1] = v0.y;
            r.cm[2] = v1.x;
            r.orsq = v1.y;
            r.soft = v2.x;
            const int tc = __double2hiint(v2.y);
            r.first_child = __double2loint(v2.y);
            r.type = tc & 7;
            r.count = tc >> 3;
          }
          if (kOffset) cls = classify_node_gap(r, blo, bhi, g, P.ox, P.oy, P.oz, gap2);
          else cls = classify_node_gap_nooff(r, blo, bhi, g, gap2);
        }
      }
      bool near = false;
      if (cls == kClsQuad) {
        // a target may be inside twoh of the centre (SPLINEQ's softened
        // branch), with a relative margin; the box gap is the one the opening
        // test measured
        const double reach = (r.soft + g.soft_max) * (1.0 + 1e-5);
        near = !(gap2 > reach * reach);
      }
      PROF_MARK(w, 1);
      {  // terminals go straight to the bucket's lists
        const unsigned lt = (1u << lane) - 1u;
        const bool pc = (cls == kClsQuad || cls == kClsMono);
        const unsigned m = __ballot_sync(kFull, pc);
        const int n = __popc(m);
        opens32 += n;  // internal children: accepted (P2C) here, opened below
        if (n && fits) {
          fits = make_room(n, rpc, pc0, L.pc_pool, L.cursor + 0, L.cap_pc, L.region, lane);
          if (fits && pc)
            L.pc_pool[rpc.cur + __popc(m & lt)] =
                node | (cls == kClsMono ? (int)0x80000000 : 0) | (near ? 0x40000000 : 0);
          if (fits) rpc.cur += (unsigned long long)n;
        }
        const bool pp = (cls == kClsP2P);
        const unsigned mp = __ballot_sync(kFull, pp);
        const int npp = __popc(mp);
        if (npp && fits) {
          fits = make_room(npp, rpp, pp0, L.pp_pool, L.cursor + 1, L.cap_pp, L.region, lane);
          if (fits && pp) L.pp_pool[rpp.cur + __popc(mp & lt)] = node;
          if (fits) rpp.cur += (unsigned long long)npp;
        }
      }
      {
        const bool op = (cls == kClsOpen);
        const unsigned m = __ballot_sync(kFull, op);
        opens32 += __popc(m);
        if (sp + __popc(m) > kWlStack) {
          ok = false;
          break;
        }
        if (op) w.stack[sp + __popc(m & ((1u << lane) - 1u))] = r.first_child;
        sp += __popc(m);
      }
      __syncwarp();
      PROF_MARK(w, 2);
      if (sp == 0) break;
      nexp = sp < 4 ? sp : 4;
      sp -= nexp;
      pop = sp;
    }
    if (!ok && lane == 0) atomicOr(P.status, kErrStack);
    if (!fits && lane == 0) atomicOr(P.status, kErrPool);
    const unsigned npc = (unsigned)(rpc.cur - pc0), npp = (unsigned)(rpp.cur - pp0);
    if (lane == 0) {
      const bool good = ok && fits;
      L.pc_start[lb] = (int64_t)pc0;
      L.pc_count[lb] = good ? (int32_t)npc : 0;
      L.pp_start[lb] = (int64_t)pp0;
      L.pp_count[lb] = good ? (int32_t)npp : 0;
    }
    max_len = max(max_len, max(npc, npp));
    c_pc += (unsigned long long)npc * (unsigned long long)ntot;
    c_open += opens32;
    if (P.bucket_work && lane == 0) {  // eval_p2p adds the P2P pairs
      unsigned long long wk = (unsigned long long)npc * (unsigned long long)ntot;
      if (P.accumulate) wk += P.bucket_work[b];
      P.bucket_work[b] = wk;
    }
    PROF_MARK(w, 4);
  }
  PROF_MARK(w, 5);
  PROF_FLUSH(w, 16);
  if (lane == 0) {
    atomicAdd(&P.counters[1], c_pc);
    atomicAdd(&P.counters[2], c_open);
    atomicMax(L.max_len, max_len);
  }
}

// ---------------------------------------------------------------- phase B
constexpr int kEvWarps = 4;
// CTAs per SM of eval_p2c (72 registers, no spills; 6 and 8 measured 0.2 and
// 0.3 ms slower at N = 2^24: more CTAs take shared memory from the L1 that
// holds the node records)
#ifndef PT_P2C_MINB
#define PT_P2C_MINB 7
#endif
// CTAs per SM of eval_p2p (72 registers; with the 256-bit leaf-record loads
// 7 measured 0.3 ms faster than 8 at 64 registers, which spills more)
#ifndef PT_P2P_MINB
#define PT_P2P_MINB 7
#endif

// Per-warp shared memory of eval_p2p ...
struct EvalWarp {
  BucketGeom geom;
  float4 st[6][32];            // staged source pairs px, pz, pr; rows 3-4 hold second-target sums
  int32_t ps0[kWlBuf];         // first particle of each leaf - its stream position
  float4 lof[kWlBuf];          // leaf offsets cm_leaf - cm_bucket (FP32)
  int32_t lsel[kWlBuf];        // leaves of the current kind in a block
  PROF_FIELDS
};

// ... and of eval_p2c (kept apart: shared memory taken from one kernel's
// CTAs is L1 lost to its node records)
struct EvalWarpC {
  BucketGeom geom;
  float4 st[5][32];            // staged node pairs, five rows (offset, mass, traceless moments)
  float4 ks[2][32];            // each lane's compensated sums and their compensations
  int32_t spec[kWlBuf];        // the chunk's near and monopole entries (scalar pass)
  PROF_FIELDS
};

// Per-lane target of a 32-target chunk, replicated over G lane groups (lanes
// past G * nt idle: a warp's loop runs as long as its target with the fewest
// lanes, so a ragged split would not finish sooner).  eval_p2p switches to
// two targets per lane (EvTarget2) where that needs fewer iterations.
struct EvTarget {
  int t, grp, G, nt;
  float tx, ty, tz, ts;
};

__device__ __forceinline__ EvTarget ev_target(const Particles& p, const BucketGeom& g, int t0, int nt, int lane) {
  EvTarget x;
  x.nt = nt;
  x.t = lane % nt;
  x.grp = lane / nt;
  x.G = 32 / nt;
  x.tx = x.ty = x.tz = x.ts = 0.f;
  if (x.grp < x.G) {
    const int i = t0 + x.t;
    x.tx = (float)(p.x[i] - g.cm[0]);
    x.ty = (float)(p.y[i] - g.cm[1]);
    x.tz = (float)(p.z[i] - g.cm[2]);
    x.ts = (float)p.soft[i];
  }
  return x;
}

struct Kahan4 {
  float s[4], c[4];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < 4; k++) s[k] = c[k] = 0.f;
  }
  __device__ __forceinline__ void add(int k, float v) {
    const float y = v - c[k];
    const float t = s[k] + y;
    c[k] = (t - s[k]) - y;
    s[k] = t;
  }
};

// Two targets per lane (P2P): lane l of group l / h holds targets 2 (l % h)
// and 2 (l % h) + 1 (h = ceil(nt / 2); t2 == nt when there is none), so each
// staged source meets two targets per packed instruction.
struct EvTarget2 {
  int t1, t2, grp, G, nt;
  float2 tx, ty, tz, ts;
};

// Two targets per lane wherever there are two: each staged source pair then
// meets four targets' worth of work per iteration, which halves the shared-
// memory loads and loop overhead per interaction (measured 1.7 ms faster at
// N = 2^24 than choosing it only where it takes fewer iterations).
__device__ __forceinline__ bool ev_two_targets(int nt) { return nt >= 2; }

__device__ __forceinline__ EvTarget2 ev_target2(const Particles& p, const BucketGeom& g, int t0, int nt, int lane) {
  EvTarget2 x;
  const int h = (nt + 1) >> 1;
  x.nt = nt;
  x.G = 32 / h;
  x.grp = lane / h;
  x.t1 = 2 * (lane % h);
  x.t2 = min(x.t1 + 1, nt);
  x.tx = x.ty = x.tz = x.ts = make_float2(0.f, 0.f);
  if (x.grp < x.G) {
    const int i1 = t0 + x.t1, i2 = t0 + min(x.t2, nt - 1);  // no second target: the first again
    x.tx = make_float2((float)(p.x[i1] - g.cm[0]), (float)(p.x[i2] - g.cm[0]));
    x.ty = make_float2((float)(p.y[i1] - g.cm[1]), (float)(p.y[i2] - g.cm[1]));
    x.tz = make_float2((float)(p.z[i1] - g.cm[2]), (float)(p.z[i2] - g.cm[2]));
    x.ts = make_float2((float)p.soft[i1], (float)p.soft[i2]);
  }
  return x;
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  const float y = v - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// The second target's compensated sums of a two-target lane live in rows 3
// and 4 of the staging area (P2P stages rows 0-2 only).
__device__ __forceinline__ void ev_two_zero(EvalWarp& w, int lane) {
  __syncwarp();  // earlier readers of the area (the last chunk's reduction) are done
  w.st[3][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
  w.st[4][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// ev_finish for two-target lanes (P2P: adds to ax, ay, az and pot_full).
__device__ __forceinline__ void ev_finish2(EvalWarp& w, const Kahan4& K, const EvTarget2& x, const TravParams& P,
                                           int t0, int lane) {
  const float4 s2 = w.st[3][lane], c2 = w.st[4][lane];
  double* red = reinterpret_cast<double*>(&w.st[0][0]);
  __syncwarp();
  if (x.grp < x.G) {
    const int b1 = 4 * (x.grp * x.nt + x.t1);
#pragma unroll
    for (int k = 0; k < 4; k++) red[b1 + k] = (double)K.s[k] - (double)K.c[k];
    if (x.t2 < x.nt) {
      const int b2 = 4 * (x.grp * x.nt + x.t2);
      red[b2 + 0] = (double)s2.x - (double)c2.x;
      red[b2 + 1] = (double)s2.y - (double)c2.y;
      red[b2 + 2] = (double)s2.z - (double)c2.z;
      red[b2 + 3] = (double)s2.w - (double)c2.w;
    }
  }
  __syncwarp();
  if (lane < x.nt) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int gg = 0; gg < x.G; gg++)
      for (int k = 0; k < 4; k++) v[k] += red[4 * (gg * x.nt + lane) + k];
    const int i = t0 + lane;
    P.p.ax[i] += v[0];
    P.p.ay[i] += v[1];
    P.p.az[i] += v[2];
    P.p.potf[i] += v[3];
  }
}

// Sum the G lane groups of each target and store or add the result.  P2C
// (p2c): pot_full gets every node's potential, pot the quadrupole node()
// terms only (the reference's potential: pmono, the monopole nodes' part, is
// left out); P2P adds to pot_full only (GravityVisitor::leaf applies none).
template <class W>
__device__ __forceinline__ void ev_finish(W& w, const Kahan4& K, float pmono, const EvTarget& x,
                                          const TravParams& P, int t0, int lane, bool p2c, bool store) {
  double* red = reinterpret_cast<double*>(&w.st[0][0]);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 4; k++) red[5 * lane + k] = (double)K.s[k] - (double)K.c[k];
  red[5 * lane + 4] = (double)pmono;
  __syncwarp();
  if (lane < x.nt) {
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int gg = 0; gg < x.G; gg++)
      for (int k = 0; k < 5; k++) v[k] += red[5 * (gg * x.nt + lane) + k];
    const int i = t0 + lane;
    if (store) {
      P.p.ax[i] = v[0];
      P.p.ay[i] = v[1];
      P.p.az[i] = v[2];
      P.p.pot[i] = p2c ? v[3] - v[4] : 0.0;
      P.p.potf[i] = v[3];
    } else {
      P.p.ax[i] += v[0];
      P.p.ay[i] += v[1];
      P.p.az[i] += v[2];
      if (p2c) P.p.pot[i] += v[3] - v[4];
      P.p.potf[i] += v[3];
    }
  }
  __syncwarp();
}

__device__ __forceinline__ bool next_bucket(const TravParams& P, int lane, int64_t& b, int& tnode) {
  const unsigned bi = grab_bucket(P.work, P.smq, lane);
  b = P.b_begin + (int64_t)bi;
  if (b >= P.b_end) return false;
  tnode = P.buckets[b];
  return true;
}

// FP32 offset of a node's centre of mass (plus the replica offset) from the
// bucket's, computed in FP64 as the walk computes it.

// 256-bit loads (sm_100): half a 64-byte walk record, or a whole 32-byte
// FP32 node record, with one instruction (the read-only path: these kernels
// never write the node arrays)
// (a 256-bit load needs a 32-byte aligned address: the arrays come from
// cudaMalloc, and their records are 64 and 32 bytes long)
static_assert(sizeof(WalkRec) == 64 && sizeof(QuadRecF) == 32, "records of 64 and 32 bytes");
__device__ __forceinline__ double4 ld_nc_d4(const void* p) {
  double4 v;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ void ld_nc_f8(const void* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

__device__ __forceinline__ float4 node_offset(const WalkRec* __restrict__ walk, int node, const TravParams& P,
                                              const BucketGeom& g) {
  const double4 c = ld_nc_d4(walk + node);  // cm x, y, z, orsq | reach
  return make_float4((float)((c.x + P.ox) - g.cm[0]), (float)((c.y + P.oy) - g.cm[1]),
                     (float)((c.z + P.oz) - g.cm[2]), 0.f);
}

// The FP32 node record (mass, soft, xx, xy), (xz, yy, yz, zz).
__device__ __forceinline__ void load_quadf(const QuadRecF* __restrict__ q, int node, float4& r0, float4& r1) {
  ld_nc_f8(q + node, r0, r1);
}

struct P2cTerm {
  float ax, ay, az, pf;
};

// One P2C term in scalar form for the rare nodes the packed loop leaves out:
// a node whose softening sphere may reach a target (SPLINEQ's softened
// branch, GravityVisitor::node, examples/GravityVisitor.h:184-224) or a
// monopole node (addGravity, :130-139: no second moments, never softened --
// it is given a NaN softening, so SPLINEQ takes its unsoftened branch).
__device__ __noinline__ P2cTerm ev_p2c_scalar(float ox, float oy, float oz, float M, float soft, float4 q0,
                                              float2 q1, float tx, float ty, float tz, float ts) {
  // q0 = (xx, xy, xz, yy), q1 = (yz, zz)
  const float rx = tx - ox, ry = ty - oy, rz = tz - oz;
  const float r2 = rx * rx + ry * ry + rz * rz;
  const float dir = rsqrtf(r2);
  float a, b, c, d;
  splineq_f32(dir, r2, soft + ts, a, b, c, d);
  const float qx = q0.x * rx + q0.y * ry + q0.z * rz;
  const float qy = q0.y * rx + q0.w * ry + q1.x * rz;
  const float qz = q0.z * rx + q1.x * ry + q1.y * rz;
  const float qir = 0.5f * (qx * rx + qy * ry + qz * rz);
  const float tr = 0.5f * (q0.x + q0.w + q1.y);
  const float qir3 = b * M + d * qir - c * tr;
  P2cTerm t;
  t.pf = -M * a - c * qir + b * tr;
  t.ax = -qir3 * rx + c * qx;
  t.ay = -qir3 * ry + c * qy;
  t.az = -qir3 * rz + c * qz;
  return t;
}

// The staged node pairs k = grp, grp + G, ... of one chunk against this
// lane's target (GravityVisitor::node, examples/GravityVisitor.h:184-224, in
// packed FP32).  Near and monopole nodes are staged as zero-mass padding and
// evaluated apart (ev_p2c_specials), so this loop has no branch.
//
// The moments are staged traceless, Qt = Q - (trace Q / 3) I.  With
// a = 1/r, b = a^3, c = 3 b a^2, d = 5 c a^2 the reference's unsoftened terms
// (qir = r.Q.r / 2, tr = trace Q / 2)
//   pot = -M a - c qir + b tr,  acc = -(b M + d qir - c tr) r + c Q r
// equal, since c r^2 = 3 b and d r^2 = 5 c,
//   pot = -M a - c qt,          acc = -(b M + d qt) r + c Qt r
// with qt = r.Qt.r / 2: the trace terms cancel exactly, which saves three of
// 37 operations per evaluation and one staged row.
__device__ __forceinline__ void ev_p2c_pairs(const EvalWarpC& w, const EvTarget& x, int npair, float2 ntx, float2 nty,
                                             float2 ntz, float2& ax2, float2& ay2, float2& az2, float2& pp2,
                                             float2& mm2) {
  const float2 mthree = make_float2(-3.f, -3.f), m25 = make_float2(-2.5f, -2.5f), half = make_float2(0.5f, 0.5f);
  const float4* sp = &w.st[0][x.grp];  // rows st[1..4] follow at +32 each
  for (int k = x.grp; k < npair; k += x.G, sp += x.G) {
    const float4 P0 = sp[0], P1 = sp[32];
    const float2 rx = __fadd2_rn(make_float2(P0.x, P0.y), ntx);  // r' = o - t = -r
    const float2 ry = __fadd2_rn(make_float2(P0.z, P0.w), nty);
    const float2 rz = __fadd2_rn(make_float2(P1.x, P1.y), ntz);
    float2 r2 = __fmul2_rn(rx, rx);
    r2 = __ffma2_rn(ry, ry, r2);
    r2 = __ffma2_rn(rz, rz, r2);
    const float4 P2 = sp[64], P3 = sp[96], P4 = sp[128];
    const float2 a = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 d2 = __fmul2_rn(a, a);
    const float2 bb = __fmul2_rn(a, d2);                       // b = 1/r^3
    const float2 nc = __fmul2_rn(__fmul2_rn(bb, d2), mthree);  // -c = -3/r^5
    const float2 xx = make_float2(P2.x, P2.y), xy = make_float2(P2.z, P2.w);
    const float2 xz = make_float2(P3.x, P3.y), yy = make_float2(P3.z, P3.w);
    const float2 yz = make_float2(P4.x, P4.y), zz = make_float2(P4.z, P4.w);
    const float2 qx = __ffma2_rn(xz, rz, __ffma2_rn(xy, ry, __fmul2_rn(xx, rx)));  // q' = Qt r' = -Qt r
    const float2 qy = __ffma2_rn(yz, rz, __ffma2_rn(yy, ry, __fmul2_rn(xy, rx)));
    const float2 qz = __ffma2_rn(zz, rz, __ffma2_rn(yz, ry, __fmul2_rn(xz, rx)));
    const float2 cq = __fmul2_rn(nc, __ffma2_rn(qz, rz, __ffma2_rn(qy, ry, __fmul2_rn(qx, rx))));  // -2 c qt
    const float2 M = make_float2(P1.z, P1.w);
    // A = b M + d qt = b M - (5 / 2) a^2 (-2 c qt); acc += A r' - c q'; pot += -c qt - M a
    const float2 A = __ffma2_rn(__fmul2_rn(d2, m25), cq, __fmul2_rn(bb, M));
    ax2 = __ffma2_rn(nc, qx, __ffma2_rn(A, rx, ax2));
    ay2 = __ffma2_rn(nc, qy, __ffma2_rn(A, ry, ay2));
    az2 = __ffma2_rn(nc, qz, __ffma2_rn(A, rz, az2));
    pp2 = __ffma2_rn(half, cq, pp2);
    mm2 = __ffma2_rn(M, a, mm2);
  }
}

// The chunk's near and monopole entries w.spec[0..ns), spread over the lane
// groups, in scalar form; a monopole node's potential also goes to pmono
// (left out of the reference's potential).
__device__ __forceinline__ void ev_p2c_specials(const EvalWarpC& w, const TravParams& P, const EvTarget& x, int ns,
                                                float2& ax2, float2& ay2, float2& az2, float2& pp2, float& pmono) {
  const float qnan = __int_as_float(0x7fc00000);
  for (int j = x.grp; j < ns; j += x.G) {
    const int e = w.spec[j];
    const int node = e & 0x3fffffff;
    const float4 o = node_offset(P.walk, node, P, w.geom);
    float4 r0, r1;  // (mass, soft, xx, xy), (xz, yy, yz, zz)
    load_quadf(P.quadf, node, r0, r1);
    const bool mono = e < 0;
    const float4 q0 = mono ? make_float4(0.f, 0.f, 0.f, 0.f) : make_float4(r0.z, r0.w, r1.x, r1.y);
    const float2 q1 = mono ? make_float2(0.f, 0.f) : make_float2(r1.z, r1.w);
    const P2cTerm t = ev_p2c_scalar(o.x, o.y, o.z, r0.x, mono ? qnan : r0.y, q0, q1, x.tx, x.ty, x.tz, x.ts);
    ax2.x += t.ax;
    ay2.x += t.ay;
    az2.x += t.az;
    pp2.x += t.pf;
    if (mono) pmono += t.pf;
  }
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kEvWarps * 32, kMinBlocks) eval_p2c(TravParams P, ListParams L,
                                                                     const Mom* __restrict__ mom) {
  __shared__ EvalWarpC warps[kEvWarps];
  EvalWarpC& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const float kPad = 1.0e10f;
  int64_t b;
  int tnode;
  PROF_START(w);
  while (next_bucket(P, lane, b, tnode)) {
    if (tnode < 0 || tnode >= P.nnodes) continue;
    const int64_t lb = b - P.b_begin;
    const int64_t start = L.pc_start[lb];
    const int count = L.pc_count[lb];
    if (count == 0 && P.accumulate) continue;  // nothing to add (the first walk stores, even zeros)
    __syncwarp();
    if (lane == 0) load_bucket_geom(mom, tnode, w.geom);
    __syncwarp();
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const EvTarget x = ev_target(P.p, w.geom, t0, nt, lane);
      const float2 ntx = make_float2(-x.tx, -x.tx), nty = make_float2(-x.ty, -x.ty), ntz = make_float2(-x.tz, -x.tz);
      // compensated sums in shared memory (added to once every four chunks)
      w.ks[0][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
      w.ks[1][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
      // plain packed sums over four chunks, then one compensated add
      float2 ax2 = make_float2(0.f, 0.f), ay2 = ax2, az2 = ax2, pp2 = ax2, mm2 = ax2;
      float pmono = 0.f;  // the monopole nodes' potential (left out of pot)
      // list entries of the coming chunk, loaded a chunk ahead so that only
      // the node records wait at staging time
      int en0 = (2 * lane < count) ? L.pc_pool[start + 2 * lane] : 0;
      int en1 = (2 * lane + 1 < count) ? L.pc_pool[start + 2 * lane + 1] : 0;
      PROF_MARK(w, 0);
      for (int cs = 0; cs < count; cs += 64) {
        const int ec[2] = {en0, en1};
        if (cs + 64 < count) {
          const int qn = cs + 64 + 2 * lane;
          en0 = (qn < count) ? L.pc_pool[start + qn] : 0;
          en1 = (qn + 1 < count) ? L.pc_pool[start + qn + 1] : 0;
        }
        // stage this lane's two nodes as a pair; near and monopole nodes
        // (bits 30 / 31) become zero-mass padding and go to the scalar list
        float4 o[2], r0[2], r1[2];
        bool spec[2] = {false, false};
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int q = cs + 2 * lane + h;
          o[h] = make_float4(kPad, kPad, kPad, 0.f);
          r0[h] = make_float4(0.f, 0.f, 0.f, 0.f);
          r1[h] = r0[h];
          if (q < count) {
            const int e = ec[h];
            spec[h] = (e & 0xc0000000) != 0;
            if (!spec[h]) {
              const int node = e & 0x3fffffff;
              o[h] = node_offset(P.walk, node, P, w.geom);
              load_quadf(P.quadf, node, r0[h], r1[h]);  // (mass, soft, xx, xy), (xz, yy, yz, zz)
            }
          }
        }
        const unsigned m0 = __ballot_sync(kFull, spec[0]), m1 = __ballot_sync(kFull, spec[1]);
        const int ns = __popc(m0) + __popc(m1);
        __syncwarp();
        if (spec[0] || spec[1]) {  // chunk order: by lane, then h
          const unsigned lt = (1u << lane) - 1u;
          const int at = __popc(m0 & lt) + __popc(m1 & lt);
          if (spec[0]) w.spec[at] = ec[0];
          if (spec[1]) w.spec[at + (spec[0] ? 1 : 0)] = ec[1];
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {  // traceless moments: xx, yy, zz less a third of the trace
          const float t3 = (r0[h].z + r1[h].y + r1[h].w) * (1.0f / 3.0f);
          r0[h].z -= t3;
          r1[h].y -= t3;
          r1[h].w -= t3;
        }
        w.st[0][lane] = make_float4(o[0].x, o[1].x, o[0].y, o[1].y);
        w.st[1][lane] = make_float4(o[0].z, o[1].z, r0[0].x, r0[1].x);
        w.st[2][lane] = make_float4(r0[0].z, r0[1].z, r0[0].w, r0[1].w);
        w.st[3][lane] = make_float4(r1[0].x, r1[1].x, r1[0].y, r1[1].y);
        w.st[4][lane] = make_float4(r1[0].z, r1[1].z, r1[0].w, r1[1].w);
        __syncwarp();
        const int npair = (min(64, count - cs) + 1) >> 1;
        PROF_MARK(w, 1);
        if (x.grp < x.G) {
          ev_p2c_pairs(w, x, npair, ntx, nty, ntz, ax2, ay2, az2, pp2, mm2);
          PROF_MARK(w, 2);
          if (ns) ev_p2c_specials(w, P, x, ns, ax2, ay2, az2, pp2, pmono);
          PROF_MARK(w, 3);
        }
        if (((cs >> 6) & 3) == 3 || cs + 64 >= count) {
          float4 ks = w.ks[0][lane], kc = w.ks[1][lane];
          kahan_add(ks.x, kc.x, ax2.x + ax2.y);
          kahan_add(ks.y, kc.y, ay2.x + ay2.y);
          kahan_add(ks.z, kc.z, az2.x + az2.y);
          kahan_add(ks.w, kc.w, (pp2.x + pp2.y) - (mm2.x + mm2.y));
          w.ks[0][lane] = ks;
          w.ks[1][lane] = kc;
          ax2 = ay2 = az2 = pp2 = mm2 = make_float2(0.f, 0.f);
        }
      }
      Kahan4 K;
      {
        const float4 ks = w.ks[0][lane], kc = w.ks[1][lane];
        K.s[0] = ks.x; K.s[1] = ks.y; K.s[2] = ks.z; K.s[3] = ks.w;
        K.c[0] = kc.x; K.c[1] = kc.y; K.c[2] = kc.z; K.c[3] = kc.w;
      }
      ev_finish(w, K, pmono, x, P, t0, lane, true, P.accumulate == 0);
      PROF_MARK(w, 4);
    }
  }
  PROF_MARK(w, 5);
  PROF_FLUSH(w, 0);
}

// eval_p2c with two targets per lane: each staged node meets the lane's two
// targets in one packed instruction, so a node is read from shared memory
// once for two evaluations.  The chunk's nodes are staged one per entry:
// na = (offset x, y, z, mass), nq = traceless (xx, xy, xz, yy), nr =
// traceless (yz, zz): 40 bytes per node instead of 40 bytes per evaluation.
struct EvalWarpC2 {
  BucketGeom geom;
  float4 na[64];
  float4 nq[64];
  float2 nr[64];
  float4 ks[4][32];  // compensated sums: target 1 (sum, compensation), target 2 (sum, compensation)
  int32_t spec[kWlBuf];
  PROF_FIELDS
};

// The chunk's nodes k = grp, grp + G, ... < nn against the lane's two
// targets (halves of every packed value); the same terms as ev_p2c_pairs.
__device__ __forceinline__ void ev_p2c_nodes2(const EvalWarpC2& w, const EvTarget2& x, int nn, float2 ntx,
                                              float2 nty, float2 ntz, float2& ax2, float2& ay2, float2& az2,
                                              float2& pp2, float2& mm2) {
  const float2 mthree = make_float2(-3.f, -3.f), m25 = make_float2(-2.5f, -2.5f), half = make_float2(0.5f, 0.5f);
  for (int k = x.grp; k < nn; k += x.G) {
    const float4 A = w.na[k];
    const float2 rx = __fadd2_rn(make_float2(A.x, A.x), ntx);  // r' = o - t = -r
    const float2 ry = __fadd2_rn(make_float2(A.y, A.y), nty);
    const float2 rz = __fadd2_rn(make_float2(A.z, A.z), ntz);
    float2 r2 = __fmul2_rn(rx, rx);
    r2 = __ffma2_rn(ry, ry, r2);
    r2 = __ffma2_rn(rz, rz, r2);
    const float4 Q = w.nq[k];
    const float2 Q2 = w.nr[k];
    const float2 a = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 d2 = __fmul2_rn(a, a);
    const float2 bb = __fmul2_rn(a, d2);
    const float2 nc = __fmul2_rn(__fmul2_rn(bb, d2), mthree);
    const float2 xx = make_float2(Q.x, Q.x), xy = make_float2(Q.y, Q.y), xz = make_float2(Q.z, Q.z);
    const float2 yy = make_float2(Q.w, Q.w), yz = make_float2(Q2.x, Q2.x), zz = make_float2(Q2.y, Q2.y);
    const float2 qx = __ffma2_rn(xz, rz, __ffma2_rn(xy, ry, __fmul2_rn(xx, rx)));
    const float2 qy = __ffma2_rn(yz, rz, __ffma2_rn(yy, ry, __fmul2_rn(xy, rx)));
    const float2 qz = __ffma2_rn(zz, rz, __ffma2_rn(yz, ry, __fmul2_rn(xz, rx)));
    const float2 cq = __fmul2_rn(nc, __ffma2_rn(qz, rz, __ffma2_rn(qy, ry, __fmul2_rn(qx, rx))));
    const float2 M = make_float2(A.w, A.w);
    const float2 AA = __ffma2_rn(__fmul2_rn(d2, m25), cq, __fmul2_rn(bb, M));
    ax2 = __ffma2_rn(nc, qx, __ffma2_rn(AA, rx, ax2));
    ay2 = __ffma2_rn(nc, qy, __ffma2_rn(AA, ry, ay2));
    az2 = __ffma2_rn(nc, qz, __ffma2_rn(AA, rz, az2));
    pp2 = __ffma2_rn(half, cq, pp2);
    mm2 = __ffma2_rn(M, a, mm2);
  }
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kEvWarps * 32, kMinBlocks) eval_p2c2(TravParams P, ListParams L,
                                                                      const Mom* __restrict__ mom) {
  __shared__ EvalWarpC2 warps[kEvWarps];
  EvalWarpC2& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const float kPad = 1.0e10f;
  const float qnan = __int_as_float(0x7fc00000);
  int64_t b;
  int tnode;
  PROF_START(w);
  while (next_bucket(P, lane, b, tnode)) {
    if (tnode < 0 || tnode >= P.nnodes) continue;
    const int64_t lb = b - P.b_begin;
    const int64_t start = L.pc_start[lb];
    const int count = L.pc_count[lb];
    if (count == 0 && P.accumulate) continue;  // nothing to add (the first walk stores, even zeros)
    __syncwarp();
    if (lane == 0) load_bucket_geom(mom, tnode, w.geom);
    __syncwarp();
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const EvTarget2 x = ev_target2(P.p, w.geom, t0, nt, lane);
      const bool two = x.t2 < nt;  // the lane has a second target
      const float2 ntx = make_float2(-x.tx.x, -x.tx.y), nty = make_float2(-x.ty.x, -x.ty.y),
                   ntz = make_float2(-x.tz.x, -x.tz.y);
#pragma unroll
      for (int r = 0; r < 4; r++) w.ks[r][lane] = make_float4(0.f, 0.f, 0.f, 0.f);
      float2 ax2 = make_float2(0.f, 0.f), ay2 = ax2, az2 = ax2, pp2 = ax2, mm2 = ax2;
      float2 pmono = make_float2(0.f, 0.f);  // the monopole nodes' potential (left out of pot)
      int en0 = (2 * lane < count) ? L.pc_pool[start + 2 * lane] : 0;
      int en1 = (2 * lane + 1 < count) ? L.pc_pool[start + 2 * lane + 1] : 0;
      PROF_MARK(w, 0);
      for (int cs = 0; cs < count; cs += 64) {
        const int ec[2] = {en0, en1};
        if (cs + 64 < count) {
          const int qn = cs + 64 + 2 * lane;
          en0 = (qn < count) ? L.pc_pool[start + qn] : 0;
          en1 = (qn + 1 < count) ? L.pc_pool[start + qn + 1] : 0;
        }
        float4 o[2], r0[2], r1[2];
        bool spec[2] = {false, false};
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int q = cs + 2 * lane + h;
          o[h] = make_float4(kPad, kPad, kPad, 0.f);
          r0[h] = make_float4(0.f, 0.f, 0.f, 0.f);
          r1[h] = r0[h];
          if (q < count) {
            const int e = ec[h];
            spec[h] = (e & 0xc0000000) != 0;
            if (!spec[h]) {
              const int node = e & 0x3fffffff;
              o[h] = node_offset(P.walk, node, P, w.geom);
              load_quadf(P.quadf, node, r0[h], r1[h]);  // (mass, soft, xx, xy), (xz, yy, yz, zz)
            }
          }
        }
        const unsigned m0 = __ballot_sync(kFull, spec[0]), m1 = __ballot_sync(kFull, spec[1]);
        const int ns = __popc(m0) + __popc(m1);
        __syncwarp();
        if (spec[0] || spec[1]) {  // chunk order: by lane, then h
          const unsigned lt = (1u << lane) - 1u;
          const int at = __popc(m0 & lt) + __popc(m1 & lt);
          if (spec[0]) w.spec[at] = ec[0];
          if (spec[1]) w.spec[at + (spec[0] ? 1 : 0)] = ec[1];
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {  // traceless moments: xx, yy, zz less a third of the trace
          const float t3 = (r0[h].z + r1[h].y + r1[h].w) * (1.0f / 3.0f);
          w.na[2 * lane + h] = make_float4(o[h].x, o[h].y, o[h].z, r0[h].x);
          w.nq[2 * lane + h] = make_float4(r0[h].z - t3, r0[h].w, r1[h].x, r1[h].y - t3);
          w.nr[2 * lane + h] = make_float2(r1[h].z, r1[h].w - t3);
        }
        __syncwarp();
        const int nn = min(64, count - cs);
        PROF_MARK(w, 1);
        if (x.grp < x.G) {
          ev_p2c_nodes2(w, x, nn, ntx, nty, ntz, ax2, ay2, az2, pp2, mm2);
          PROF_MARK(w, 2);
          for (int j = x.grp; j < ns; j += x.G) {  // near and monopole nodes, scalar
            const int e = w.spec[j];
            const int node = e & 0x3fffffff;
            const float4 of = node_offset(P.walk, node, P, w.geom);
            float4 q0r, q1r;
            load_quadf(P.quadf, node, q0r, q1r);
            const bool mono = e < 0;
            const float4 q0 = mono ? make_float4(0.f, 0.f, 0.f, 0.f) : make_float4(q0r.z, q0r.w, q1r.x, q1r.y);
            const float2 q1 = mono ? make_float2(0.f, 0.f) : make_float2(q1r.z, q1r.w);
            const float sf = mono ? qnan : q0r.y;
            const P2cTerm t = ev_p2c_scalar(of.x, of.y, of.z, q0r.x, sf, q0, q1, x.tx.x, x.ty.x, x.tz.x, x.ts.x);
            ax2.x += t.ax;
            ay2.x += t.ay;
            az2.x += t.az;
            pp2.x += t.pf;
            if (mono) pmono.x += t.pf;
            if (two) {
              const P2cTerm u = ev_p2c_scalar(of.x, of.y, of.z, q0r.x, sf, q0, q1, x.tx.y, x.ty.y, x.tz.y, x.ts.y);
              ax2.y += u.ax;
              ay2.y += u.ay;
              az2.y += u.az;
              pp2.y += u.pf;
              if (mono) pmono.y += u.pf;
            }
          }
          PROF_MARK(w, 3);
        }
        if (((cs >> 6) & 3) == 3 || cs + 64 >= count) {
          float4 s1 = w.ks[0][lane], c1 = w.ks[1][lane], s2 = w.ks[2][lane], c2 = w.ks[3][lane];
          kahan_add(s1.x, c1.x, ax2.x);
          kahan_add(s1.y, c1.y, ay2.x);
          kahan_add(s1.z, c1.z, az2.x);
          kahan_add(s1.w, c1.w, pp2.x - mm2.x);
          kahan_add(s2.x, c2.x, ax2.y);
          kahan_add(s2.y, c2.y, ay2.y);
          kahan_add(s2.z, c2.z, az2.y);
          kahan_add(s2.w, c2.w, pp2.y - mm2.y);
          w.ks[0][lane] = s1;
          w.ks[1][lane] = c1;
          w.ks[2][lane] = s2;
          w.ks[3][lane] = c2;
          ax2 = ay2 = az2 = pp2 = mm2 = make_float2(0.f, 0.f);
        }
      }
      // per target slot (group, target): ax, ay, az, pot_full, monopole part
      double* red = reinterpret_cast<double*>(&w.na[0]);  // na, nq, nr: 2560 bytes = 64 slots x 5
      const float4 s1 = w.ks[0][lane], c1 = w.ks[1][lane], s2 = w.ks[2][lane], c2 = w.ks[3][lane];
      __syncwarp();
      if (x.grp < x.G) {
        double* r1 = red + 5 * (x.grp * nt + x.t1);
        r1[0] = (double)s1.x - (double)c1.x;
        r1[1] = (double)s1.y - (double)c1.y;
        r1[2] = (double)s1.z - (double)c1.z;
        r1[3] = (double)s1.w - (double)c1.w;
        r1[4] = (double)pmono.x;
        if (two) {
          double* r2 = red + 5 * (x.grp * nt + x.t2);
          r2[0] = (double)s2.x - (double)c2.x;
          r2[1] = (double)s2.y - (double)c2.y;
          r2[2] = (double)s2.z - (double)c2.z;
          r2[3] = (double)s2.w - (double)c2.w;
          r2[4] = (double)pmono.y;
        }
      }
      __syncwarp();
      if (lane < nt) {
        double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int gg = 0; gg < x.G; gg++)
          for (int k = 0; k < 5; k++) v[k] += red[5 * (gg * nt + lane) + k];
        const int i = t0 + lane;
        if (P.accumulate == 0) {
          P.p.ax[i] = v[0];
          P.p.ay[i] = v[1];
          P.p.az[i] = v[2];
          P.p.pot[i] = v[3] - v[4];
          P.p.potf[i] = v[3];
        } else {
          P.p.ax[i] += v[0];
          P.p.ay[i] += v[1];
          P.p.az[i] += v[2];
          P.p.pot[i] += v[3] - v[4];
          P.p.potf[i] += v[3];
        }
      }
      __syncwarp();  // red is the next chunk's staging area
      PROF_MARK(w, 4);
    }
  }
  PROF_MARK(w, 5);
  PROF_FLUSH(w, 0);
}

// One source of a near leaf: Newtonian beyond the softening reach, the spline
// inside it, nothing for the particle itself (r2 == 0).  pp sums +m a.
__device__ __forceinline__ void ev_near_source(float m, float dx, float dy, float dz, float r2, float reach2,
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

// Leaf of chunk positions 2 lane and 2 lane + 1 (chunk start cs): the leaf
// covering position cs plus the leaves that start in (cs, q] -- one bit per
// start position, OR-reduced over the warp, counted with popc.  preA / preB =
// stream position of the lane's leaves lane and lane + 32.  Warp-uniform.
__device__ __forceinline__ void chunk_leaves(int cs, int preA, int preB, int lane, int& lo, int& lo1) {
  unsigned long long bits = 0ull;
  const int pa = preA - cs, pb = preB - cs;
  if (pa > 0 && pa < 64) bits |= 1ull << pa;
  if (pb > 0 && pb < 64) bits |= 1ull << pb;
  const unsigned long long starts =
      ((unsigned long long)__reduce_or_sync(kFull, (unsigned)(bits >> 32)) << 32) |
      __reduce_or_sync(kFull, (unsigned)bits);
  const int b0 = __popc(__ballot_sync(kFull, preA <= cs)) + __popc(__ballot_sync(kFull, preB <= cs)) - 1;
  lo = b0 + __popcll(starts & ((2ull << (2 * lane)) - 1ull));
  lo1 = lo + (int)((starts >> (2 * lane + 1)) & 1ull);
}


// P2P of the selected leaves w.lsel[0..nleaves) (GravityVisitor::leaf,
// examples/GravityVisitor.h:144-160, in FP32): their sources are staged 64
// per chunk as 32 interleaved pairs px = (x_a, x_b, y_a, y_b), pz = (z_a,
// z_b, m_a, m_b), relative to the bucket, and evaluated with packed FP32.
template <bool kFar, bool kTwo, class Tgt>
__device__ __forceinline__ void ev_p2p_leaves(EvalWarp& w, int base, int nleaves, const TravParams& P,
                                              const Tgt& x, int lane, Kahan4& K) {
  int s0a = 0, s0b = 0, na = 0, nb = 0;
  // the block pass left each leaf's first particle in ps0, its particle
  // count in lsel and its offset in lof, from index base on
  if (lane < nleaves) {
    s0a = w.ps0[base + lane];
    na = w.lsel[base + lane];
  }
  if (lane + 32 < nleaves) {
    s0b = w.ps0[base + lane + 32];
    nb = w.lsel[base + lane + 32];
  }
  int inca = na, incb = nb;
  for (int o = 1; o < 32; o <<= 1) {
    const int ya = __shfl_up_sync(kFull, inca, o), yb = __shfl_up_sync(kFull, incb, o);
    if (lane >= o) {
      inca += ya;
      incb += yb;
    }
  }
  const int tota = __shfl_sync(kFull, inca, 31);
  const int total = tota + __shfl_sync(kFull, incb, 31);
  // stream position of each leaf's first source, in registers (past the
  // block: never reached); ps0 becomes source index - stream position
  const int preA = (lane < nleaves) ? inca - na : INT_MAX;
  const int preB = (lane + 32 < nleaves) ? tota + incb - nb : INT_MAX;
  if (lane < nleaves) w.ps0[base + lane] = s0a - preA;
  if (lane + 32 < nleaves) w.ps0[base + lane + 32] = s0b - preB;
  // a leaf node always holds a particle: two leaves never start together
  if (__any_sync(kFull, (lane < nleaves && na == 0) || (lane + 32 < nleaves && nb == 0)) && lane == 0)
    atomicOr(P.status, kErrCapacity);
  __syncwarp();
  PROF_MARK(w, 1);
  const float kPadPos = 1.0e10f;
  const float gs = (float)w.geom.soft_max;
  float2 ntx, nty, ntz;
  if constexpr (kTwo) {
    ntx = make_float2(-x.tx.x, -x.tx.y);
    nty = make_float2(-x.ty.x, -x.ty.y);
    ntz = make_float2(-x.tz.x, -x.tz.y);
  } else {
    ntx = make_float2(-x.tx, -x.tx);
    nty = make_float2(-x.ty, -x.ty);
    ntz = make_float2(-x.tz, -x.tz);
  }
  // plain packed sums over the block's chunks, one compensated add at its end
  float2 ax2 = make_float2(0.f, 0.f), ay2 = ax2, az2 = ax2, pp2 = ax2;  // pp2 sums +m/r
  for (int cs = 0; cs < total; cs += 64) {
    {  // stage this lane's two sources
      const int q0 = cs + 2 * lane;
      int lo, lo1;
      chunk_leaves(cs, preA, preB, lane, lo, lo1);
      float4 ra = make_float4(kPadPos, kPadPos, kPadPos, 0.f), rb = ra;
      float4 oa = make_float4(0.f, 0.f, 0.f, 0.f), ob = oa;
      float sa = 0.f, sb = 0.f;
      if (q0 < total) {
        oa = w.lof[base + lo];
        const int j = w.ps0[base + lo] + q0;
        ra = P.srcf[j];
        if (!kFar) sa = P.softf[j];
      }
      if (q0 + 1 < total) {
        ob = w.lof[base + lo1];
        const int j = w.ps0[base + lo1] + q0 + 1;
        rb = P.srcf[j];
        if (!kFar) sb = P.softf[j];
      }
      __syncwarp();
      w.st[0][lane] = make_float4(ra.x + oa.x, rb.x + ob.x, ra.y + oa.y, rb.y + ob.y);
      w.st[1][lane] = make_float4(ra.z + oa.z, rb.z + ob.z, ra.w, rb.w);
      if (!kFar) {
        const float qa = sa + gs, qb = sb + gs;
        // a padded source (zero mass) takes the Newtonian branch
        w.st[2][lane] = make_float4(ra.w != 0.f ? qa * qa : -1.f, rb.w != 0.f ? qb * qb : -1.f, sa, sb);
      }
      __syncwarp();
    }
    const int np = (min(64, total - cs) + 1) >> 1;
    PROF_MARK(w, 2);
    if constexpr (kTwo) {
      if (x.grp < x.G) {
        const float4* sp = &w.st[0][x.grp];
        for (int k = x.grp; k < np; k += x.G, sp += x.G) {
          const float4 X = sp[0], Z = sp[32];
          float4 R = make_float4(0.f, 0.f, 0.f, 0.f);
          if (!kFar) R = sp[64];
#pragma unroll
          for (int h = 0; h < 2; h++) {  // source a, then source b, against both targets
            const float sx = h ? X.y : X.x, sy = h ? X.w : X.z, sz = h ? Z.y : Z.x, sm = h ? Z.w : Z.z;
            const float2 dx = __fadd2_rn(make_float2(sx, sx), ntx);
            const float2 dy = __fadd2_rn(make_float2(sy, sy), nty);
            const float2 dz = __fadd2_rn(make_float2(sz, sz), ntz);
            float2 r2 = __fmul2_rn(dx, dx);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            const float reach2 = h ? R.y : R.x;
            if (kFar || ((r2.x > reach2) && (r2.y > reach2))) {
              const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
              const float2 mr = __fmul2_rn(make_float2(sm, sm), ri);
              const float2 mr3 = __fmul2_rn(mr, __fmul2_rn(ri, ri));
              ax2 = __ffma2_rn(dx, mr3, ax2);
              ay2 = __ffma2_rn(dy, mr3, ay2);
              az2 = __ffma2_rn(dz, mr3, az2);
              pp2 = __fadd2_rn(pp2, mr);
            } else {
              const float ss = h ? R.w : R.z;
              ev_near_source(sm, dx.x, dy.x, dz.x, r2.x, reach2, ss, x.ts.x, ax2.x, ay2.x, az2.x, pp2.x);
              ev_near_source(sm, dx.y, dy.y, dz.y, r2.y, reach2, ss, x.ts.y, ax2.y, ay2.y, az2.y, pp2.y);
            }
          }
        }
      }
    } else {
    if (x.grp < x.G) {
      const float4* sp = &w.st[0][x.grp];  // rows st[1], st[2] follow at +32, +64
      for (int k = x.grp; k < np; k += x.G, sp += x.G) {
        const float4 X = sp[0], Z = sp[32];
        const float2 dx = __fadd2_rn(make_float2(X.x, X.y), ntx);
        const float2 dy = __fadd2_rn(make_float2(X.z, X.w), nty);
        const float2 dz = __fadd2_rn(make_float2(Z.x, Z.y), ntz);
        float2 r2 = __fmul2_rn(dx, dx);
        r2 = __ffma2_rn(dy, dy, r2);
        r2 = __ffma2_rn(dz, dz, r2);
        bool fast = true;
        float4 R = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!kFar) {
          R = sp[64];
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
          ev_near_source(Z.z, dx.x, dy.x, dz.x, r2.x, R.x, R.z, x.ts, ax2.x, ay2.x, az2.x, pp2.x);
          ev_near_source(Z.w, dx.y, dy.y, dz.y, r2.y, R.y, R.w, x.ts, ax2.y, ay2.y, az2.y, pp2.y);
        }
      }
    }
    }
    PROF_MARK(w, 3);
  }
  if constexpr (kTwo) {
    K.add(0, ax2.x);
    K.add(1, ay2.x);
    K.add(2, az2.x);
    K.add(3, -pp2.x);
    float4 s2 = w.st[3][lane], c2 = w.st[4][lane];
    kahan_add(s2.x, c2.x, ax2.y);
    kahan_add(s2.y, c2.y, ay2.y);
    kahan_add(s2.z, c2.z, az2.y);
    kahan_add(s2.w, c2.w, -pp2.y);
    w.st[3][lane] = s2;
    w.st[4][lane] = c2;
  } else {
    K.add(0, ax2.x + ax2.y);
    K.add(1, ay2.x + ay2.y);
    K.add(2, az2.x + az2.y);
    K.add(3, -(pp2.x + pp2.y));
  }
  __syncwarp();
}

// The bucket's P2P list in blocks of 64 entries, each leaf record read once:
// the near test (p2p_leaf_near's, on the whole record read with two 256-bit
// loads), the particle range and the FP32 offset go to shared memory with the
// far leaves first, and the far and near leaves are then evaluated from there
// (a separate marking pass over the list read every record twice: 0.6 ms at
// N = 2^24).  Returns the source particles of the listed leaves, as the
// reference counts P2P work (n_src * n_tgt per leaf(), src/Traverser.h:27).
template <bool kTwo, class Tgt>
__device__ __forceinline__ unsigned long long ev_p2p_blocks(EvalWarp& w, const TravParams& P,
                                                                  const ListParams& L, const Tgt& x, int64_t start,
                                                                  int count, int lane, Kahan4& K) {
  unsigned long long nsrc = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int blk = 0; blk < count; blk += 64) {
    bool v[2], nr[2];
    int ps[2], pc[2];
    float4 of[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int q = blk + lane + 32 * h;
      v[h] = q < count;
      nr[h] = false;
      ps[h] = pc[h] = 0;
      of[h] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (v[h]) {
        const int e = L.pp_pool[start + q] & 0x7fffffff;
        const double4 c = ld_nc_d4(P.walk + e);  // cm x, y, z, reach
        float4 a, b;                             // soft_max, first_child, type, count, pstart, pcount, pad
        ld_nc_f8(reinterpret_cast<const char*>(P.walk + e) + 32, a, b);
        ps[h] = __float_as_int(b.y);
        pc[h] = __float_as_int(b.z);
        const double smax = __hiloint2double(__float_as_int(a.y), __float_as_int(a.x));
        const double cx = __dadd_rn(c.x, P.ox), cy = __dadd_rn(c.y, P.oy), cz = __dadd_rn(c.z, P.oz);
        const double gap2 = box_gap2_exact(w.geom.lo, w.geom.hi, cx, cy, cz);
        const double reach = c.w + smax + w.geom.soft_max;
        nr[h] = !(gap2 > reach * reach);
        of[h] = make_float4((float)((c.x + P.ox) - w.geom.cm[0]), (float)((c.y + P.oy) - w.geom.cm[1]),
                            (float)((c.z + P.oz) - w.geom.cm[2]), 0.f);
      }
    }
    nsrc += __reduce_add_sync(kFull, (unsigned)(pc[0] + pc[1]));
    const unsigned f0 = __ballot_sync(kFull, v[0] && !nr[0]), f1 = __ballot_sync(kFull, v[1] && !nr[1]);
    const unsigned n0 = __ballot_sync(kFull, v[0] && nr[0]), n1 = __ballot_sync(kFull, v[1] && nr[1]);
    const int nf = __popc(f0) + __popc(f1), nn = __popc(n0) + __popc(n1);
    __syncwarp();  // the previous block's readers of lsel / ps0 / lof are done
#pragma unroll
    for (int h = 0; h < 2; h++) {
      if (v[h]) {
        const int pos = nr[h] ? nf + (h ? __popc(n0) + __popc(n1 & lt) : __popc(n0 & lt))
                              : (h ? __popc(f0) + __popc(f1 & lt) : __popc(f0 & lt));
        w.ps0[pos] = ps[h];
        w.lsel[pos] = pc[h];
        w.lof[pos] = of[h];
      }
    }
    __syncwarp();
    if (nf) ev_p2p_leaves<true, kTwo>(w, 0, nf, P, x, lane, K);
    if (nn) ev_p2p_leaves<false, kTwo>(w, nf, nn, P, x, lane, K);
  }
  return nsrc;
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kEvWarps * 32, kMinBlocks) eval_p2p(TravParams P, ListParams L,
                                                                     const Mom* __restrict__ mom) {
  __shared__ EvalWarp warps[kEvWarps];
  EvalWarp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  unsigned long long c_pp = 0;
  int64_t b;
  int tnode;
  PROF_START(w);
  while (next_bucket(P, lane, b, tnode)) {
    if (tnode < 0 || tnode >= P.nnodes) continue;
    const int64_t lb = b - P.b_begin;
    const int64_t start = L.pp_start[lb];
    const int count = L.pp_count[lb];
    if (count == 0) continue;  // P2P only adds (the outer replica walks leave most lists empty)
    __syncwarp();
    if (lane == 0) load_bucket_geom(mom, tnode, w.geom);
    __syncwarp();
    const int tbase = P.walk[tnode].pstart, ntot = P.walk[tnode].pcount;
    unsigned long long nsrc = 0;
    PROF_MARK(w, 0);
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      if (ev_two_targets(nt)) {
        const EvTarget2 x = ev_target2(P.p, w.geom, t0, nt, lane);
        ev_two_zero(w, lane);
        Kahan4 K;
        K.zero();
        nsrc = ev_p2p_blocks<true>(w, P, L, x, start, count, lane, K);
        ev_finish2(w, K, x, P, t0, lane);
        PROF_MARK(w, 4);
        continue;
      }
      const EvTarget x = ev_target(P.p, w.geom, t0, nt, lane);
      Kahan4 K;
      K.zero();
      nsrc = ev_p2p_blocks<false>(w, P, L, x, start, count, lane, K);
      ev_finish(w, K, 0.f, x, P, t0, lane, false, false);
      PROF_MARK(w, 4);
    }
    // P2P pairs as the reference counts them (n_src * n_tgt per leaf(),
    // src/Traverser.h:27); the walk wrote the bucket's P2C work before
    c_pp += nsrc * (unsigned long long)ntot;
    if (P.bucket_work && lane == 0) P.bucket_work[b] += nsrc * (unsigned long long)ntot;
  }
  PROF_MARK(w, 5);
  PROF_FLUSH(w, 8);
  if (lane == 0) atomicAdd(&P.counters[0], c_pp);
}

#if PT_PROF
extern "C" int pt_debug_prof(unsigned long long* out) {
  if (cudaMemcpyFromSymbol(out, g_prof, sizeof(g_prof)) != cudaSuccess) return -1;
  unsigned long long z[32] = {};
  return cudaMemcpyToSymbol(g_prof, z, sizeof(z)) == cudaSuccess ? 0 : -1;
}
#endif

// ---------------------------------------------------------------- launchers
int walk_lists_grid(int sms) { return sms * PT_WALK_MINB; }  // the CTAs resident

void launch_walk_lists(const TravParams& P, const ListParams& L, const Mom* mom, int grid, cudaStream_t st) {
  note_launch();
  if (P.ox == 0.0 && P.oy == 0.0 && P.oz == 0.0) walk_lists<false><<<grid, kWlWarps * 32, 0, st>>>(P, L, mom);
  else walk_lists<true><<<grid, kWlWarps * 32, 0, st>>>(P, L, mom);
}
void launch_eval_lists(const TravParams& P, const ListParams& L, const Mom* mom, int grid, cudaStream_t st,
                       unsigned* work2) {
  TravParams Q = P;
  Q.work = work2;
  if (P.smq) Q.smq = P.smq + 256;  // P2P's queues follow P2C's
  note_launch();
  // the replica walks after the first (periodic passes) leave short P2C
  // lists, where the one-target kernel's smaller per-bucket work measured
  // faster (256^3 lattice pass 212 against 220 ms); the first walk and every
  // non-periodic pass take the two-target kernel (Plummer N = 2^24: 3.5 ms
  // faster)
  if (P.accumulate) eval_p2c<PT_P2C_MINB><<<grid, kEvWarps * 32, 0, st>>>(P, L, mom);
  else eval_p2c2<PT_P2C_MINB><<<grid, kEvWarps * 32, 0, st>>>(P, L, mom);
  note_launch();
  eval_p2p<PT_P2P_MINB><<<grid, kEvWarps * 32, 0, st>>>(Q, L, mom);
}

}  // namespace pt
