// k_sph.cu -- the SPH example's density pass on the gravity tree: k = 32
// nearest neighbours of every particle (DensityVisitor, examples/
// DensityVisitor.h, walked with startUpAndDown, examples/SPH.C:77-86) and the
// M4-kernel density (DensityFn, examples/SPH.C:11-37; kernelM4,
// examples/SPHUtils.h:20-26).  FP64, compiled with -fmad=false so that
// d2 = dx*dx + dy*dy + dz*dz (dx = x_i - x_j) is the reference's value bit for
// bit; the neighbour set is the exact k nearest (the particle itself
// included), which the reference's conservative open() also yields.
//
// One warp per bucket; each of its targets keeps its current 32 best
// (d2, particle) as a list sorted ascending across the 32 lanes (lane e holds
// entry e), in a per-warp global scratch (coalesced, L1-resident).  Candidates
// come in batches of 32 (one per lane): a ballot against the target's 32nd
// entry discards a batch that cannot improve the list; otherwise the passing
// candidates are inserted (a few) or bitonic-sorted and merged (many).  Ties
// are broken by particle index, so the list is the k smallest (d2, index).
//   1. The lists start from a window of 64 particles around the bucket in key
//      order (spatially close), which bounds every target's ball.
//   2. A depth-first walk from the root visits a node if some target's ball
//      reaches its box (DensityVisitor::open with Space::intersect's <=),
//      children pushed far to near, and buffers the leaves it reaches; the
//      buffer is flushed (its particles batched against every target) when
//      full and at the end, and each flush shrinks the balls that later
//      visits test.
//   3. DensityFn: ball^2 = the 32nd d2, density summed over the list.
// The pressure pass that follows (sph_pressure_kernel) restates ForceFn
// (examples/SPH.C:39-64) and doSPHCalc (examples/SPHUtils.h:64-133): one warp
// per particle, lane e = its e-th neighbour from the density pass.  The divv
// corrector and the particle's own pressure acceleration and PdV work are warp
// sums; the opposite reaction on each neighbour (ThreadStateHolder's opposing
// effects, applied after the pass in the reference) is an FP64 atomic add, so
// its summation order is not fixed.
#include <math_constants.h>

#include "pt_internal.cuh"
#include "pt_walk.cuh"

namespace pt {

constexpr int kSphK = 32;
constexpr int kKnnWarps = 4;
constexpr int kKnnStack = 640;   // pending frames: 4 popped per step, <= 32 pushed
constexpr int kKnnLeaves = 128;  // leaves buffered between flushes
constexpr int kKnnChunk = 128;   // candidates staged per pass over the targets
constexpr int kKnnNone = 0x7fffffff;

struct KnnWarp {
  double cx[kKnnChunk], cy[kKnnChunk], cz[kKnnChunk];  // staged candidates
  int32_t ci[kKnnChunk];
  double tx[32], ty[32], tz[32];  // the chunk's targets
  double kd[32];                  // each target's list's last entry
  int32_t ki[32];
  int32_t stack[kKnnStack];
  int32_t leaf[kKnnLeaves];
};

__device__ __forceinline__ double box_d2(const double lo[3], const double hi[3], double x, double y, double z) {
  double d = 0.0, t;
  t = (x < lo[0]) ? __dadd_rn(lo[0], -x) : ((x > hi[0]) ? __dadd_rn(x, -hi[0]) : 0.0);
  d = __dadd_rn(d, __dmul_rn(t, t));
  t = (y < lo[1]) ? __dadd_rn(lo[1], -y) : ((y > hi[1]) ? __dadd_rn(y, -hi[1]) : 0.0);
  d = __dadd_rn(d, __dmul_rn(t, t));
  t = (z < lo[2]) ? __dadd_rn(lo[2], -z) : ((z > hi[2]) ? __dadd_rn(z, -hi[2]) : 0.0);
  d = __dadd_rn(d, __dmul_rn(t, t));
  return d;
}

// kernelM4 (examples/SPHUtils.h:20-26), scaled: (pi h^3) W for ar2 = (r/h)^2.
__device__ __forceinline__ double kernel_m4(double ar2) {
  double ak = 2.0 - sqrt(ar2);
  if (ar2 < 1.0) ak = (1.0 - 0.75 * ak * ar2);
  else ak = 0.25 * ak * ak * ak;
  return ak;
}

// (d, i) before (e, j): smaller d2, then smaller index.
__device__ __forceinline__ bool knn_before(double d, int i, double e, int j) { return d < e || (d == e && i < j); }

// One compare-exchange stage across lanes lane and lane ^ j; the lower lane of
// the pair keeps the smaller element when up, the larger otherwise.
__device__ __forceinline__ void knn_stage(double& d, int& i, int j, bool up, int lane) {
  const double pd = __shfl_xor_sync(kFull, d, j);
  const int pi = __shfl_xor_sync(kFull, i, j);
  const bool keep_min = (((lane & j) == 0) == up);
  const bool pb = knn_before(pd, pi, d, i);
  if (keep_min ? pb : (!pb && (pd != d || pi != i))) {
    d = pd;
    i = pi;
  }
}

// Sort the 32 lanes' (d, i) ascending (bitonic network).
__device__ __forceinline__ void knn_sort32(double& d, int& i, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) knn_stage(d, i, j, (lane & k) == 0 || k == 32, lane);
}

// List (ascending across lanes) <- the 32 smallest of list and batch
// (ascending): the element-wise minimum with the reversed batch is bitonic and
// holds them; one bitonic merge sorts it.
__device__ __forceinline__ void knn_merge(double& ld, int& li, double bd, int bi, int lane) {
  const double rd = __shfl_sync(kFull, bd, 31 - lane);
  const int ri = __shfl_sync(kFull, bi, 31 - lane);
  if (knn_before(rd, ri, ld, li)) {
    ld = rd;
    li = ri;
  }
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) knn_stage(ld, li, j, true, lane);
}

// Insert one candidate (cd, ci), known to beat the list's last entry.
__device__ __forceinline__ void knn_insert(double& ld, int& li, double cd, int ci, int lane) {
  const int pos = __popc(__ballot_sync(kFull, knn_before(ld, li, cd, ci)));  // entries that stay ahead
  const double ud = __shfl_up_sync(kFull, ld, 1);
  const int ui = __shfl_up_sync(kFull, li, 1);
  if (lane == pos) {
    ld = cd;
    li = ci;
  } else if (lane > pos) {
    ld = ud;
    li = ui;
  }
}

// The cnt staged candidates against every target of the chunk (nt of them),
// target by target: a target's list (global scratch, lane e = entry e) is
// loaded once, on the first batch of 32 that can improve it.
__device__ __forceinline__ void knn_chunk(KnnWarp& w, int nt, int cnt, double* __restrict__ Ld,
                                          int32_t* __restrict__ Li, int lane) {
  __syncwarp();
  for (int t = 0; t < nt; t++) {
    const double xt = w.tx[t], yt = w.ty[t], zt = w.tz[t];
    double kd = w.kd[t];
    int ki = w.ki[t];
    bool loaded = false;
    double ld = CUDART_INF;
    int li = kKnnNone;
    for (int b = 0; b < cnt; b += 32) {
      const int c = b + lane;
      const int j = (c < cnt) ? w.ci[c] : -1;
      double d2 = CUDART_INF;
      if (j >= 0) {
        const double dx = __dadd_rn(xt, -w.cx[c]), dy = __dadd_rn(yt, -w.cy[c]), dz = __dadd_rn(zt, -w.cz[c]);
        d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      }
      const bool pass = j >= 0 && knn_before(d2, j, kd, ki);
      const unsigned m = __ballot_sync(kFull, pass);
      if (m == 0u) continue;
      if (!loaded) {
        ld = Ld[t * 32 + lane];
        li = Li[t * 32 + lane];
        loaded = true;
      }
      if (__popc(m) <= 12) {
        unsigned r = m;
        while (r) {
          const int src = __ffs(r) - 1;
          r &= r - 1u;
          const double cd = __shfl_sync(kFull, d2, src);
          const int cj = __shfl_sync(kFull, j, src);
          // an earlier insertion of this batch may have raised the bar past it
          if (knn_before(cd, cj, kd, ki)) {
            knn_insert(ld, li, cd, cj, lane);
            kd = __shfl_sync(kFull, ld, 31);
            ki = __shfl_sync(kFull, li, 31);
          }
        }
      } else {
        double cd = pass ? d2 : CUDART_INF;
        int cj = pass ? j : kKnnNone;
        knn_sort32(cd, cj, lane);
        knn_merge(ld, li, cd, cj, lane);
        kd = __shfl_sync(kFull, ld, 31);
        ki = __shfl_sync(kFull, li, 31);
      }
    }
    if (loaded) {
      Ld[t * 32 + lane] = ld;
      Li[t * 32 + lane] = li;
      if (lane == 0) {
        w.kd[t] = kd;
        w.ki[t] = ki;
      }
    }
  }
  __syncwarp();
}

// Stage candidate j (or none) in slot c.
__device__ __forceinline__ void knn_stage_candidate(KnnWarp& w, const Particles& p, int c, int j) {
  w.ci[c] = j;
  if (j >= 0) {
    w.cx[c] = p.x[j];
    w.cy[c] = p.y[j];
    w.cz[c] = p.z[j];
  }
}

// The buffered leaves' particles, minus the window [w0, w1), staged
// kKnnChunk at a time.  (Sorting each flush's leaves by distance first
// measured slower: the sort costs more than the merges it saves.)
__device__ __forceinline__ void knn_flush(const Particles& p, const WalkRec* __restrict__ walk, KnnWarp& w, int nt,
                                          int nleaf, int w0, int w1, double* Ld, int32_t* Li, int lane) {
  int fill = 0;
  for (int l = 0; l < nleaf; l++) {
    const int nd = w.leaf[l];
    const int s0 = walk[nd].pstart, sn = walk[nd].pcount;
    for (int base = 0; base < sn;) {
      const int take = min(min(sn - base, 32), kKnnChunk - fill);
      __syncwarp();
      if (lane < take) {
        const int j = s0 + base + lane;
        knn_stage_candidate(w, p, fill + lane, (j >= w0 && j < w1) ? -1 : j);
      }
      fill += take;
      base += take;
      if (fill == kKnnChunk) {
        knn_chunk(w, nt, fill, Ld, Li, lane);
        fill = 0;
      }
    }
  }
  if (fill > 0) knn_chunk(w, nt, fill, Ld, Li, lane);
}

// Squared gap between two boxes (0 if they overlap).
__device__ __forceinline__ double box_box_gap2(const double alo[3], const double ahi[3], const double blo[3],
                                               const double bhi[3]) {
  double d = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double g = fmax(fmax(alo[k] - bhi[k], blo[k] - ahi[k]), 0.0);
    d += g * g;
  }
  return d;
}

// The largest ball^2 (last list entry) over the chunk's targets.
__device__ __forceinline__ double knn_rmax2(const KnnWarp& w, int lane) {
  double r = w.kd[lane];  // -1 in the slots of absent targets
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(kFull, r, o));
  return r;
}

__global__ void __launch_bounds__(kKnnWarps * 32, 7) sph_density_kernel(Particles p, int64_t n,
                                                                        const Mom* __restrict__ mom,
                                                                        const WalkRec* __restrict__ walk,
                                                                        const int32_t* __restrict__ buckets,
                                                                        int64_t nbuckets, int64_t nnodes,
                                                                        double* __restrict__ density,
                                                                        double* __restrict__ ballsq,
                                                                        int32_t* __restrict__ nbr,
                                                                        double* __restrict__ nd2, double* lists_d,
                                                                        int32_t* lists_i, unsigned* work,
                                                                        unsigned* status) {
  __shared__ KnnWarp warps[kKnnWarps];
  KnnWarp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int64_t slot = (int64_t)blockIdx.x * kKnnWarps + (threadIdx.x >> 5);
  double* Ld = lists_d + slot * 1024;
  int32_t* Li = lists_i + slot * 1024;
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(work, 1u);
    bi = __shfl_sync(kFull, bi, 0);
    if ((int64_t)bi >= nbuckets) break;
    const int tnode = buckets[bi];
    if (tnode < 0 || tnode >= nnodes) {
      if (lane == 0) atomicOr(status, kErrCapacity);
      continue;
    }
    const int tbase = walk[tnode].pstart, ntot = walk[tnode].pcount;
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const bool act = lane < nt;
      double x = 0.0, y = 0.0, z = 0.0;
      if (act) {
        x = p.x[t0 + lane];
        y = p.y[t0 + lane];
        z = p.z[t0 + lane];
      }
      __syncwarp();
      w.tx[lane] = x;
      w.ty[lane] = y;
      w.tz[lane] = z;
      w.kd[lane] = act ? CUDART_INF : -1.0;  // no target: no ball
      w.ki[lane] = kKnnNone;
      for (int t = 0; t < nt; t++) {
        Ld[t * 32 + lane] = CUDART_INF;
        Li[t * 32 + lane] = kKnnNone;
      }
      // 1. a window of 64 particles around the chunk in key order
      const int64_t wl = max((int64_t)0, min((int64_t)t0 + nt / 2 - 32, n - 64));
      const int w0 = (int)wl, w1 = (int)min(n, wl + 64);
      knn_stage_candidate(w, p, lane, w0 + lane < w1 ? w0 + lane : -1);
      knn_stage_candidate(w, p, 32 + lane, w0 + 32 + lane < w1 ? w0 + 32 + lane : -1);
      knn_chunk(w, nt, 64, Ld, Li, lane);
      // 2. the walk, 32 children (4 opened nodes) per step: a node is kept
      // if its box comes within the largest ball of the bucket's particle box
      // (a superset of DensityVisitor::open's per-target test, with a margin
      // for rounding); the leaves kept are buffered and flushed after 4, 8,
      // 16, ... so that the balls shrink early
      const double blo[3] = {mom[tnode].lo[0], mom[tnode].lo[1], mom[tnode].lo[2]};
      const double bhi[3] = {mom[tnode].hi[0], mom[tnode].hi[1], mom[tnode].hi[2]};
      double rmax = knn_rmax2(w, lane);
      int sp = 0, nleaf = 0, fthr = 4, nexp = 1, pop = -1;
      bool ok = true;
      while (true) {
        const int e = lane >> 3, c = lane & 7;
        int node = -1;
        if (pop < 0) {
          if (lane == 0) node = 0;
        } else if (e < nexp) {
          node = w.stack[pop + e] + c;
        }
        bool keep = false, internal = false;
        int first = 0;
        if (node >= 0) {
          if (node >= nnodes) {
            atomicOr(status, kErrCapacity);
          } else {
            const int type = walk[node].type;
            if (type == kTypeLeaf || type == kTypeInternal) {
              internal = (type == kTypeInternal);
              first = walk[node].first_child;
              const double* lo = mom[node].lo;
              const double* hi = mom[node].hi;
              const double nlo[3] = {lo[0], lo[1], lo[2]}, nhi[3] = {hi[0], hi[1], hi[2]};
              keep = box_box_gap2(nlo, nhi, blo, bhi) <= rmax * (1.0 + 1e-13);
              // then the per-target test itself (DensityVisitor::open)
              if (keep) {
                keep = false;
                for (int t = 0; t < nt && !keep; t++)
                  keep = box_d2(nlo, nhi, w.tx[t], w.ty[t], w.tz[t]) <= w.kd[t];
              }
            }
          }
        }
        const unsigned lt = (1u << lane) - 1u;
        const unsigned ml = __ballot_sync(kFull, keep && !internal);
        const unsigned mi = __ballot_sync(kFull, keep && internal);
        if (sp + __popc(mi) > kKnnStack || nleaf + __popc(ml) > kKnnLeaves) {
          ok = false;
          break;
        }
        __syncwarp();
        if (keep && !internal) w.leaf[nleaf + __popc(ml & lt)] = node;
        if (keep && internal) w.stack[sp + __popc(mi & lt)] = first;
        nleaf += __popc(ml);
        sp += __popc(mi);
        __syncwarp();
        if (nleaf >= fthr || (sp == 0 && nleaf > 0)) {
          knn_flush(p, walk, w, nt, nleaf, w0, w1, Ld, Li, lane);
          nleaf = 0;
          fthr = min(2 * fthr, kKnnLeaves - 32);
          rmax = knn_rmax2(w, lane);
        }
        if (sp == 0) break;
        nexp = sp < 4 ? sp : 4;
        sp -= nexp;
        pop = sp;
      }
      if (!ok && lane == 0) atomicOr(status, kErrStack);
      // 3. DensityFn over each target's list (ascending: the ball is its last
      // found entry)
      for (int t = 0; t < nt; t++) {
        const double ld = Ld[t * 32 + lane];
        const int li = Li[t * 32 + lane];
        const bool found = li != kKnnNone;
        const int cnt = __popc(__ballot_sync(kFull, found));
        const double rsq = __shfl_sync(kFull, ld, max(cnt - 1, 0));
        const double fBall = sqrt(rsq), ih2 = 4.0 / rsq;
        double term = found ? kernel_m4(ld * ih2) * p.m[li] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) term += __shfl_xor_sync(kFull, term, o);
        const int i = t0 + t;
        if (lane == 0 && cnt > 0) {
          density[i] = term / (0.125 * M_PI * (rsq * fBall));
          ballsq[i] = rsq;
        }
        if (nbr) {
          nbr[(int64_t)i * kSphK + lane] = found ? li : -1;
          nd2[(int64_t)i * kSphK + lane] = found ? ld : -1.0;
        }
      }
      __syncwarp();
    }
  }
}

// dkernelM4 (examples/SPHUtils.h:40-49), scaled: (pi h^5 / |dx|^2) dx.gradW.
__device__ __forceinline__ double dkernel_m4(double ar2) {
  double adk = sqrt(ar2);
  if (ar2 < 1.0) adk = -3 + 2.25 * adk;
  else adk = -0.75 * (2.0 - adk) * (2.0 - adk) / adk;
  return adk;
}

__device__ __forceinline__ double warp_sum_f64(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

static_assert(kSphK == 32, "the pressure pass maps one neighbour to one lane");

// visc = 0, aFac = vFac = 1, H = 0 as in doSPHCalc; u and the outputs in
// sorted order; the outputs start at zero.
__global__ void __launch_bounds__(256) sph_pressure_kernel(Particles p, const double* __restrict__ density,
                                                           const double* __restrict__ ballsq,
                                                           const double* __restrict__ u,
                                                           const int32_t* __restrict__ nbr,
                                                           const double* __restrict__ nd2, int64_t n,
                                                           double* __restrict__ ax, double* __restrict__ ay,
                                                           double* __restrict__ az, double* __restrict__ pdv,
                                                           unsigned* status) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const double gammam1 = 5.0 / 3.0 - 1.;
  for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const int32_t q = nbr[i * kSphK + lane];
    const double fd2 = nd2[i * kSphK + lane];
    const bool bad = q >= n;
    if (__any_sync(kFull, bad) && lane == 0) atomicOr(status, kErrCapacity);
    const bool live = q >= 0 && !bad;
    const double rsq = ballsq[i], fBall = sqrt(rsq), ih2 = 4.0 / rsq;
    const double rhoi = density[i];
    double rhoq = 1.0, mq = 0.0, divvi = 0.0, divvj = 0.0;
    if (live) {
      rhoq = density[q];
      mq = p.m[q];
      double rs1 = dkernel_m4(fd2 * ih2);
      rs1 *= fd2 * mq;
      divvi = rs1;
      divvj = rs1 / rhoq;
    }
    divvi = warp_sum_f64(divvi);
    divvj = warp_sum_f64(divvj);
    divvi /= rhoi;
    const double corr = (divvj != 0.0 ? divvi / divvj : 1.0);
    double sax = 0.0, say = 0.0, saz = 0.0, spdv = 0.0;
    bool acc_bad = false;  // doSPHCalc asserts isfinite(acc) (examples/SPHUtils.h:122)
    if (live) {
      const double xi = p.x[i], yi = p.y[i], zi = p.z[i];
      const double ph = 0.5 * fBall, ih2b = 4. / (fBall * fBall);
      const double fNorm1 = 0.5 * M_1_PI * ih2b * ih2b / ph;
      const double dx = p.x[q] - xi, dy = p.y[q] - yi, dz = p.z[q] - zi;
      const double fDist2 = dx * dx + dy * dy + dz * dz;
      double rs1 = dkernel_m4(fDist2 * ih2b);
      rs1 *= fNorm1;
      rs1 *= corr;
      const double aR = rs1 * p.m[i], bR = rs1 * mq;
      const double dvx = p.vx[q] - p.vx[i], dvy = p.vy[q] - p.vy[i], dvz = p.vz[q] - p.vz[i];
      const double dvdotdr = 1.0 * (dvx * dx + dvy * dy + dvz * dz) + fDist2 * 0.0;
      const double aP = u[i] * gammam1 / rhoq, bP = u[q] * gammam1 / rhoi;
      const double visc = 0.0;
      double PdV = bR * 0.5 * visc * dvdotdr;
      PdV += bR * aP * dvdotdr;
      spdv = PdV;
      const double acc = (aP + bP) + visc;
      acc_bad = !isfinite(acc);
      const double s = acc * bR;
      sax = s * dx;
      say = s * dy;
      saz = s * dz;
      if (q != i) {  // the particle's own entry has dx = 0 and adds nothing
        PdV = aR * 0.5 * visc * dvdotdr;
        PdV += aR * aP * dvdotdr;
        const double so = -acc * aR;
        atomicAdd(ax + q, so * dx);
        atomicAdd(ay + q, so * dy);
        atomicAdd(az + q, so * dz);
        atomicAdd(pdv + q, PdV);
      }
    }
    if (__any_sync(kFull, acc_bad) && lane == 0) atomicOr(status, kErrSphNonFinite);
    sax = warp_sum_f64(sax);
    say = warp_sum_f64(say);
    saz = warp_sum_f64(saz);
    spdv = warp_sum_f64(spdv);
    if (lane == 0) {
      atomicAdd(ax + i, sax);
      atomicAdd(ay + i, say);
      atomicAdd(az + i, saz);
      atomicAdd(pdv + i, spdv);
    }
  }
}

// The SPH example's integration after its pressure pass: Particle::kick then
// Particle::perturb (src/Particle.C:7-21) with the SPH fields.  Particle i is
// in sorted order (accelerations, PdV work, positions, velocities); u, u_pred
// and the predicted velocities are kept in caller order and reached through
// p.order.  Same association as the reference: (a dt) / 2, a dt, v dt,
// PdV (0.5e-7 dt); this file is compiled without FMA contraction.
__global__ void __launch_bounds__(256) sph_kick_perturb_kernel(Particles p, const double* __restrict__ ax,
                                                               const double* __restrict__ ay,
                                                               const double* __restrict__ az,
                                                               const double* __restrict__ pdv, double* __restrict__ u,
                                                               double* __restrict__ u_pred, double* __restrict__ vpx,
                                                               double* __restrict__ vpy, double* __restrict__ vpz,
                                                               int64_t n, double dt) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = p.order[i];
    const double a[3] = {ax[i], ay[i], az[i]};
    double v[3] = {p.vx[i], p.vy[i], p.vz[i]};
    double vp[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      v[d] += a[d] * dt / 2;    // kick
      v[d] += (a[d] * dt / 2);  // perturb
      vp[d] = v[d] + (a[d] * dt);
    }
    p.x[i] += (v[0] * dt);
    p.y[i] += (v[1] * dt);
    p.z[i] += (v[2] * dt);
    p.vx[i] = v[0];
    p.vy[i] = v[1];
    p.vz[i] = v[2];
    vpx[c] = vp[0];
    vpy[c] = vp[1];
    vpz[c] = vp[2];
    const double uDelta = 0.5e-7 * dt;
    const double w = pdv[i];
    const double uc = u[c] - w * uDelta;
    u[c] = uc;
    u_pred[c] = uc - w * uDelta;
  }
}

int sph_k() { return kSphK; }

void launch_sph_kick_perturb(Particles p, const double* ax, const double* ay, const double* az, const double* pdv,
                             double* u, double* u_pred, double* vpx, double* vpy, double* vpz, int64_t n, double dt,
                             int grid, cudaStream_t st) {
  if (n <= 0) return;
  note_launch();
  sph_kick_perturb_kernel<<<grid, 256, 0, st>>>(p, ax, ay, az, pdv, u, u_pred, vpx, vpy, vpz, n, dt);
}

void launch_sph_pressure(Particles p, const double* density, const double* ballsq, const double* u,
                         const int32_t* nbr, const double* nd2, int64_t n, double* ax, double* ay, double* az,
                         double* pdv, unsigned* status, int grid, cudaStream_t st) {
  note_launch();
  sph_pressure_kernel<<<grid, 256, 0, st>>>(p, density, ballsq, u, nbr, nd2, n, ax, ay, az, pdv, status);
}

int sph_knn_slots(int grid) { return grid * kKnnWarps; }

void launch_sph_density(Particles p, int64_t n, const Mom* mom, const WalkRec* walk, const int32_t* buckets,
                        int64_t nbuckets, int64_t nnodes, double* density, double* ballsq, int32_t* nbr, double* nd2,
                        double* lists_d, int32_t* lists_i, unsigned* work, unsigned* status, int grid,
                        cudaStream_t st) {
  note_launch();
  sph_density_kernel<<<grid, kKnnWarps * 32, 0, st>>>(p, n, mom, walk, buckets, nbuckets, nnodes, density, ballsq,
                                                      nbr, nd2, lists_d, lists_i, work, status);
}

}  // namespace pt
