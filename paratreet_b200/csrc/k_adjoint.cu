// k_adjoint.cu -- K10 adjoint of the force pass for a fixed interaction list.
//
// Given a cotangent abar_i on every acceleration, computes
//   xbar_k = d/dx_k sum_i abar_i . a_i   and   mbar_k = d/dm_k sum_i abar_i . a_i
// for the interactions recorded by the last force pass (each bucket's leaf()
// P2P sources and node() P2C nodes, examples/GravityVisitor.h:130-224).
//
//  adjoint_lists   one warp per bucket, FP64 (work layout at AdjWarp below):
//    P2P  a_i += m_j b(r) d,  d = x_j - x_i (SPLINE, :87-120).  The tidal
//         tensor T = b I + (b'(r)/r) d d^T gives xbar_i -= m_j T abar_i,
//         xbar_j += m_j T abar_i, mbar_j += b d.abar_i (source terms summed
//         in shared memory over the bucket's targets, then one atomic add per
//         source).
//    P2C  a_i += f(r) with r = x_i - cm, f = -(bM + d q - c tr) r + c Q r
//         (quadrupole, unsoftened branch) or f = -M r / r^3 (monopole).  The
//         symmetric Jacobian J = df/dr gives xbar_i += J abar_i, and the
//         node receives cmbar -= J abar_i, Mbar += df/dM . abar_i and the six
//         Qbar components, summed in shared memory and added atomically.
//  adjoint_upward  the upward pass (examples/MultipoleMoments.h:204-353) in
//         closed form: M = sum m_k, cm = sum m_k x_k / M,
//         Q_ab = sum m_k (x_k - cm)_a (x_k - cm)_b, so every internal ancestor
//         n of particle k contributes xbar_k += (m_k/M) cmbar + m_k S (x_k - cm)
//         and mbar_k += Mbar + cmbar.(x_k - cm)/M + (x_k - cm)^T Qbar (x_k - cm).
// The softened quadrupole branch cannot occur with uniform softening (the
// walk sends overlapping softening spheres to the monopole); if it does, the
// status word reports it and the term is skipped.
#include "pt_internal.cuh"

namespace pt {

constexpr int kAdjWarps = 4;
constexpr unsigned kAdjFull = 0xffffffffu;

// Phase timers of a diagnostic build (PT_PROF=1), summed per phase into
// g_prof_adj: P2C windows, P2P windows, the target-side sums.
#ifndef PT_PROF
#define PT_PROF 0
#endif
#if PT_PROF
__device__ unsigned long long g_prof_adj[8];
#define ADJ_T0 unsigned t_prev_ = (unsigned)clock();
#define ADJ_MARK(i) if (lane == 0) { const unsigned t_ = (unsigned)clock(); atomicAdd(&g_prof_adj[i], (unsigned long long)(t_ - t_prev_)); t_prev_ = t_; }
#else
#define ADJ_T0
#define ADJ_MARK(i)
#endif


__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kAdjFull, v, o);
  return v;
}

// SPLINE force term b(r) and its derivative db/dr, from r^2 and 1/r.
__device__ __forceinline__ void spline_b_db(double r2, double ir, double twoh, double& b, double& db) {
  if (r2 < twoh * twoh) {
    const double r = r2 * ir;
    const double dih = 2.0 / twoh;
    const double u = r * dih;
    const double d3 = dih * dih * dih, d4 = d3 * dih;
    if (u < 1.0) {
      b = d3 * (4.0 / 3.0 - 6.0 / 5.0 * u * u + 0.5 * u * u * u);
      db = d4 * (-12.0 / 5.0 * u + 1.5 * u * u);
    } else {
      const double ir3 = ir * ir * ir;
      b = -1.0 / 15.0 * ir3 + d3 * (8.0 / 3.0 - 3.0 * u + 6.0 / 5.0 * u * u - 1.0 / 6.0 * u * u * u);
      db = 0.2 * ir3 * ir + d4 * (-3.0 + 12.0 / 5.0 * u - 0.5 * u * u);
    }
  } else {
    b = ir * ir * ir;
    db = -3.0 * b * ir;
  }
}

// Work layout of adjoint_lists: one warp per bucket, the bucket's n_t targets
// two per lane in groups of h = ceil(n_t / 2) lanes, replicated over
// G = floor(32 / h) lane groups (as the evaluation kernels do).  A chunk of up
// to 32 list nodes, or of 32 source particles of the listed leaves, is staged
// in shared memory with one adjoint accumulator row per staged slot; group g
// takes the slots g, g + G, ...  Inside a group, at step s lane t handles its
// group's slot number (s + t) mod L (L = max(h, the group's slots)), so no two
// lanes touch one slot in a step and each (target, slot) pair is visited once;
// a __syncwarp separates the steps.  The
// target-side terms stay in registers; the source-side ones are added to the
// slot's row and flushed with one atomic add per slot and value after the
// chunk.  Atomic adds make the last bits of the results order-dependent.
struct AdjWarp {
  double st[12][32];   // staged slot data: P2C cm x/y/z, M, xx, xy, xz, yy, yz, zz, kind, soft; P2P x/y/z, m, soft
  double acc[10][32];  // per slot adjoint rows: node (cm x/y/z, M, 6 moments) or source (x/y/z, m)
  int32_t sidx[32];    // the slot's node or particle index
  int32_t lnode[32];   // P2P: the window's leaves
  int32_t lincl[32];   // P2P: inclusive prefix of their particle counts
  int32_t lpst[32];    // P2P: their first particles
};

// One target of a lane: position, softening and cotangent.
struct AdjTgt {
  double x, y, z, s, ax, ay, az;
};

// The lane's targets: lane l of group l / h holds targets 2 (l mod h) and
// 2 (l mod h) + 1 (h = ceil(n_t / 2), t2 == n_t when there is none), so every
// staged slot is read, and its row updated, once for two pairs (Hernquist
// N = 262,144, theta 0.6: 13.4 -> 11.8 ms against one target per lane).
struct AdjTarget {
  int t1, t2, tl, h, grp, G, nt;
  bool act, two;
  AdjTgt a, b;
};

// P2C terms of one (target, staged node k) pair: the target-side Jacobian
// term j (returned in jx, jy, jz) and the ten node-side terms added to c.
// False for the softened quadrupole branch (reported, not differentiated).
__device__ __forceinline__ bool adj_p2c_terms(const AdjWarp& w, int k, const AdjTgt& x, double& jx, double& jy,
                                              double& jz, double c[10], unsigned* status) {
  const double rx = x.x - w.st[0][k], ry = x.y - w.st[1][k], rz = x.z - w.st[2][k];
  const double M = w.st[3][k];
  const double r2 = rx * rx + ry * ry + rz * rz;
  const double ir = rsqrt(r2);
  const double ir2 = ir * ir;
  const double ra = rx * x.ax + ry * x.ay + rz * x.az;
  if (w.st[10][k] == 2.0) {  // monopole: f = -M r / r^3
    const double b3 = ir2 * ir;
    const double t = 3.0 * b3 * ir2 * ra;
    jx = -M * (b3 * x.ax - t * rx);
    jy = -M * (b3 * x.ay - t * ry);
    jz = -M * (b3 * x.az - t * rz);
    c[3] += -b3 * ra;
  } else {
    const double twoh = w.st[11][k] + x.s;
    if (r2 < twoh * twoh) {  // the softened quadrupole branch: reported, not differentiated
      atomicOr(status, kErrAdjointSoftened);
      return false;
    }
    const double xx = w.st[4][k], xy = w.st[5][k], xz = w.st[6][k];
    const double yy = w.st[7][k], yz = w.st[8][k], zz = w.st[9][k];
    const double bb = ir2 * ir, cc = 3.0 * bb * ir2, dd = 5.0 * cc * ir2, ee = 7.0 * dd * ir2;
    const double qx = xx * rx + xy * ry + xz * rz;
    const double qy = xy * rx + yy * ry + yz * rz;
    const double qz = xz * rx + yz * ry + zz * rz;
    const double qq = 0.5 * (qx * rx + qy * ry + qz * rz);
    const double tr = 0.5 * (xx + yy + zz);
    const double s = bb * M + dd * qq - cc * tr;
    const double qra = qx * x.ax + qy * x.ay + qz * x.az;
    const double qax = xx * x.ax + xy * x.ay + xz * x.az;
    const double qay = xy * x.ax + yy * x.ay + yz * x.az;
    const double qaz = xz * x.ax + yz * x.ay + zz * x.az;
    const double k1 = (cc * M + ee * qq - dd * tr) * ra - dd * qra;
    jx = -s * x.ax + k1 * rx + cc * qax - dd * ra * qx;
    jy = -s * x.ay + k1 * ry + cc * qay - dd * ra * qy;
    jz = -s * x.az + k1 * rz + cc * qaz - dd * ra * qz;
    c[3] += -bb * ra;
    const double h = -dd * ra;
    c[4] += h * 0.5 * rx * rx + cc * ra * 0.5 + cc * x.ax * rx;
    c[5] += h * 0.5 * ry * ry + cc * ra * 0.5 + cc * x.ay * ry;
    c[6] += h * 0.5 * rz * rz + cc * ra * 0.5 + cc * x.az * rz;
    c[7] += h * rx * ry + cc * (x.ax * ry + x.ay * rx);
    c[8] += h * rx * rz + cc * (x.ax * rz + x.az * rx);
    c[9] += h * ry * rz + cc * (x.ay * rz + x.az * ry);
  }
  c[0] -= jx;
  c[1] -= jy;
  c[2] -= jz;
  return true;
}

// P2P terms of one (target, staged source k) pair: T = b I + (b'/r) d d^T
// with d = x_k - x_i; the target gets -m_k T abar_i (returned as s), the
// source +m_k T abar_i and mbar_k += b d.abar_i (added to c[0..3]).
__device__ __forceinline__ void adj_p2p_terms(const AdjWarp& w, int k, const AdjTgt& x, double& gx, double& gy,
                                              double& gz, double c[4]) {
  const double dx = w.st[0][k] - x.x, dy = w.st[1][k] - x.y, dz = w.st[2][k] - x.z;
  const double r2 = dx * dx + dy * dy + dz * dz;
  if (r2 == 0.0) return;
  const double ir = rsqrt(r2);
  double bb, db;
  spline_b_db(r2, ir, w.st[4][k] + x.s, bb, db);
  const double da = dx * x.ax + dy * x.ay + dz * x.az;
  const double kk = db * ir * da;
  const double mj = w.st[3][k];
  const double sx = mj * (bb * x.ax + kk * dx), sy = mj * (bb * x.ay + kk * dy), sz = mj * (bb * x.az + kk * dz);
  gx -= sx;
  gy -= sy;
  gz -= sz;
  c[0] += sx;
  c[1] += sy;
  c[2] += sz;
  c[3] += bb * da;
}

// The rotation over the n staged slots of a chunk (see AdjWarp), with the
// lane's one or two targets; kP2C picks the pair kind.  Every lane runs the
// same number of steps.
template <bool kP2C>
__device__ __forceinline__ void adj_rotate(AdjWarp& w, int n, const AdjTarget& x, double g[6], unsigned* status) {
  const int mg = (x.grp < x.G && x.grp < n) ? (n - x.grp + x.G - 1) / x.G : 0;  // this group's slots
  const int mmax = (n + x.G - 1) / x.G;
  const int L = max(x.h, mmax);
  for (int st = 0; st < L; st++) {
    const int local = (st + x.tl) % L;
    if (x.act && local < mg) {
      const int k = x.grp + x.G * local;
      if (kP2C) {
        double c[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        double jx, jy, jz;
        if (adj_p2c_terms(w, k, x.a, jx, jy, jz, c, status)) {
          g[0] += jx;
          g[1] += jy;
          g[2] += jz;
        }
        if (x.two && adj_p2c_terms(w, k, x.b, jx, jy, jz, c, status)) {
          g[3] += jx;
          g[4] += jy;
          g[5] += jz;
        }
#pragma unroll
        for (int q = 0; q < 10; q++) w.acc[q][k] += c[q];
      } else {
        double c[4] = {0.0, 0.0, 0.0, 0.0};
        adj_p2p_terms(w, k, x.a, g[0], g[1], g[2], c);
        if (x.two) adj_p2p_terms(w, k, x.b, g[3], g[4], g[5], c);
#pragma unroll
        for (int q = 0; q < 4; q++) w.acc[q][k] += c[q];
      }
    }
    __syncwarp();
  }
}

__device__ __forceinline__ AdjTgt adj_load_target(const AdjParams& A, int i) {
  AdjTgt t;
  t.x = A.p.x[i]; t.y = A.p.y[i]; t.z = A.p.z[i]; t.s = A.p.soft[i];
  t.ax = A.cax[i]; t.ay = A.cay[i]; t.az = A.caz[i];
  return t;
}

// CTAs per SM of adjoint_lists: 5 (96 registers, a little spilled) measured
// faster than the 4 that 124 registers allow (13.0 -> 11.7 ms); 6 and 7 spill
// far more (14.4 and 15.8 ms)
#ifndef PT_ADJ_MINB
#define PT_ADJ_MINB 5
#endif
__global__ void __launch_bounds__(kAdjWarps * 32, PT_ADJ_MINB) adjoint_lists(AdjParams A) {
  __shared__ AdjWarp warps[kAdjWarps];
  AdjWarp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  ADJ_T0
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(A.work, 1u);
    bi = __shfl_sync(kAdjFull, bi, 0);
    const int64_t b = (int64_t)bi;
    if (b >= A.nbuckets) break;
    const int tnode = A.buckets[b];
    if (tnode < 0 || tnode >= A.nnodes) {
      if (lane == 0) atomicOr(A.status, kErrCapacity);
      continue;
    }
    const int tbase = A.walk[tnode].pstart, ntot = A.walk[tnode].pcount;
    const int64_t e0 = A.list_off[b], e1 = A.list_off[b + 1];
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      AdjTarget x;
      x.nt = nt;
      x.h = (nt + 1) >> 1;
      x.G = 32 / x.h;
      x.grp = lane / x.h;
      x.tl = lane % x.h;
      x.act = x.grp < x.G;
      x.t1 = 2 * x.tl;
      x.t2 = min(x.t1 + 1, nt);
      x.two = x.act && x.t2 < nt;
      x.a = x.b = AdjTgt{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (x.act) x.a = adj_load_target(A, t0 + x.t1);
      if (x.two) x.b = adj_load_target(A, t0 + x.t2);
      double g[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // target-side sums of the lane's targets
      ADJ_MARK(0);
      // P2C: the list's nodes, 32 at a time
      for (int64_t win = e0; win < e1; win += 32) {
        const int64_t e = win + lane;
        int node = -1, kind = 0;
        if (e < e1) {
          kind = A.list_kind[e];
          node = A.list_node[e];
          if (node < 0 || node >= A.nnodes) {
            atomicOr(A.status, kErrCapacity);
            kind = 0;
          } else if (kind != 0 && A.walk[node].count == 0) {
            kind = 0;  // node() of an empty node adds nothing
          }
        }
        const bool sel = e < e1 && kind != 0;
        const unsigned m = __ballot_sync(kAdjFull, sel);
        const int n = __popc(m);
        if (n == 0) continue;
        __syncwarp();
        if (sel) {
          const int k = __popc(m & ((1u << lane) - 1u));
          const WalkRec& r = A.walk[node];
          const QuadRec q = A.quad[node];
          w.sidx[k] = node;
          w.st[0][k] = r.cm[0]; w.st[1][k] = r.cm[1]; w.st[2][k] = r.cm[2];
          w.st[3][k] = q.mass;
          w.st[4][k] = q.xx; w.st[5][k] = q.xy; w.st[6][k] = q.xz;
          w.st[7][k] = q.yy; w.st[8][k] = q.yz; w.st[9][k] = q.zz;
          w.st[10][k] = (double)kind;
          w.st[11][k] = q.soft;
        }
#pragma unroll
        for (int q = 0; q < 10; q++) w.acc[q][lane] = 0.0;
        __syncwarp();
        adj_rotate<true>(w, n, x, g, A.status);
        if (lane < n) {
          double* na = A.nadj + 10 * (int64_t)w.sidx[lane];
#pragma unroll
          for (int q = 0; q < 10; q++) atomicAdd(na + q, w.acc[q][lane]);
        }
        __syncwarp();
      }
      ADJ_MARK(1);
      // P2P: the listed leaves' particles, 32 at a time
      for (int64_t win = e0; win < e1; win += 32) {
        const int64_t e = win + lane;
        int node = -1;
        bool sel = false;
        if (e < e1 && A.list_kind[e] == 0) {
          node = A.list_node[e];
          sel = node >= 0 && node < A.nnodes;
        }
        const unsigned m = __ballot_sync(kAdjFull, sel);
        const int nl = __popc(m);
        if (nl == 0) continue;
        int cnt = 0, pst = 0;
        if (sel) {
          cnt = A.walk[node].pcount;
          pst = A.walk[node].pstart;
        }
        int inc = cnt;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(kAdjFull, inc, o);
          if (lane >= o) inc += y;
        }
        const int total = __shfl_sync(kAdjFull, inc, 31);
        __syncwarp();
        if (sel) {
          const int k = __popc(m & ((1u << lane) - 1u));
          w.lnode[k] = node;
          w.lincl[k] = inc;
          w.lpst[k] = pst;
        }
        __syncwarp();
        for (int cs = 0; cs < total; cs += 32) {
          const int q = cs + lane;
          const int n = min(32, total - cs);
          if (q < total) {
            int lo = 0, hi = nl - 1;  // the first leaf with inclusive prefix > q
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (w.lincl[mid] > q) hi = mid;
              else lo = mid + 1;
            }
            const int first = (lo == 0) ? 0 : w.lincl[lo - 1];
            const int j = w.lpst[lo] + (q - first);
            w.sidx[lane] = j;
            w.st[0][lane] = A.p.x[j]; w.st[1][lane] = A.p.y[j]; w.st[2][lane] = A.p.z[j];
            w.st[3][lane] = A.p.m[j]; w.st[4][lane] = A.p.soft[j];
          }
#pragma unroll
          for (int r = 0; r < 4; r++) w.acc[r][lane] = 0.0;
          __syncwarp();
          adj_rotate<false>(w, n, x, g, A.status);
          if (lane < n) {
            const int j = w.sidx[lane];
            atomicAdd(&A.gx[j], w.acc[0][lane]);
            atomicAdd(&A.gy[j], w.acc[1][lane]);
            atomicAdd(&A.gz[j], w.acc[2][lane]);
            atomicAdd(&A.gm[j], w.acc[3][lane]);
          }
          __syncwarp();
        }
      }
      ADJ_MARK(2);
      // the target-side sums of the G groups: slot (group, target) rows in
      // the staging area (G n_t <= 64 slots)
      double* red = &w.st[0][0];
      __syncwarp();
      if (x.act) {
        const int s1 = 3 * (x.grp * nt + x.t1);
        red[s1] = g[0]; red[s1 + 1] = g[1]; red[s1 + 2] = g[2];
        if (x.two) {
          const int s2 = 3 * (x.grp * nt + x.t2);
          red[s2] = g[3]; red[s2 + 1] = g[4]; red[s2 + 2] = g[5];
        }
      }
      __syncwarp();
      if (lane < nt) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int gg = 0; gg < x.G; gg++) {
          const int sl = 3 * (gg * nt + lane);
          sx += red[sl];
          sy += red[sl + 1];
          sz += red[sl + 2];
        }
        const int i = t0 + lane;
        atomicAdd(&A.gx[i], sx);
        atomicAdd(&A.gy[i], sy);
        atomicAdd(&A.gz[i], sz);
      }
      __syncwarp();
      ADJ_MARK(3);
    }
  }
}

#if PT_PROF
extern "C" int pt_debug_prof_adj(unsigned long long* out) {
  if (cudaMemcpyFromSymbol(out, g_prof_adj, sizeof(g_prof_adj)) != cudaSuccess) return -1;
  unsigned long long z[8] = {};
  return cudaMemcpyToSymbol(g_prof_adj, z, sizeof(z)) == cudaSuccess ? 0 : -1;
}
#endif

// Node adjoints -> particles through the closed-form upward pass.
__global__ void __launch_bounds__(kAdjWarps * 32) adjoint_upward(AdjParams A) {
  const int lane = threadIdx.x & 31;
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (b >= A.nbuckets) return;
  const int leaf = A.buckets[b];
  const int ps = A.walk[leaf].pstart, pc = A.walk[leaf].pcount;
  for (int tc = 0; tc < pc; tc += 32) {
    const bool act = tc + lane < pc;
    const int k = ps + tc + lane;
    double xk = 0.0, yk = 0.0, zk = 0.0, mk = 0.0;
    if (act) { xk = A.p.x[k]; yk = A.p.y[k]; zk = A.p.z[k]; mk = A.p.m[k]; }
    double gx = 0.0, gy = 0.0, gz = 0.0, gm = 0.0;
    int n = A.parent[leaf];
    int guard = 0;
    while (n >= 0 && guard++ < 64) {
      const Mom& q = A.mom[n];
      const double M = q.mass;
      if (M != 0.0) {
        const double* a = A.nadj + 10 * (int64_t)n;
        const double cbx = a[0], cby = a[1], cbz = a[2], Mb = a[3];
        const double Qxx = a[4], Qyy = a[5], Qzz = a[6], Qxy = a[7], Qxz = a[8], Qyz = a[9];
        const double dx = xk - q.cm[0], dy = yk - q.cm[1], dz = zk - q.cm[2];
        const double f = mk / M;
        gx += f * cbx + mk * (2.0 * Qxx * dx + Qxy * dy + Qxz * dz);
        gy += f * cby + mk * (Qxy * dx + 2.0 * Qyy * dy + Qyz * dz);
        gz += f * cbz + mk * (Qxz * dx + Qyz * dy + 2.0 * Qzz * dz);
        gm += Mb + (cbx * dx + cby * dy + cbz * dz) / M + Qxx * dx * dx + Qyy * dy * dy + Qzz * dz * dz +
              Qxy * dx * dy + Qxz * dx * dz + Qyz * dy * dz;
      }
      n = A.parent[n];
    }
    if (act) {
      A.gx[k] += gx;
      A.gy[k] += gy;
      A.gz[k] += gz;
      A.gm[k] += gm;
    }
  }
}

void launch_adjoint(const AdjParams& A, int grid, cudaStream_t st) {
  note_launch();
  adjoint_lists<<<grid, kAdjWarps * 32, 0, st>>>(A);
  if (A.nbuckets > 0) {
    note_launch();
    adjoint_upward<<<(unsigned)((A.nbuckets * 32 + kAdjWarps * 32 - 1) / (kAdjWarps * 32)), kAdjWarps * 32, 0, st>>>(A);
  }
}

}  // namespace pt
