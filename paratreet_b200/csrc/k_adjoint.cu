// k_adjoint.cu -- K10 adjoint of the force pass for a fixed interaction list.
//
// Given a cotangent abar_i on every acceleration, computes
//   xbar_k = d/dx_k sum_i abar_i . a_i   and   mbar_k = d/dm_k sum_i abar_i . a_i
// for the interactions recorded by the last force pass (each bucket's leaf()
// P2P sources and node() P2C nodes, examples/GravityVisitor.h:130-224).
//
//  adjoint_lists   one warp per bucket, lanes = targets, FP64:
//    P2P  a_i += m_j b(r) d,  d = x_j - x_i (SPLINE, :87-120).  The tidal
//         tensor T = b I + (b'(r)/r) d d^T gives xbar_i -= m_j T abar_i,
//         xbar_j += m_j T abar_i, mbar_j += b d.abar_i (source terms summed over
//         the warp's targets, then one atomic add per source).
//    P2C  a_i += f(r) with r = x_i - cm, f = -(bM + d q - c tr) r + c Q r
//         (quadrupole, unsoftened branch) or f = -M r / r^3 (monopole).  The
//         symmetric Jacobian J = df/dr gives xbar_i += J abar_i, and the
//         node receives cmbar -= J abar_i, Mbar += df/dM . abar_i and the six
//         Qbar components, summed over the warp and added atomically.
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


__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kAdjFull, v, o);
  return v;
}

// SPLINE force term b(r) and its derivative db/dr.
__device__ __forceinline__ void spline_b_db(double r2, double twoh, double& b, double& db) {
  const double r = sqrt(r2);
  if (r < twoh) {
    const double dih = 2.0 / twoh;
    const double u = r * dih;
    const double d3 = dih * dih * dih, d4 = d3 * dih;
    if (u < 1.0) {
      b = d3 * (4.0 / 3.0 - 6.0 / 5.0 * u * u + 0.5 * u * u * u);
      db = d4 * (-12.0 / 5.0 * u + 1.5 * u * u);
    } else {
      const double ir = 1.0 / r;
      const double ir3 = ir * ir * ir;
      b = -1.0 / 15.0 * ir3 + d3 * (8.0 / 3.0 - 3.0 * u + 6.0 / 5.0 * u * u - 1.0 / 6.0 * u * u * u);
      db = 0.2 * ir3 * ir + d4 * (-3.0 + 12.0 / 5.0 * u - 0.5 * u * u);
    }
  } else {
    const double ir = 1.0 / r;
    b = ir * ir * ir;
    db = -3.0 * b * ir;
  }
}

__global__ void __launch_bounds__(kAdjWarps * 32) adjoint_lists(AdjParams A) {
  __shared__ double stage[kAdjWarps][5][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double(*st)[32] = stage[wid];
  while (true) {
    unsigned bi = 0;
    if (lane == 0) bi = atomicAdd(A.work, 1u);
    bi = __shfl_sync(kAdjFull, bi, 0);
    const int64_t b = (int64_t)bi;
    if (b >= A.nbuckets) break;
    const int tnode = A.buckets[b];
    const int tbase = A.walk[tnode].pstart, ntot = A.walk[tnode].pcount;
    const int64_t e0 = A.list_off[b], e1 = A.list_off[b + 1];
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const bool act = lane < nt;
      double xi = 0.0, yi = 0.0, zi = 0.0, si = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
      if (act) {
        const int i = t0 + lane;
        xi = A.p.x[i]; yi = A.p.y[i]; zi = A.p.z[i]; si = A.p.soft[i];
        ax = A.cax[i]; ay = A.cay[i]; az = A.caz[i];
      }
      double gxi = 0.0, gyi = 0.0, gzi = 0.0;
      for (int64_t e = e0; e < e1; e++) {
        const int node = A.list_node[e];
        const int kind = A.list_kind[e];
        if (node < 0 || node >= A.nnodes) {
          if (lane == 0) atomicOr(A.status, kErrCapacity);
          continue;
        }
        const WalkRec w = A.walk[node];
        if (kind == 0) {  // P2P with the leaf's particles
          for (int base = 0; base < w.pcount; base += 32) {
            const int cnt = min(32, w.pcount - base);
            __syncwarp();
            if (lane < cnt) {
              const int j = w.pstart + base + lane;
              st[0][lane] = A.p.x[j]; st[1][lane] = A.p.y[j]; st[2][lane] = A.p.z[j];
              st[3][lane] = A.p.m[j]; st[4][lane] = A.p.soft[j];
            }
            __syncwarp();
            for (int jj = 0; jj < cnt; jj++) {
              double sx = 0.0, sy = 0.0, sz = 0.0, sm = 0.0;
              if (act) {
                const double dx = st[0][jj] - xi, dy = st[1][jj] - yi, dz = st[2][jj] - zi;
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 != 0.0) {
                  double bb, db;
                  spline_b_db(r2, st[4][jj] + si, bb, db);
                  const double da = dx * ax + dy * ay + dz * az;
                  const double k = db / sqrt(r2) * da;
                  const double mj = st[3][jj];
                  const double tx = bb * ax + k * dx, ty = bb * ay + k * dy, tz = bb * az + k * dz;
                  sx = mj * tx; sy = mj * ty; sz = mj * tz;
                  gxi -= sx; gyi -= sy; gzi -= sz;
                  sm = bb * da;
                }
              }
              sx = wsum(sx); sy = wsum(sy); sz = wsum(sz); sm = wsum(sm);
              if (lane == 0) {
                const int j = w.pstart + base + jj;
                atomicAdd(&A.gx[j], sx);
                atomicAdd(&A.gy[j], sy);
                atomicAdd(&A.gz[j], sz);
                atomicAdd(&A.gm[j], sm);
              }
            }
          }
        } else {  // P2C: quadrupole (kind 1) or softened-overlap monopole (kind 2)
          const QuadRec q = A.quad[node];
          double c[10];
#pragma unroll
          for (int k = 0; k < 10; k++) c[k] = 0.0;
          if (act && w.count > 0) {
            const double rx = xi - w.cm[0], ry = yi - w.cm[1], rz = zi - w.cm[2];
            const double r2 = rx * rx + ry * ry + rz * rz;
            const double ir = 1.0 / sqrt(r2);
            const double ir2 = ir * ir;
            const double ra = rx * ax + ry * ay + rz * az;
            double jx, jy, jz;
            if (kind == 2) {  // f = -M r / r^3
              const double b3 = ir2 * ir;
              const double t = 3.0 * b3 * ir2 * ra;
              jx = -q.mass * (b3 * ax - t * rx);
              jy = -q.mass * (b3 * ay - t * ry);
              jz = -q.mass * (b3 * az - t * rz);
              c[3] = -b3 * ra;
            } else {
              const double twoh = q.soft + si;
              if (r2 < twoh * twoh) {
                atomicOr(A.status, kErrAdjointSoftened);
                jx = jy = jz = 0.0;
              } else {
                const double bb = ir2 * ir, cc = 3.0 * bb * ir2, dd = 5.0 * cc * ir2, ee = 7.0 * dd * ir2;
                const double qx = q.xx * rx + q.xy * ry + q.xz * rz;
                const double qy = q.xy * rx + q.yy * ry + q.yz * rz;
                const double qz = q.xz * rx + q.yz * ry + q.zz * rz;
                const double qq = 0.5 * (qx * rx + qy * ry + qz * rz);
                const double tr = 0.5 * (q.xx + q.yy + q.zz);
                const double s = bb * q.mass + dd * qq - cc * tr;
                const double qra = qx * ax + qy * ay + qz * az;
                const double qax = q.xx * ax + q.xy * ay + q.xz * az;
                const double qay = q.xy * ax + q.yy * ay + q.yz * az;
                const double qaz = q.xz * ax + q.yz * ay + q.zz * az;
                const double k1 = (cc * q.mass + ee * qq - dd * tr) * ra - dd * qra;
                jx = -s * ax + k1 * rx + cc * qax - dd * ra * qx;
                jy = -s * ay + k1 * ry + cc * qay - dd * ra * qy;
                jz = -s * az + k1 * rz + cc * qaz - dd * ra * qz;
                c[3] = -bb * ra;
                const double h = -dd * ra;
                c[4] = h * 0.5 * rx * rx + cc * ra * 0.5 + cc * ax * rx;
                c[5] = h * 0.5 * ry * ry + cc * ra * 0.5 + cc * ay * ry;
                c[6] = h * 0.5 * rz * rz + cc * ra * 0.5 + cc * az * rz;
                c[7] = h * rx * ry + cc * (ax * ry + ay * rx);
                c[8] = h * rx * rz + cc * (ax * rz + az * rx);
                c[9] = h * ry * rz + cc * (ay * rz + az * ry);
              }
            }
            gxi += jx; gyi += jy; gzi += jz;
            c[0] = -jx; c[1] = -jy; c[2] = -jz;
          }
#pragma unroll
          for (int k = 0; k < 10; k++) c[k] = wsum(c[k]);
          if (lane < 10) {
            double v = c[0];
#pragma unroll
            for (int k = 1; k < 10; k++)
              if (lane == k) v = c[k];
            atomicAdd(&A.nadj[10 * (int64_t)node + lane], v);
          }
        }
      }
      if (act) {
        const int i = t0 + lane;
        atomicAdd(&A.gx[i], gxi);
        atomicAdd(&A.gy[i], gyi);
        atomicAdd(&A.gz[i], gzi);
      }
    }
  }
}

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
