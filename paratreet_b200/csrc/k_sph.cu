// k_sph.cu -- the SPH example's density pass on the gravity tree: k = 32
// nearest neighbours of every particle (DensityVisitor, examples/
// DensityVisitor.h, walked with startUpAndDown, examples/SPH.C:77-86) and the
// M4-kernel density (DensityFn, examples/SPH.C:11-37; kernelM4,
// examples/SPHUtils.h:20-26).  FP64, compiled with -fmad=false so that
// d2 = dx*dx + dy*dy + dz*dz (dx = x_i - x_j) is the reference's value bit for
// bit; the neighbour set is the exact k nearest (the particle itself
// included), which the reference's conservative open() also yields.
//
// One warp per bucket, lanes = target particles (chunks of 32).  Each lane
// keeps a max-heap of its k best (d2, particle) in shared memory.  The walk is
// depth first from the root; a popped node is visited if any lane's heap is
// not full or its ball (the current k-th d2) reaches the node's box
// (DensityVisitor::open with Space::intersect's <=), so balls that shrank
// since the push prune more; children are pushed far to near (distance of
// their boxes to the bucket's centre) so the nearest subtree is searched first.
//
// The pressure pass that follows (sph_pressure_kernel) restates ForceFn
// (examples/SPH.C:39-64) and doSPHCalc (examples/SPHUtils.h:64-133): one warp
// per particle, lane e = its e-th neighbour from the density pass.  The divv
// corrector and the particle's own pressure acceleration and PdV work are warp
// sums; the opposite reaction on each neighbour (ThreadStateHolder's opposing
// effects, applied after the pass in the reference) is an FP64 atomic add, so
// its summation order is not fixed.
#include "pt_internal.cuh"
#include "pt_walk.cuh"

namespace pt {

constexpr int kSphK = 32;
constexpr int kSphWarps = 2;
constexpr int kSphStack = 256;  // pending nodes: <= 21 levels x 7 siblings + the root

struct SphWarp {
  double hd[kSphK][32];  // heap distances^2, column per lane
  int32_t hi[kSphK][32]; // heap particles (sorted order)
  int32_t stack[kSphStack];
  double sx[32], sy[32], sz[32];
  int32_t sidx[32];
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

__global__ void __launch_bounds__(kSphWarps * 32) sph_density_kernel(Particles p, const Mom* __restrict__ mom,
                                                                      const WalkRec* __restrict__ walk,
                                                                      const int32_t* __restrict__ buckets,
                                                                      int64_t nbuckets, int64_t nnodes,
                                                                      double* __restrict__ density,
                                                                      double* __restrict__ ballsq,
                                                                      int32_t* __restrict__ nbr,
                                                                      double* __restrict__ nd2, unsigned* work,
                                                                      unsigned* status) {
  __shared__ SphWarp warps[kSphWarps];
  SphWarp& w = warps[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
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
    const double gx = mom[tnode].cm[0], gy = mom[tnode].cm[1], gz = mom[tnode].cm[2];
    for (int tc = 0; tc < ntot; tc += 32) {
      const int t0 = tbase + tc, nt = min(32, ntot - tc);
      const bool act = lane < nt;
      double xi = 0.0, yi = 0.0, zi = 0.0;
      if (act) {
        xi = p.x[t0 + lane];
        yi = p.y[t0 + lane];
        zi = p.z[t0 + lane];
      }
      int cnt = 0;  // heap entries of this lane
      int sp = 0;
      if (lane == 0) w.stack[0] = 0;
      sp = 1;
      bool ok = true;
      __syncwarp();
      while (sp > 0) {
        const int node = w.stack[sp - 1];
        sp--;
        __syncwarp();
        if (node < 0 || node >= nnodes) {
          if (lane == 0) atomicOr(status, kErrCapacity);
          continue;
        }
        const WalkRec& r = walk[node];
        const int type = r.type;
        if (type != kTypeLeaf && type != kTypeInternal) continue;
        // open: some lane's heap is not full, or its ball reaches the box
        const Mom& q = mom[node];
        bool want = false;
        if (act) want = (cnt < kSphK) || (box_d2(q.lo, q.hi, xi, yi, zi) <= w.hd[0][lane]);
        if (!__any_sync(kFull, want)) continue;
        if (type == kTypeInternal) {
          // children far to near by the distance of their boxes to the bucket centre
          const int c = lane & 7;
          const int child = r.first_child + c;
          double dc = -1.0;
          bool live = false;
          if (lane < 8 && child < nnodes) {
            const int ct = walk[child].type;
            live = (ct == kTypeLeaf || ct == kTypeInternal);
            if (live) dc = box_d2(mom[child].lo, mom[child].hi, gx, gy, gz);
          }
          const unsigned lm = __ballot_sync(kFull, live) & 0xffu;
          const int nlive = __popc(lm);
          if (sp + nlive > kSphStack) {
            ok = false;
            break;
          }
          int rank = 0;  // children nearer than this one (ties: lower index first)
#pragma unroll
          for (int o = 0; o < 8; o++) {
            const double d = __shfl_sync(kFull, dc, o);
            const bool lv = (lm >> o) & 1u;
            if (live && lv && o != c && (d < dc || (d == dc && o < c))) rank++;
          }
          if (live) w.stack[sp + nlive - 1 - rank] = child;  // the nearest ends on top
          sp += nlive;
          __syncwarp();
          continue;
        }
        // leaf: every lane tests every particle (DensityVisitor::leaf)
        const int s0 = r.pstart, sn = r.pcount;
        for (int base = 0; base < sn; base += 32) {
          const int cntj = min(32, sn - base);
          __syncwarp();
          if (lane < cntj) {
            const int j = s0 + base + lane;
            w.sx[lane] = p.x[j];
            w.sy[lane] = p.y[j];
            w.sz[lane] = p.z[j];
            w.sidx[lane] = j;
          }
          __syncwarp();
          if (act) {
            for (int jj = 0; jj < cntj; jj++) {
              const double dx = __dadd_rn(xi, -w.sx[jj]), dy = __dadd_rn(yi, -w.sy[jj]),
                           dz = __dadd_rn(zi, -w.sz[jj]);
              const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
              if (cnt < kSphK) {  // push and sift up
                int pos = cnt++;
                while (pos > 0) {
                  const int par = (pos - 1) >> 1;
                  if (!(w.hd[par][lane] < d2)) break;
                  w.hd[pos][lane] = w.hd[par][lane];
                  w.hi[pos][lane] = w.hi[par][lane];
                  pos = par;
                }
                w.hd[pos][lane] = d2;
                w.hi[pos][lane] = w.sidx[jj];
              } else if (d2 < w.hd[0][lane]) {  // replace the farthest and sift down
                int pos = 0;
                while (true) {
                  int ch = 2 * pos + 1;
                  if (ch >= kSphK) break;
                  if (ch + 1 < kSphK && w.hd[ch + 1][lane] > w.hd[ch][lane]) ch++;
                  if (!(w.hd[ch][lane] > d2)) break;
                  w.hd[pos][lane] = w.hd[ch][lane];
                  w.hi[pos][lane] = w.hi[ch][lane];
                  pos = ch;
                }
                w.hd[pos][lane] = d2;
                w.hi[pos][lane] = w.sidx[jj];
              }
            }
          }
        }
        __syncwarp();
      }
      if (!ok && lane == 0) atomicOr(status, kErrStack);
      // DensityFn: rsq = the heap's largest d2
      if (act && cnt > 0) {
        const int i = t0 + lane;
        const double rsq = w.hd[0][lane], fBall = sqrt(rsq), ih2 = 4.0 / rsq;
        double dens = 0.0;
        for (int e = 0; e < cnt; e++) dens += kernel_m4(w.hd[e][lane] * ih2) * p.m[w.hi[e][lane]];
        dens /= (0.125 * M_PI * (rsq * fBall));
        density[i] = dens;
        ballsq[i] = rsq;
        if (nbr) {
          for (int e = 0; e < kSphK; e++) {
            nbr[(int64_t)i * kSphK + e] = e < cnt ? w.hi[e][lane] : -1;
            nd2[(int64_t)i * kSphK + e] = e < cnt ? w.hd[e][lane] : -1.0;
          }
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

int sph_k() { return kSphK; }

void launch_sph_pressure(Particles p, const double* density, const double* ballsq, const double* u,
                         const int32_t* nbr, const double* nd2, int64_t n, double* ax, double* ay, double* az,
                         double* pdv, unsigned* status, int grid, cudaStream_t st) {
  note_launch();
  sph_pressure_kernel<<<grid, 256, 0, st>>>(p, density, ballsq, u, nbr, nd2, n, ax, ay, az, pdv, status);
}

void launch_sph_density(Particles p, const Mom* mom, const WalkRec* walk, const int32_t* buckets, int64_t nbuckets,
                        int64_t nnodes, double* density, double* ballsq, int32_t* nbr, double* nd2, unsigned* work,
                        unsigned* status, int grid, cudaStream_t st) {
  note_launch();
  sph_density_kernel<<<grid, kSphWarps * 32, 0, st>>>(p, mom, walk, buckets, nbuckets, nnodes, density, ballsq, nbr,
                                                      nd2, work, status);
}

}  // namespace pt
