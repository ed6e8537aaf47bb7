// k_ewald.cu -- periodic gravity: the Ewald correction applied after the
// replica walks, and an FP64 periodic (Ewald) direct sum used as the force
// error yardstick.  FP64; compiled with -fmad=false.
//
// ewald_correction restates LeafEwaldFn (examples/Ewald.h:3-199,
// non-HEXADECAPOLE branch) per particle: the root cell's monopole and
// quadrupole (about the root centre of mass) are summed over real-space images
// within rcut*L (images inside the replica hole, already walked by the tree,
// contribute -erf instead of erfc, i.e. Ewald minus direct) and over the
// reciprocal-space table built on the host as in EwaldData::EwaldInit
// (examples/Ewald.C:80-163).  alpha = 2/L; close to the origin the series
// expansion of the reference is used (r^2 < 1.2e-3 L^2).  One thread per
// particle: the work is ~(2*ceil(rcut)+1)^3 image terms plus n_h table terms,
// all from registers, so the kernel is FP64-pipe bound, not memory bound.
#include "pt_internal.cuh"
#include "pt_fp64.cuh"

namespace pt {

__global__ void __launch_bounds__(128) ewald_correction(Particles p, int64_t i0, int64_t i1, EwaldRoot R,
                                                        const double4* __restrict__ htab) {
  const int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= i1) return;
  const double L = R.L;
  const double Q2 = 0.5 * (R.xx + R.yy + R.zz);
  int nEwReps = (int)ceil(R.rcut);
  nEwReps = nEwReps > R.n_replicas ? nEwReps : R.n_replicas;
  const double fEwCut2 = R.rcut * R.rcut * L * L;
  const double fInner2 = 1.2e-3 * L * L;
  const double alpha = 2.0 / L;
  const double alpha2 = alpha * alpha;
  const double k1 = M_PI / (alpha2 * L * L * L);
  const double ka = 2.0 * alpha / sqrt(M_PI);
  double fPot = R.mass * k1;
  double ax = 0.0, ay = 0.0, az = 0.0;
  const double dx = p.x[i] - R.cm[0], dy = p.y[i] - R.cm[1], dz = p.z[i] - R.cm[2];
  for (int ix = -nEwReps; ix <= nEwReps; ++ix) {
    const bool inx = (ix >= -R.n_replicas && ix <= R.n_replicas);
    const double x = dx + ix * L;
    for (int iy = -nEwReps; iy <= nEwReps; ++iy) {
      const bool inxy = (inx && iy >= -R.n_replicas && iy <= R.n_replicas);
      const double y = dy + iy * L;
      for (int iz = -nEwReps; iz <= nEwReps; ++iz) {
        const bool hole = (inxy && iz >= -R.n_replicas && iz <= R.n_replicas);
        const double z = dz + iz * L;
        double r2 = x * x + y * y + z * z;
        if (r2 > fEwCut2 && !hole) continue;
        double g0, g1, g2, g3;
        if (r2 < fInner2) {  // series about the origin
          double alphan = ka;
          r2 *= alpha2;
          g0 = alphan * ((1.0 / 3.0) * r2 - 1.0);
          alphan *= 2 * alpha2;
          g1 = alphan * ((1.0 / 5.0) * r2 - (1.0 / 3.0));
          alphan *= 2 * alpha2;
          g2 = alphan * ((1.0 / 7.0) * r2 - (1.0 / 5.0));
          alphan *= 2 * alpha2;
          g3 = alphan * ((1.0 / 9.0) * r2 - (1.0 / 7.0));
        } else {
          const double dir = 1 / sqrt(r2);
          const double dir2 = dir * dir;
          double a = exp(-r2 * alpha2);
          a *= ka * dir2;
          g0 = hole ? -erf(alpha / dir) : erfc(alpha / dir);
          g0 *= dir;
          g1 = g0 * dir2 + a;
          double alphan = 2 * alpha2;
          g2 = 3 * g1 * dir2 + alphan * a;
          alphan *= 2 * alpha2;
          g3 = 5 * g2 * dir2 + alphan * a;
        }
        const double Q2mirx = R.xx * x + R.xy * y + R.xz * z;
        const double Q2miry = R.xy * x + R.yy * y + R.yz * z;
        const double Q2mirz = R.xz * x + R.yz * y + R.zz * z;
        const double Q2mir = 0.5 * (Q2mirx * x + Q2miry * y + Q2mirz * z);
        const double Qta = g1 * R.mass - g2 * Q2 + g3 * Q2mir;
        fPot -= g0 * R.mass - g1 * Q2 + g2 * Q2mir;
        ax += g2 * (Q2mirx) - x * Qta;
        ay += g2 * (Q2miry) - y * Qta;
        az += g2 * (Q2mirz) - z * Qta;
      }
    }
  }
  for (int h = 0; h < R.n_h; ++h) {  // reciprocal space
    const double4 e = htab[h];        // hx, hy, hz (2 pi / L units), hCfac (hSfac = 0 without HEXADECAPOLE)
    const double hdotx = e.x * dx + e.y * dy + e.z * dz;
    double s, c;
    sincos(hdotx, &s, &c);
    fPot += e.w * c;
    ax += e.x * (e.w * s);
    ay += e.y * (e.w * s);
    az += e.z * (e.w * s);
  }
  p.pot[i] += fPot;
  p.potf[i] += fPot;
  p.ax[i] += ax;
  p.ay[i] += ay;
  p.az[i] += az;
}

// ---------------------------------------------------------------- yardstick
// Reciprocal structure factors S(k) = sum_j m_j (cos k.x_j, sin k.x_j), one
// block per k vector.
__global__ void __launch_bounds__(256) ewald_structure(const double* __restrict__ x, const double* __restrict__ y,
                                                       const double* __restrict__ z, const double* __restrict__ m,
                                                       int64_t n, const double4* __restrict__ kv, int nk,
                                                       double* __restrict__ S) {
  const int k = blockIdx.x;
  if (k >= nk) return;
  const double4 K = kv[k];
  double sc = 0.0, ss = 0.0;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    double s, c;
    sincos(K.x * x[j] + K.y * y[j] + K.z * z[j], &s, &c);
    sc += m[j] * c;
    ss += m[j] * s;
  }
  __shared__ double rc[256], rs[256];
  rc[threadIdx.x] = sc;
  rs[threadIdx.x] = ss;
  __syncthreads();
  for (int o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) {
      rc[threadIdx.x] += rc[threadIdx.x + o];
      rs[threadIdx.x] += rs[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    S[2 * k] = rc[0];
    S[2 * k + 1] = rs[0];
  }
}

constexpr int kEwTile = 128;

// Real-space part + minimum-image spline correction, source-sliced partials
// (blockIdx.y = source slice; the host adds the slices in a fixed order).
__global__ void __launch_bounds__(kEwTile) ewald_real(const double* __restrict__ x, const double* __restrict__ y,
                                                      const double* __restrict__ z, const double* __restrict__ m,
                                                      const double* __restrict__ soft, int64_t n,
                                                      const int32_t* __restrict__ tgt, int64_t nt, int nsplit,
                                                      double L, double alpha, double rcut,
                                                      double* __restrict__ part) {
  __shared__ double sx[kEwTile], sy[kEwTile], sz[kEwTile], sm[kEwTile], ss[kEwTile];
  const int64_t t = blockIdx.x * (int64_t)kEwTile + threadIdx.x;
  const bool ok = t < nt;
  const int i = ok ? tgt[t] : 0;
  const double xi = x[i], yi = y[i], zi = z[i], si = soft[i];
  const double rc2 = rcut * rcut;
  const double ka = 2.0 * alpha / sqrt(M_PI);
  const int nimg = (int)ceil(rcut / L + 0.5);
  double ax = 0.0, ay = 0.0, az = 0.0, pp = 0.0;
  const int64_t per = (n + nsplit - 1) / nsplit;
  const int64_t j0 = per * blockIdx.y, j1 = min(n, j0 + per);
  for (int64_t base = j0; base < j1; base += kEwTile) {
    __syncthreads();
    const int64_t j = base + threadIdx.x;
    if (j < j1) {
      sx[threadIdx.x] = x[j];
      sy[threadIdx.x] = y[j];
      sz[threadIdx.x] = z[j];
      sm[threadIdx.x] = m[j];
      ss[threadIdx.x] = soft[j];
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kEwTile, j1 - base);
    if (!ok) continue;
    for (int k = 0; k < cnt; k++) {
      // minimum image first
      double d0x = sx[k] - xi, d0y = sy[k] - yi, d0z = sz[k] - zi;
      d0x -= L * rint(d0x / L);
      d0y -= L * rint(d0y / L);
      d0z -= L * rint(d0z / L);
      const double mj = sm[k];
      for (int a = -nimg; a <= nimg; a++) {
        const double dx = d0x + a * L;
        if (dx * dx > rc2) continue;
        for (int b = -nimg; b <= nimg; b++) {
          const double dy = d0y + b * L;
          if (dx * dx + dy * dy > rc2) continue;
          for (int c = -nimg; c <= nimg; c++) {
            const double dz = d0z + c * L;
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > rc2 || r2 == 0.0) continue;
            const double r = sqrt(r2);
            const double ec = erfc(alpha * r);
            const double f = (ec + ka * r * exp(-alpha * alpha * r2)) / (r2 * r);
            ax += mj * f * dx;
            ay += mj * f * dy;
            az += mj * f * dz;
            pp -= mj * ec / r;
          }
        }
      }
      // spline softening for the nearest image, as the tree evaluates it
      const double r2 = d0x * d0x + d0y * d0y + d0z * d0z;
      const double twoh = ss[k] + si;
      if (r2 != 0.0 && r2 < twoh * twoh) {
        double a, b;
        spline_f64(r2, twoh, a, b);
        const double r = sqrt(r2);
        const double corr = b - 1.0 / (r2 * r);
        ax += mj * corr * d0x;
        ay += mj * corr * d0y;
        az += mj * corr * d0z;
        pp -= mj * (a - 1.0 / r);
      }
    }
  }
  if (ok) {
    double* o = part + ((int64_t)blockIdx.y * nt + t) * 4;
    o[0] = ax;
    o[1] = ay;
    o[2] = az;
    o[3] = pp;
  }
}

// Reciprocal part for each target from the structure factors; S[2 nk] holds
// the total mass M (the k = 0 "structure factor").  The potential also gets the
// neutralising-background constant pi M / (alpha^2 V) and the self-image term
// 2 alpha m_i / sqrt(pi) (the reciprocal sum includes the target's own mass).
__global__ void __launch_bounds__(128) ewald_recip(const double* __restrict__ x, const double* __restrict__ y,
                                                   const double* __restrict__ z, const double* __restrict__ m,
                                                   const int32_t* __restrict__ tgt, int64_t nt,
                                                   const double4* __restrict__ kv, int nk,
                                                   const double* __restrict__ S, double alpha, double V,
                                                   double* __restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int i = tgt[t];
  double ax = 0.0, ay = 0.0, az = 0.0;
  double pp = M_PI * S[2 * nk] / (alpha * alpha * V) + 2.0 * alpha / sqrt(M_PI) * m[i];
  for (int k = 0; k < nk; k++) {
    const double4 K = kv[k];  // kx, ky, kz, 4 pi / V * exp(-k^2 / 4 alpha^2) / k^2
    double s, c;
    sincos(K.x * x[i] + K.y * y[i] + K.z * z[i], &s, &c);
    const double sc = S[2 * k], ss = S[2 * k + 1];
    const double f = K.w * (s * sc - c * ss);
    ax -= f * K.x;
    ay -= f * K.y;
    az -= f * K.z;
    pp -= K.w * (c * sc + s * ss);
  }
  out[4 * t + 0] = ax;
  out[4 * t + 1] = ay;
  out[4 * t + 2] = az;
  out[4 * t + 3] = pp;
}

void launch_ewald_correction(Particles p, int64_t i0, int64_t i1, const EwaldRoot& R, const double4* htab,
                             cudaStream_t st) {
  if (i1 > i0) { note_launch(); ewald_correction<<<(unsigned)((i1 - i0 + 127) / 128), 128, 0, st>>>(p, i0, i1, R, htab); }
}
void launch_ewald_structure(const double* x, const double* y, const double* z, const double* m, int64_t n,
                            const double4* kv, int nk, double* S, cudaStream_t st) {
  if (nk > 0) { note_launch(); ewald_structure<<<nk, 256, 0, st>>>(x, y, z, m, n, kv, nk, S); }
}
void launch_ewald_real(const double* x, const double* y, const double* z, const double* m, const double* soft,
                       int64_t n, const int32_t* tgt, int64_t nt, int nsplit, double L, double alpha, double rcut,
                       double* part, cudaStream_t st) {
  dim3 grid((unsigned)((nt + kEwTile - 1) / kEwTile), nsplit);
  if (nt > 0) { note_launch(); ewald_real<<<grid, kEwTile, 0, st>>>(x, y, z, m, soft, n, tgt, nt, nsplit, L, alpha, rcut, part); }
}
void launch_ewald_recip(const double* x, const double* y, const double* z, const double* m, const int32_t* tgt,
                        int64_t nt, const double4* kv, int nk, const double* S, double alpha, double V, double* out,
                        cudaStream_t st) {
  if (nt > 0) {
    note_launch();
    ewald_recip<<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(x, y, z, m, tgt, nt, kv, nk, S, alpha, V, out);
  }
}

}  // namespace pt
