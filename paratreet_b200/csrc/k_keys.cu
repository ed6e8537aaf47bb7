// k_keys.cu -- bounding box, universe and SFC keys (compiled with -fmad=false).
//
//  K1 bbox_partial / bbox_final: FP64 min/max reduction of the positions
//     (the reference's bbox reduction, src/Reader.C:92,106 and
//     src/Partition.h:368-378) and Driver::remakeUniverse (src/Driver.h:67-80)
//     evaluated by one thread on the device.  min/max are exact, so the
//     result does not depend on the reduction order.
//  K2 make_keys: Decomposition::assignKeys (src/Decomposition.C:58-64):
//     21-bit-per-dimension Morton key in FP64, x most significant, plus the
//     placeholder bit 63; emits the identity payload for the sort.
#include <cfloat>

#include "pt_internal.cuh"

namespace pt {

__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// partial[6 * block + k]: min x,y,z then max x,y,z over the block's slice.
__global__ void __launch_bounds__(256) bbox_partial(const double* __restrict__ x, const double* __restrict__ y,
                                                    const double* __restrict__ z, int64_t n,
                                                    double* __restrict__ partial, unsigned* status) {
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double p[3] = {x[i], y[i], z[i]};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      bad |= !isfinite(p[d]);
      mn[d] = fmin(mn[d], p[d]);
      mx[d] = fmax(mx[d], p[d]);
    }
  }
  if (bad) atomicOr(status, kErrNonFinite);
  __shared__ double s[6][8];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    double a = warp_min(mn[d]), b = warp_max(mx[d]);
    if (lane == 0) { s[d][w] = a; s[3 + d][w] = b; }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    int k = threadIdx.x;
    double v = s[k][0];
    for (int i = 1; i < (int)(blockDim.x >> 5); i++) v = (k < 3) ? fmin(v, s[k][i]) : fmax(v, s[k][i]);
    partial[6 * blockIdx.x + k] = v;
  }
}

// out[0..2] universe lo, out[3..5] universe hi, out[6..11] particle bbox.
__global__ void bbox_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
  __shared__ double s[6];
  if (threadIdx.x < 6) {
    int k = threadIdx.x;
    double v = (k < 3) ? DBL_MAX : -DBL_MAX;
    for (int b = 0; b < nblocks; b++) v = (k < 3) ? fmin(v, partial[6 * b + k]) : fmax(v, partial[6 * b + k]);
    s[k] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // Driver::remakeUniverse, src/Driver.h:67-80
    double sx = s[3] - s[0], sy = s[4] - s[1], sz = s[5] - s[2];
    double m = (sx > sy) ? sx : sy;
    m = (m > sz) ? m : sz;
    const double fEps = 1.0 + 1.91e-6;
    double h = fEps * 0.5 * m;
    for (int d = 0; d < 3; d++) {
      double c = (s[d] + s[3 + d]) / 2.0;
      out[d] = c - h;
      out[3 + d] = c + h;
      out[6 + d] = s[d];
      out[9 + d] = s[3 + d];
    }
  }
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x001f00000000ffffull;
  v = (v | (v << 16)) & 0x001f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__device__ __forceinline__ uint32_t quantize21(double p, double lo, double hi) {
  double t = (p - lo) / (hi - lo);
  double s = t * 2097152.0;
  if (!(s >= 0.0)) return 0u;
  if (s >= 2097151.0) return 2097151u;
  return (uint32_t)s;
}

__global__ void __launch_bounds__(256) make_keys(const double* __restrict__ x, const double* __restrict__ y,
                                                 const double* __restrict__ z, int64_t n,
                                                 const double* __restrict__ uni, uint64_t* __restrict__ key,
                                                 uint32_t* __restrict__ idx) {
  const double lo0 = uni[0], lo1 = uni[1], lo2 = uni[2], hi0 = uni[3], hi1 = uni[4], hi2 = uni[5];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t qx = quantize21(x[i], lo0, hi0), qy = quantize21(y[i], lo1, hi1), qz = quantize21(z[i], lo2, hi2);
    key[i] = (spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz) | (1ull << 63);
    idx[i] = (uint32_t)i;
  }
}

// max |v|^2 over particles as (ordered) uint64 bits of a non-negative double.
__global__ void __launch_bounds__(256) vmax2_kernel(const double* __restrict__ vx, const double* __restrict__ vy,
                                                    const double* __restrict__ vz, int64_t n,
                                                    unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double w = vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i];
    m = fmax(m, w);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

void launch_bbox(const double* x, const double* y, const double* z, int64_t n, double* partial, int nblocks,
                 double* uni, unsigned* status, cudaStream_t st) {
  note_launch();
  bbox_partial<<<nblocks, 256, 0, st>>>(x, y, z, n, partial, status);
  note_launch();
  bbox_final<<<1, 32, 0, st>>>(partial, nblocks, uni);
}

void launch_keys(const double* x, const double* y, const double* z, int64_t n, const double* uni, uint64_t* key,
                 uint32_t* idx, int grid, cudaStream_t st) {
  note_launch();
  make_keys<<<grid, 256, 0, st>>>(x, y, z, n, uni, key, idx);
}

void launch_vmax2(const double* vx, const double* vy, const double* vz, int64_t n, unsigned long long* out,
                  int grid, cudaStream_t st) {
  note_launch();
  vmax2_kernel<<<grid, 256, 0, st>>>(vx, vy, vz, n, out);
}

}  // namespace pt
