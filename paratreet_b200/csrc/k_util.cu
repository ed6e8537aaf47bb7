// k_util.cu -- small data-movement kernels: sorted-order <-> caller-order.
#include "pt_internal.cuh"

namespace pt {

template <typename T>
__global__ void __launch_bounds__(256) scatter_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                      const int32_t* __restrict__ order, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[order[i]] = in[i];
}

__global__ void __launch_bounds__(256) iota_kernel(int32_t* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)i;
}

__global__ void __launch_bounds__(256) inverse_kernel(const int32_t* __restrict__ order, int32_t* __restrict__ inv,
                                                      int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    inv[order[i]] = (int32_t)i;
}

__global__ void __launch_bounds__(256) map_kernel(const int32_t* __restrict__ inv, const int32_t* __restrict__ in,
                                                  int32_t* __restrict__ out, int64_t n) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = inv[in[i]];
}

// y += alpha * x for three arrays (the chain's kick and drift, caller order).
__global__ void __launch_bounds__(256) axpy3_kernel(int64_t n, double alpha, const double* __restrict__ x0,
                                                    const double* __restrict__ x1, const double* __restrict__ x2,
                                                    double* __restrict__ y0, double* __restrict__ y1,
                                                    double* __restrict__ y2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    y0[i] += alpha * x0[i];
    y1[i] += alpha * x1[i];
    y2[i] += alpha * x2[i];
  }
}

// out[i] = in[idx[i]] with a signed permutation (sorted slot -> caller index).
__global__ void __launch_bounds__(256) gather_by_order(const double* __restrict__ in, double* __restrict__ out,
                                                       const int32_t* __restrict__ order, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[order[i]];
}

__global__ void __launch_bounds__(256) axpy1_kernel(int64_t n, double alpha, const double* __restrict__ x,
                                                    double* __restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += alpha * x[i];
}

void launch_axpy1(int64_t n, double alpha, const double* x, double* y, int grid, cudaStream_t st) {
  if (n > 0) { note_launch(); axpy1_kernel<<<grid, 256, 0, st>>>(n, alpha, x, y); }
}
void launch_axpy3(int64_t n, double alpha, const double* x0, const double* x1, const double* x2, double* y0,
                  double* y1, double* y2, int grid, cudaStream_t st) {
  if (n > 0) { note_launch(); axpy3_kernel<<<grid, 256, 0, st>>>(n, alpha, x0, x1, x2, y0, y1, y2); }
}
void launch_gather_by_order(const double* in, double* out, const int32_t* order, int64_t n, int grid,
                            cudaStream_t st) {
  if (n > 0) { note_launch(); gather_by_order<<<grid, 256, 0, st>>>(in, out, order, n); }
}

void launch_scatter_f64(const double* in, double* out, const int32_t* order, int64_t n, int grid, cudaStream_t st) {
  if (n > 0) { note_launch(); scatter_kernel<double><<<grid, 256, 0, st>>>(in, out, order, n); }
}
void launch_scatter_u64(const uint64_t* in, uint64_t* out, const int32_t* order, int64_t n, int grid,
                        cudaStream_t st) {
  if (n > 0) { note_launch(); scatter_kernel<uint64_t><<<grid, 256, 0, st>>>(in, out, order, n); }
}
void launch_iota_i32(int32_t* out, int64_t n, int grid, cudaStream_t st) {
  if (n > 0) { note_launch(); iota_kernel<<<grid, 256, 0, st>>>(out, n); }
}
void launch_inverse_perm(const int32_t* order, int32_t* inv, int64_t n, int grid, cudaStream_t st) {
  if (n > 0) { note_launch(); inverse_kernel<<<grid, 256, 0, st>>>(order, inv, n); }
}
void launch_map_index(const int32_t* inv, const int32_t* in, int32_t* out, int64_t n, cudaStream_t st) {
  if (n > 0) { note_launch(); map_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(inv, in, out, n); }
}

// ------------------------------------------------- interaction-list digests
// Order-independent digest of one bucket's interaction list: the sum (mod
// 2^64) of a 64-bit mix of (node, class) over its entries, class 0 = P2P leaf,
// 1 = quadrupole P2C node, 2 = monopole P2C node (the near flags of the
// two-phase lists are not part of it).  Equal lists give equal digests
// whatever their order.
__device__ __forceinline__ unsigned long long entry_mix(unsigned node, unsigned cls) {
  unsigned long long z = (((unsigned long long)node << 2) | cls) + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Recorded lists (CSR: list_off, node, kind 0 / 1 / 2), one warp per bucket.
__global__ void __launch_bounds__(256) digest_recorded(const int64_t* __restrict__ off,
                                                       const int32_t* __restrict__ node,
                                                       const int8_t* __restrict__ kind, int64_t nb,
                                                       unsigned long long* __restrict__ dig,
                                                       int64_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (b >= nb) return;
  const int64_t e0 = off[b], e1 = off[b + 1];
  unsigned long long s = 0;
  for (int64_t e = e0 + lane; e < e1; e += 32) s += entry_mix((unsigned)node[e], (unsigned)kind[e]);
  s = warp_sum_u64(s);
  if (lane == 0) {
    dig[b] = s;
    cnt[b] = e1 - e0;
  }
}

// Two-phase lists: per bucket a P2C run (bit 31 monopole, bit 30 near) and a
// P2P run (bit 31 near) in the pools, one warp per bucket.
__global__ void __launch_bounds__(256) digest_two_phase(const int32_t* __restrict__ pc_pool,
                                                        const int32_t* __restrict__ pp_pool,
                                                        const int64_t* __restrict__ pc_start,
                                                        const int32_t* __restrict__ pc_count,
                                                        const int64_t* __restrict__ pp_start,
                                                        const int32_t* __restrict__ pp_count, int64_t nb,
                                                        unsigned long long* __restrict__ dig,
                                                        int64_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (b >= nb) return;
  unsigned long long s = 0;
  const int64_t c0 = pc_start[b], p0 = pp_start[b];
  const int nc = pc_count[b], np = pp_count[b];
  for (int k = lane; k < nc; k += 32) {
    const int e = pc_pool[c0 + k];
    s += entry_mix((unsigned)(e & 0x3fffffff), e < 0 ? 2u : 1u);
  }
  for (int k = lane; k < np; k += 32) s += entry_mix((unsigned)(pp_pool[p0 + k] & 0x7fffffff), 0u);
  s = warp_sum_u64(s);
  if (lane == 0) {
    dig[b] = s;
    cnt[b] = (int64_t)nc + np;
  }
}

// The two-phase pools as CSR lists: per bucket its P2P leaves (kind 0), then
// its P2C nodes (kind 1 quadrupole, 2 monopole), one warp per bucket.
__global__ void __launch_bounds__(256) pools_to_csr(const int32_t* __restrict__ pc_pool,
                                                    const int32_t* __restrict__ pp_pool,
                                                    const int64_t* __restrict__ pc_start,
                                                    const int32_t* __restrict__ pc_count,
                                                    const int64_t* __restrict__ pp_start,
                                                    const int32_t* __restrict__ pp_count, int64_t nb,
                                                    const int64_t* __restrict__ off, int32_t* __restrict__ node,
                                                    int8_t* __restrict__ kind) {
  const int lane = threadIdx.x & 31;
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (b >= nb) return;
  const int64_t o = off[b], c0 = pc_start[b], p0 = pp_start[b];
  const int nc = pc_count[b], np = pp_count[b];
  for (int k = lane; k < np; k += 32) {
    node[o + k] = pp_pool[p0 + k] & 0x7fffffff;
    kind[o + k] = 0;
  }
  for (int k = lane; k < nc; k += 32) {
    const int e = pc_pool[c0 + k];
    node[o + np + k] = e & 0x3fffffff;
    kind[o + np + k] = (int8_t)(e < 0 ? 2 : 1);
  }
}

void launch_pools_to_csr(const int32_t* pc_pool, const int32_t* pp_pool, const int64_t* pc_start,
                         const int32_t* pc_count, const int64_t* pp_start, const int32_t* pp_count, int64_t nb,
                         const int64_t* off, int32_t* node, int8_t* kind, cudaStream_t st) {
  if (nb > 0) {
    note_launch();
    pools_to_csr<<<(unsigned)((nb * 32 + 255) / 256), 256, 0, st>>>(pc_pool, pp_pool, pc_start, pc_count, pp_start,
                                                                   pp_count, nb, off, node, kind);
  }
}

void launch_digest_recorded(const int64_t* off, const int32_t* node, const int8_t* kind, int64_t nb,
                            unsigned long long* dig, int64_t* cnt, cudaStream_t st) {
  if (nb > 0) {
    note_launch();
    digest_recorded<<<(unsigned)((nb * 32 + 255) / 256), 256, 0, st>>>(off, node, kind, nb, dig, cnt);
  }
}
void launch_digest_two_phase(const int32_t* pc_pool, const int32_t* pp_pool, const int64_t* pc_start,
                             const int32_t* pc_count, const int64_t* pp_start, const int32_t* pp_count, int64_t nb,
                             unsigned long long* dig, int64_t* cnt, cudaStream_t st) {
  if (nb > 0) {
    note_launch();
    digest_two_phase<<<(unsigned)((nb * 32 + 255) / 256), 256, 0, st>>>(pc_pool, pp_pool, pc_start, pc_count,
                                                                       pp_start, pp_count, nb, dig, cnt);
  }
}

}  // namespace pt
