// k_sort.cu -- K3 stable LSD radix sort of the 64-bit SFC keys with a uint32
// payload, K4 particle permutation, and the device-wide exclusive scan used
// by the sort and the octree build.
//
// Replaces std::sort(particles) (src/Subtree.h:281, Particle::operator<
// src/Particle.C:61-79), which moves ~170-byte AoS particles; here only the
// 12-byte (key, index) pairs move and the FP64 SoA is gathered once.
//
// Per 8-bit digit pass (8 passes):
//   upsweep   one CTA per 4096-key tile builds a 256-bin histogram in shared
//             memory and writes it digit-major (hist[d * tiles + t]);
//   scan      exclusive scan of the digit-major histogram gives every
//             (digit, tile) its global output offset;
//   downsweep each warp ranks its 512 contiguous keys with __match_any_sync
//             (stable: lane order = key order inside a round, rounds in
//             order), the 8 warps' per-digit counts are prefix-summed in
//             shared memory, and each key is scattered to
//             offset[d][tile] + warp prefix + local rank.
// No inter-CTA waiting anywhere: every kernel is independent of scheduling.
#include "pt_internal.cuh"

namespace pt {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;                        // rounds of 32 keys per warp
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys per CTA

__global__ void __launch_bounds__(kSortThreads) radix_upsweep(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                              uint32_t* __restrict__ hist, int tiles) {
  __shared__ uint32_t cnt[kSortWarps][256];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&cnt[0][0])[i] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; r++) {
    int64_t i = base + (int64_t)w * (32 * kSortRounds) + r * 32 + lane;
    if (i < n) atomicAdd(&cnt[w][(keys[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  uint32_t s = 0;
  for (int k = 0; k < kSortWarps; k++) s += cnt[k][threadIdx.x];
  hist[(int64_t)threadIdx.x * tiles + blockIdx.x] = s;
}

__global__ void __launch_bounds__(kSortThreads) radix_downsweep(const uint64_t* __restrict__ kin,
                                                                const uint32_t* __restrict__ vin,
                                                                uint64_t* __restrict__ kout,
                                                                uint32_t* __restrict__ vout, int64_t n, int shift,
                                                                const uint32_t* __restrict__ offs, int tiles) {
  __shared__ uint32_t wh[kSortWarps][256];
  __shared__ uint32_t gbase[256];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&wh[0][0])[i] = 0;
  gbase[threadIdx.x] = offs[(int64_t)threadIdx.x * tiles + blockIdx.x];
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)w * (32 * kSortRounds);
  uint64_t k[kSortRounds];
  uint32_t v[kSortRounds];
  uint32_t rank[kSortRounds];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    int64_t i = base + r * 32 + lane;
    bool ok = i < n;
    k[r] = ok ? kin[i] : 0ull;
    v[r] = ok ? vin[i] : 0u;
    uint32_t d = ok ? (uint32_t)((k[r] >> shift) & 0xff) : (256u + lane);
    unsigned peers = __match_any_sync(0xffffffffu, d);
    uint32_t before = 0;
    if (ok) before = wh[w][d];
    rank[r] = before + __popc(peers & lt);
    __syncwarp();
    if (ok && (31 - __clz(peers)) == lane) wh[w][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    uint32_t run = 0;
    int d = threadIdx.x;
    for (int q = 0; q < kSortWarps; q++) {
      uint32_t t = wh[q][d];
      wh[q][d] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    int64_t i = base + r * 32 + lane;
    if (i < n) {
      uint32_t d = (uint32_t)((k[r] >> shift) & 0xff);
      uint32_t dst = gbase[d] + wh[w][d] + rank[r];
      kout[dst] = k[r];
      vout[dst] = v[r];
    }
  }
}

// ---------------------------------------------------------------- scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Exclusive scan of one tile; writes the tile total to sums[blockIdx.x].
__global__ void __launch_bounds__(kScanThreads) scan_tiles(const uint32_t* in, uint32_t* out,
                                                           int64_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t wsum[kScanThreads / 32];
  int64_t base = (int64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t t = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    int64_t i = base + j;
    v[j] = (i < n) ? in[i] : 0u;
    t += v[j];
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = t;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t s = (lane < kScanThreads / 32) ? wsum[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanThreads / 32) wsum[lane] = s;
  }
  __syncthreads();
  uint32_t run = inc - t + (w ? wsum[w - 1] : 0u);
#pragma unroll
  for (int j = 0; j < kScanItems; j++) {
    int64_t i = base + j;
    if (i < n) out[i] = run;
    run += v[j];
  }
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = run;
}

__global__ void __launch_bounds__(kScanThreads) scan_add(uint32_t* __restrict__ out, int64_t n,
                                                         const uint32_t* __restrict__ sums) {
  uint32_t a = sums[blockIdx.x];
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  for (int j = threadIdx.x; j < kScanTile; j += kScanThreads) {
    int64_t i = base + j;
    if (i < n) out[i] += a;
  }
}

__global__ void scan_total(const uint32_t* __restrict__ in, const uint32_t* __restrict__ out, int64_t n,
                           uint32_t* total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *total = (n > 0) ? out[n - 1] + in[n - 1] : 0u;
}

// Bytes of scratch scan_exclusive needs for n elements.
size_t scan_scratch_bytes(int64_t n) {
  size_t b = 0;
  int64_t m = n;
  do {
    m = (m + kScanTile - 1) / kScanTile;
    b += (size_t)(m + 17) * sizeof(uint32_t);
  } while (m > 1);
  return b + 64;
}

// out[i] = sum_{j<i} in[j]; *total (device) = sum of all.  in may equal out.
void scan_exclusive(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* scratch, uint32_t* total,
                    cudaStream_t st) {
  if (n <= 0) {
    cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
    return;
  }
  // keep the last input element for the total before an in-place scan
  uint32_t* last = scratch;
  cudaMemcpyAsync(last, in + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
  uint32_t* sums = scratch + 16;
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  scan_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, sums);
  if (tiles > 1) {
    scan_exclusive(sums, sums, tiles, sums + tiles + 1, sums + tiles, st);
    scan_add<<<(unsigned)tiles, kScanThreads, 0, st>>>(out, n, sums);
  }
  scan_total<<<1, 32, 0, st>>>(last, out + (n - 1), 1, total);
}

// ---------------------------------------------------------------- sort driver
size_t sort_hist_elems(int64_t n) {
  int64_t tiles = (n + kSortTile - 1) / kSortTile;
  return (size_t)tiles * 256;
}

// Sorts (k0, v0) in place by full 64-bit key using (k1, v1) as alternates.
// hist: sort_hist_elems(n) uint32; scratch: scan scratch for that many.
void radix_sort_pairs(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, int64_t n, uint32_t* hist,
                      uint32_t* scratch, uint32_t* total, cudaStream_t st) {
  if (n <= 1) return;
  int tiles = (int)((n + kSortTile - 1) / kSortTile);
  uint64_t *ka = k0, *kb = k1;
  uint32_t *va = v0, *vb = v1;
  for (int pass = 0; pass < 8; pass++) {
    int shift = 8 * pass;
    radix_upsweep<<<tiles, kSortThreads, 0, st>>>(ka, n, shift, hist, tiles);
    scan_exclusive(hist, hist, (int64_t)tiles * 256, scratch, total, st);
    radix_downsweep<<<tiles, kSortThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist, tiles);
    uint64_t* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  // 8 passes: the result is back in (k0, v0)
}

// ---------------------------------------------------------------- permute
template <typename T>
__global__ void __launch_bounds__(256) gather_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                     const uint32_t* __restrict__ idx, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[idx[i]];
}

void gather_f64(const double* in, double* out, const uint32_t* idx, int64_t n, int grid, cudaStream_t st) {
  gather_kernel<double><<<grid, 256, 0, st>>>(in, out, idx, n);
}
void gather_i32(const int32_t* in, int32_t* out, const uint32_t* idx, int64_t n, int grid, cudaStream_t st) {
  gather_kernel<int32_t><<<grid, 256, 0, st>>>(in, out, idx, n);
}

}  // namespace pt
