// k_sort.cu -- K3 stable LSD radix sort of the 64-bit SFC keys with a uint32
// payload (onesweep), K4 particle permutation, and the device-wide exclusive
// scan used by the octree build.
//
// Replaces std::sort(particles) (src/Subtree.h:281, Particle::operator<
// src/Particle.C:61-79), which moves ~170-byte AoS particles; here only the
// 12-byte (key, index) pairs move and the FP64 SoA is gathered once.
//
// Onesweep (one read and one write of the pairs per 8-bit digit):
//   histogram  one pass over the keys builds all eight 256-bin digit
//              histograms (shared-memory atomics, then global atomics), and
//              one small kernel turns each into exclusive digit offsets;
//   pass       per digit, each CTA claims the next 4096-key tile from an atomic
//              counter (so every earlier tile is already running), ranks its
//              keys stably with __match_any_sync (lane order = key order in a
//              round, rounds and warps in order), publishes its per-digit
//              counts, and resolves the counts of all earlier tiles by
//              decoupled look-back on 64-bit status words (flag | count).  The
//              ranked tile is staged in shared memory and written out with
//              consecutive threads on consecutive destinations.
// The look-back only waits on tiles that claimed their index earlier and
// publish their counts before waiting on anything, so it always ends; the spin
// is still bounded (spin_limit polls of an unpublished tile, 2^21 by default)
// and reports kErrSort instead of hanging.  A look-back cut short only
// under-counts a digit's exclusive prefix, so every destination stays inside
// [0, n), but the output is then not a permutation: the caller checks the
// status word before it uses the sorted indices.
#include <algorithm>

#include "pt_internal.cuh"

namespace pt {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;                        // rounds of 32 keys per warp
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys per CTA
constexpr unsigned long long kFlagAggregate = 1ull << 32;
constexpr unsigned long long kFlagInclusive = 2ull << 32;

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// All eight digit histograms in one read of the keys.
__global__ void __launch_bounds__(kSortThreads) radix_histograms(const uint64_t* __restrict__ keys, int64_t n,
                                                                 uint32_t* __restrict__ ghist) {
  __shared__ uint32_t h[8][256];
  for (int i = threadIdx.x; i < 8 * 256; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)kSortThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kSortThreads) {
    const uint64_t k = keys[i];
#pragma unroll
    for (int p = 0; p < 8; p++) atomicAdd(&h[p][(k >> (8 * p)) & 0xff], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * 256; i += kSortThreads) {
    const uint32_t c = (&h[0][0])[i];
    if (c) atomicAdd(&ghist[i], c);
  }
}

// Exclusive scan of each 256-bin histogram in place (block p = digit pass p).
__global__ void __launch_bounds__(256) radix_digit_offsets(uint32_t* __restrict__ ghist) {
  __shared__ uint32_t ws[8];
  uint32_t* g = ghist + blockIdx.x * 256;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t v = g[threadIdx.x];
  uint32_t inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) ws[w] = inc;
  __syncthreads();
  uint32_t base = 0;
  for (int q = 0; q < w; q++) base += ws[q];
  g[threadIdx.x] = base + inc - v;
}

struct OnesweepShared {
  uint32_t wh[kSortWarps][256];  // per-warp digit counts, then their warp prefixes
  uint32_t dstart[256];          // tile-local start of each digit
  uint32_t gbase[256];           // global destination of each digit's first key of this tile
  uint32_t wsum[kSortWarps];
  int tile;
  uint64_t key[kSortTile];
  uint32_t val[kSortTile];
};

__global__ void __launch_bounds__(kSortThreads, 2) radix_onesweep(const uint64_t* __restrict__ kin,
                                                                  const uint32_t* __restrict__ vin,
                                                                  uint64_t* __restrict__ kout,
                                                                  uint32_t* __restrict__ vout, int64_t n, int shift,
                                                                  const uint32_t* __restrict__ gofs,
                                                                  uint32_t* __restrict__ counter,
                                                                  unsigned long long* __restrict__ look,
                                                                  unsigned* __restrict__ status, long long spin_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  OnesweepShared& S = *reinterpret_cast<OnesweepShared*>(smem_raw);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&S.wh[0][0])[i] = 0;
  if (threadIdx.x == 0) S.tile = (int)atomicAdd(counter, 1u);
  __syncthreads();
  const int tile = S.tile;
  const int64_t tbase = (int64_t)tile * kSortTile;
  const int64_t base = tbase + (int64_t)w * (32 * kSortRounds);
  uint64_t k[kSortRounds];
  uint32_t v[kSortRounds];
  uint32_t rank[kSortRounds];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    const int64_t i = base + r * 32 + lane;
    const bool ok = i < n;
    k[r] = ok ? kin[i] : 0ull;
    v[r] = ok ? vin[i] : 0u;
    const uint32_t d = ok ? (uint32_t)((k[r] >> shift) & 0xff) : (256u + lane);
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    uint32_t before = 0;
    if (ok) before = S.wh[w][d];
    rank[r] = before + __popc(peers & lt);
    __syncwarp();
    if (ok && (31 - __clz(peers)) == lane) S.wh[w][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // thread d: the tile's count of digit d and the warp prefixes
  const int d = threadIdx.x;
  uint32_t total = 0;
  for (int q = 0; q < kSortWarps; q++) {
    const uint32_t t = S.wh[q][d];
    S.wh[q][d] = total;
    total += t;
  }
  unsigned long long* my = look + (int64_t)tile * 256 + d;
  uint32_t excl = 0;
  if (tile == 0) {
    st_relaxed_u64(my, kFlagInclusive | total);
  } else {
    st_relaxed_u64(my, kFlagAggregate | total);
    // decoupled look-back over the earlier tiles
    int64_t pt = tile - 1;
    long long spins = 0;
    while (pt >= 0) {
      const unsigned long long s = ld_relaxed_u64(look + pt * 256 + d);
      const unsigned long long f = s & (3ull << 32);
      if (f == 0) {
        if (++spins > spin_limit) {
          atomicOr(status, kErrSort);
          break;
        }
        __nanosleep(32);
        continue;
      }
      excl += (uint32_t)s;
      if (f == kFlagInclusive) break;
      pt--;
    }
    st_relaxed_u64(my, kFlagInclusive | (unsigned long long)(excl + total));
  }
  S.gbase[d] = gofs[d] + excl;
  // tile-local digit starts: exclusive scan of total over the 256 digits
  {
    uint32_t inc = total;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) S.wsum[w] = inc;
    __syncthreads();
    uint32_t b = 0;
    for (int q = 0; q < w; q++) b += S.wsum[q];
    S.dstart[d] = b + inc - total;
  }
  __syncthreads();
  // stage the ranked tile in shared memory
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    const int64_t i = base + r * 32 + lane;
    if (i < n) {
      const uint32_t dd = (uint32_t)((k[r] >> shift) & 0xff);
      const uint32_t pos = S.dstart[dd] + S.wh[w][dd] + rank[r];
      S.key[pos] = k[r];
      S.val[pos] = v[r];
    }
  }
  __syncthreads();
  const int cnt = (int)min((int64_t)kSortTile, n - tbase);
  for (int i = threadIdx.x; i < cnt; i += kSortThreads) {
    const uint64_t key = S.key[i];
    const uint32_t dd = (uint32_t)((key >> shift) & 0xff);
    const uint32_t dst = S.gbase[dd] + ((uint32_t)i - S.dstart[dd]);
    kout[dst] = key;
    vout[dst] = S.val[i];
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
  note_launch();
  scan_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, n, sums);
  if (tiles > 1) {
    scan_exclusive(sums, sums, tiles, sums + tiles + 1, sums + tiles, st);
    note_launch();
    scan_add<<<(unsigned)tiles, kScanThreads, 0, st>>>(out, n, sums);
  }
  note_launch();
  scan_total<<<1, 32, 0, st>>>(last, out + (n - 1), 1, total);
}

// ---------------------------------------------------------------- sort driver
namespace {
size_t align256(size_t b) { return (b + 255) / 256 * 256; }
}  // namespace

// Scratch of radix_sort_pairs for n keys: eight digit histograms, eight tile
// counters, and one 64-bit look-back word per (tile, digit).
size_t sort_scratch_bytes(int64_t n) {
  const int64_t tiles = (n + kSortTile - 1) / kSortTile;
  return align256(8 * 256 * sizeof(uint32_t)) + align256(8 * sizeof(uint32_t)) +
         align256((size_t)std::max<int64_t>(tiles, 1) * 256 * sizeof(unsigned long long));
}

// Sorts (k0, v0) in place by full 64-bit key using (k1, v1) as alternates.
int radix_sort_pairs(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, int64_t n, void* scratch,
                     unsigned* status, int sms, long long spin_limit, cudaStream_t st) {
  if (n <= 1) return 0;
  const int tiles = (int)((n + kSortTile - 1) / kSortTile);
  unsigned char* b = static_cast<unsigned char*>(scratch);
  uint32_t* ghist = reinterpret_cast<uint32_t*>(b);
  uint32_t* counters = reinterpret_cast<uint32_t*>(b + align256(8 * 256 * sizeof(uint32_t)));
  unsigned long long* look = reinterpret_cast<unsigned long long*>(
      b + align256(8 * 256 * sizeof(uint32_t)) + align256(8 * sizeof(uint32_t)));
  const size_t look_bytes = (size_t)tiles * 256 * sizeof(unsigned long long);
  static_assert(sizeof(OnesweepShared) <= 227 * 1024, "onesweep tile exceeds shared memory");
  if (cudaFuncSetAttribute(radix_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(OnesweepShared)) != cudaSuccess)
    return -1;
  cudaMemsetAsync(ghist, 0, align256(8 * 256 * sizeof(uint32_t)) + align256(8 * sizeof(uint32_t)), st);
  note_launch();
  radix_histograms<<<sms * 4, kSortThreads, 0, st>>>(k0, n, ghist);
  note_launch();
  radix_digit_offsets<<<8, 256, 0, st>>>(ghist);
  uint64_t *ka = k0, *kb = k1;
  uint32_t *va = v0, *vb = v1;
  for (int pass = 0; pass < 8; pass++) {
    cudaMemsetAsync(look, 0, look_bytes, st);
    note_launch();
    radix_onesweep<<<tiles, kSortThreads, sizeof(OnesweepShared), st>>>(
        ka, va, kb, vb, n, 8 * pass, ghist + 256 * pass, counters + pass, look, status, spin_limit);
    uint64_t* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  // 8 passes: the result is back in (k0, v0)
  return 0;
}

// ---------------------------------------------------------------- permute
template <typename T>
__global__ void __launch_bounds__(256) gather_kernel(const T* __restrict__ in, T* __restrict__ out,
                                                     const uint32_t* __restrict__ idx, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[idx[i]];
}

void gather_f64(const double* in, double* out, const uint32_t* idx, int64_t n, int grid, cudaStream_t st) {
  note_launch();
  gather_kernel<double><<<grid, 256, 0, st>>>(in, out, idx, n);
}
void gather_i32(const int32_t* in, int32_t* out, const uint32_t* idx, int64_t n, int grid, cudaStream_t st) {
  note_launch();
  gather_kernel<int32_t><<<grid, 256, 0, st>>>(in, out, idx, n);
}

}  // namespace pt
