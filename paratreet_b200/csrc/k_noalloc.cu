// k_noalloc.cu -- pt_direct_sum_noalloc: the FP64 direct sum for callers that
// cannot allocate device memory (compiled with -fmad=false like k_fp64.cu).
//
// Who needs it: code that drives this library from inside another
// framework's memory discipline -- a time-stepping loop that hands over
// buffers carved from its own pre-sized pool, or an embedding that budgets
// all device memory up front -- must not trigger cudaMalloc / cudaFree, which
// also synchronise the whole device.  Every other entry point works through
// a pt_handle, and creating or growing a handle allocates.  This one takes
// device pointers for all inputs and outputs and keeps its only scratch (the
// per-slice partial sums) in the fixed array below.
//
// The array is a file-scope __device__ variable of kNoAllocScratchBytes
// (8 MiB): every GPU that loads the library holds it until the process exits.
// Host code sees only a stand-in for the symbol, so the device address is
// looked up with cudaGetSymbolAddress, once per device, with that device
// current, on the first call made on that device.  Make that first call
// before any stream capture.  Every call copies the status word to host
// memory and synchronises its stream before it returns.  All calls share the
// array and it keeps the last call's contents: the status word is cleared at
// the start of every call and every partial that is read was written by the
// same call.  Calls whose work
// overlaps on the GPU (different streams, or different host threads on one
// device) race on the array and must be serialised by the caller.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/pt_gravity.h"
#include "pt_fp64.cuh"
#include "pt_internal.cuh"

namespace pt {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
constexpr size_t kNoAllocHeaderBytes = 256;  // status word, then padding
constexpr int64_t kNoAllocPartials = (int64_t)((kNoAllocScratchBytes - kNoAllocHeaderBytes) / sizeof(double));
constexpr int64_t kNoAllocMaxTargets = kNoAllocPartials / 4;  // one slice of 4 sums per target
constexpr int kNoAllocTile = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char noalloc_scratch[kNoAllocScratchBytes];

// Bounds-checked direct sum into per-slice partials (grid: target blocks x slices).
__global__ void __launch_bounds__(kNoAllocTile) noalloc_direct(const double* __restrict__ x, const double* __restrict__ y,
                                                               const double* __restrict__ z, const double* __restrict__ m,
                                                               const double* __restrict__ soft, int64_t n,
                                                               const int32_t* __restrict__ tgt, int64_t nt, int nsplit,
                                                               double* __restrict__ part, unsigned* status) {
  __shared__ double sx[kNoAllocTile], sy[kNoAllocTile], sz[kNoAllocTile], sm[kNoAllocTile], ss[kNoAllocTile];
  const int64_t t = blockIdx.x * (int64_t)kNoAllocTile + threadIdx.x;
  bool ok = t < nt;
  int i = 0;
  if (ok) {
    i = tgt[t];
    if (i < 0 || i >= n) {
      atomicOr(status, 1u);
      ok = false;
      i = 0;
    }
  }
  double xi = 0.0, yi = 0.0, zi = 0.0, si = 0.0;
  if (ok) { xi = x[i]; yi = y[i]; zi = z[i]; si = soft[i]; }
  double ax = 0.0, ay = 0.0, az = 0.0, pp = 0.0;
  const int64_t per = (n + nsplit - 1) / nsplit;
  const int64_t j0 = per * blockIdx.y, j1 = min(n, j0 + per);
  for (int64_t base = j0; base < j1; base += kNoAllocTile) {
    __syncthreads();
    const int64_t j = base + threadIdx.x;
    if (j < j1) { sx[threadIdx.x] = x[j]; sy[threadIdx.x] = y[j]; sz[threadIdx.x] = z[j]; sm[threadIdx.x] = m[j]; ss[threadIdx.x] = soft[j]; }
    __syncthreads();
    const int cnt = (int)min((int64_t)kNoAllocTile, j1 - base);
    if (ok) {
      for (int k = 0; k < cnt; k++) {
        double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
        double rsq = dx * dx + dy * dy + dz * dz;
        if (rsq != 0) {
          double a, b;
          spline_f64(rsq, ss[k] + si, a, b);
          double bm = b * sm[k];
          ax += dx * bm;
          ay += dy * bm;
          az += dz * bm;
          pp += -sm[k] * a;
        }
      }
    }
  }
  if (t < nt) {
    double* o = part + ((int64_t)blockIdx.y * nt + t) * 4;
    o[0] = ax; o[1] = ay; o[2] = az; o[3] = pp;
  }
}

// Sum the slices of each target in slice order (0.0 + s0 + s1 + ...).  When
// the direct-sum kernel flagged a target index outside [0, n), nothing is
// written: the caller's output arrays keep their contents.
__global__ void __launch_bounds__(256) noalloc_reduce(const double* __restrict__ part, int nsplit, int64_t nt,
                                                      double* __restrict__ ax, double* __restrict__ ay,
                                                      double* __restrict__ az, double* __restrict__ pot,
                                                      const unsigned* __restrict__ status) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nt || *status != 0u) return;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int sl = 0; sl < nsplit; sl++)
    for (int k = 0; k < 4; k++) s[k] += part[((int64_t)sl * nt + t) * 4 + k];
  if (ax) ax[t] = s[0];
  if (ay) ay[t] = s[1];
  if (az) az[t] = s[2];
  if (pot) pot[t] = s[3];
}

namespace {
std::mutex g_setup_mu;
unsigned char* g_scratch[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

void put_err(char* buf, size_t len, const char* msg) {
  if (buf && len) {
    std::strncpy(buf, msg, len - 1);
    buf[len - 1] = '\0';
  }
}
}  // namespace

}  // namespace pt

using namespace pt;

extern "C" int pt_direct_sum_noalloc(int64_t n, const double* x, const double* y, const double* z, const double* m,
                                     const double* soft, int64_t nt, const int32_t* targets, double* ax, double* ay,
                                     double* az, double* pot, void* stream, char* errbuf, size_t errlen) {
  put_err(errbuf, errlen, "");
  if (n < 0 || nt < 0 || n > (int64_t)INT32_MAX) {
    put_err(errbuf, errlen, "pt_direct_sum_noalloc: negative or too large n / nt");
    return PT_E_ARG;
  }
  if (nt > kNoAllocMaxTargets) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "pt_direct_sum_noalloc: %lld targets exceed the fixed scratch limit of %lld",
                  (long long)nt, (long long)kNoAllocMaxTargets);
    put_err(errbuf, errlen, msg);
    return PT_E_ARG;
  }
  if (nt == 0) return PT_OK;
  if (n == 0 || !x || !y || !z || !m || !soft || !targets) {
    put_err(errbuf, errlen, "pt_direct_sum_noalloc: null input pointer or no sources");
    return PT_E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    put_err(errbuf, errlen, "pt_direct_sum_noalloc: no usable current CUDA device");
    return PT_E_CUDA;
  }
  unsigned char* base = nullptr;
  int sms = 0;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch[dev]) {  // set-up: once per device, with that device current
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, noalloc_scratch);
      if (e != cudaSuccess || !ptr) {
        put_err(errbuf, errlen, "pt_direct_sum_noalloc: cudaGetSymbolAddress failed");
        return PT_E_CUDA;
      }
      int s = 0;
      if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || s <= 0) s = 148;
      g_sms[dev] = s;
      g_scratch[dev] = static_cast<unsigned char*>(ptr);
    }
    base = g_scratch[dev];
    sms = g_sms[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned* status = reinterpret_cast<unsigned*>(base);
  double* part = reinterpret_cast<double*>(base + kNoAllocHeaderBytes);
  const int tb = (int)((nt + kNoAllocTile - 1) / kNoAllocTile);
  int64_t nsplit = (4 * (int64_t)sms + tb - 1) / tb;
  if (nsplit > 256) nsplit = 256;
  if (nsplit > kNoAllocPartials / (4 * nt)) nsplit = kNoAllocPartials / (4 * nt);
  if (nsplit < 1) nsplit = 1;
  if (cudaMemsetAsync(status, 0, sizeof(unsigned), st) != cudaSuccess) {
    put_err(errbuf, errlen, "pt_direct_sum_noalloc: clearing the status word failed");
    return PT_E_CUDA;
  }
  dim3 grid((unsigned)tb, (unsigned)nsplit);
  note_launch();
  noalloc_direct<<<grid, kNoAllocTile, 0, st>>>(x, y, z, m, soft, n, targets, nt, (int)nsplit, part, status);
  note_launch();
  noalloc_reduce<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(part, (int)nsplit, nt, ax, ay, az, pot, status);
  unsigned h_status = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    put_err(errbuf, errlen, cudaGetErrorString(e));
    return PT_E_CUDA;
  }
  if (h_status) {
    put_err(errbuf, errlen, "pt_direct_sum_noalloc: a target index is outside [0, n)");
    return PT_E_ARG;
  }
  return PT_OK;
}
