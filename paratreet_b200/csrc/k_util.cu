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

}  // namespace pt
