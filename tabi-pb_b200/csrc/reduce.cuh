// reduce.cuh -- deterministic device reductions: per-block partial sums in a
// fixed grid, then one block adds the partials in index order.
#pragma once

namespace tabi {
namespace {

constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedThreads = 256;

// ---- deterministic reductions: per-block partials, then one block in order
template <int OP>  // 0: sum|a|, 1: sum a*b, 2: sum a*a
__global__ void __launch_bounds__(kRedThreads) reduce_partial_kernel(const double* a,
                                                                     const double* b, int n,
                                                                     double* part) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = a[i];
    if (OP == 0) acc += fabs(v);
    if (OP == 1) acc = fma(v, b[i], acc);
    if (OP == 2) acc = fma(v, v, acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double s[kRedThreads / 32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kRedThreads / 32; ++k) t += s[k];
    part[blockIdx.x] = t;
  }
}

__global__ void reduce_final_kernel(const double* part, int np, double* out) {
  __shared__ double s[kRedBlocks];
  for (int i = threadIdx.x; i < np; i += blockDim.x) s[i] = part[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < np; ++k) t += s[k];
    *out = t;
  }
}

}  // namespace
}  // namespace tabi
