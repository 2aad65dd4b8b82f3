// noalloc.cu -- tabi_energy_noalloc: the solvation / Coulomb energy of
// main.f90:144-157 (+ potential_molecule, main.f90:614-657) for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: device memory may be owned and
// budgeted by another allocator (a framework's caching allocator or a fixed
// pool that must not be fragmented), and cudaFree synchronises the whole
// device, which a latency-sensitive pipeline running other streams cannot
// afford.  This entry point therefore allocates nothing: its scratch (the
// per-atom partial potentials and Coulomb sums) is a file-scope static device
// array, g_energy_scratch, of kNoAllocScratch doubles (8 MiB), which every GPU
// that loads this library holds until the process exits.
//
// Host code only ever sees a host-side stand-in for that symbol, so the device
// address is looked up with cudaGetSymbolAddress once per device (on the first
// call made with that device current) and passed to the kernels.  The cached
// address stays valid only while the device's primary context lives: a
// cudaDeviceReset reloads the module elsewhere, so callers must not reset the
// device between calls (the header says so).
#include <cmath>
#include <mutex>

#include "tabi_impl.cuh"

namespace tabi {

namespace {

constexpr size_t kNoAllocScratch = size_t(1) << 20;  // doubles
constexpr int kMaxDevices = 64;
constexpr int kEA = 8;    // atoms per block
constexpr int kET = 256;  // threads per block

static __device__ __align__(256) double g_energy_scratch[kNoAllocScratch];

double* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of g_energy_scratch on the current device (looked up once).
double* scratch_for(int dev) {
  TABI_REQUIRE(dev >= 0 && dev < kMaxDevices, TABI_ERR_LIMIT, "device index above 63");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    TABI_CUDA(cudaGetSymbolAddress(&p, g_energy_scratch));
    TABI_REQUIRE(p != nullptr, TABI_ERR_CUDA, "cudaGetSymbolAddress returned null");
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  return g_scratch_ptr[dev];
}

// potential_molecule for kEA atoms per block, surface in the reference's
// column-major 3 x N layout; partials to part[blockIdx.y * nchr + atom]
__global__ void __launch_bounds__(kET) energy_noalloc_kernel(
    const double* __restrict__ xyz, const double* __restrict__ q,
    const double* __restrict__ area, const double* __restrict__ x, int n,
    const double* __restrict__ chrpos, int nchr, double kappa, double eps,
    double* __restrict__ part) {
  const int a0 = blockIdx.x * kEA;
  double ax[kEA], ay[kEA], az[kEA], acc[kEA];
#pragma unroll
  for (int k = 0; k < kEA; ++k) {
    int a = min(a0 + k, nchr - 1);
    ax[k] = chrpos[3 * (size_t)a];
    ay[k] = chrpos[3 * (size_t)a + 1];
    az[k] = chrpos[3 * (size_t)a + 2];
    acc[k] = 0.0;
  }
  for (int j = blockIdx.y * blockDim.x + threadIdx.x; j < n; j += gridDim.y * blockDim.x) {
    const double rx = xyz[3 * (size_t)j], ry = xyz[3 * (size_t)j + 1],
                 rz = xyz[3 * (size_t)j + 2];
    const double vx = q[3 * (size_t)j], vy = q[3 * (size_t)j + 1], vz = q[3 * (size_t)j + 2];
    const double A = area[j];
    const double w1 = A * x[j], w2 = A * x[n + j];
#pragma unroll
    for (int k = 0; k < kEA; ++k) {
      double dx = rx - ax[k], dy = ry - ay[k], dz = rz - az[k];
      double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      double inv = rsqrt(r2);
      double rs = r2 * inv;
      double G0 = kOneOver4Pi * inv;
      double kr = kappa * rs;
      double e = exp(-kr);
      double c = fma(vx, dx, fma(vy, dy, vz * dz)) * inv;
      double tp1 = G0 * inv;
      double tp2 = (1.0 + kr) * e;
      double H1 = (c * tp1) * fma(-eps, tp2, 1.0);  // G1 - eps G2
      double H2 = G0 * (1.0 - e);                   // G0 - Gk
      acc[k] = fma(H1, w1, fma(H2, w2, acc[k]));
    }
  }
  __shared__ double s[kEA][kET / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kEA; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) s[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < kEA && a0 + (int)threadIdx.x < nchr) {
    double t = 0.0;
    for (int qq = 0; qq < kET / 32; ++qq) t += s[threadIdx.x][qq];
    part[(size_t)blockIdx.y * nchr + a0 + threadIdx.x] = t;
  }
}

// per atom k: sum_{l>k} q_k q_l / (eps0 dist)  (main.f90:149-155)
__global__ void coulomb_noalloc_kernel(const double* __restrict__ chrpos,
                                       const double* __restrict__ atmchr, int nchr,
                                       double eps0, double* __restrict__ out) {
  const int k = blockIdx.x;
  const double xk = chrpos[3 * (size_t)k], yk = chrpos[3 * (size_t)k + 1],
               zk = chrpos[3 * (size_t)k + 2], qk = atmchr[k];
  double acc = 0.0;
  for (int l = k + 1 + threadIdx.x; l < nchr; l += blockDim.x) {
    double dx = xk - chrpos[3 * (size_t)l], dy = yk - chrpos[3 * (size_t)l + 1],
           dz = zk - chrpos[3 * (size_t)l + 2];
    acc += 1.0 / eps0 / sqrt(dx * dx + dy * dy + dz * dz) * qk * atmchr[l];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int qq = 0; qq < (int)(blockDim.x >> 5); ++qq) t += s[qq];
    out[k] = t;
  }
}

// soleng = 1/2 * 332.0716 * 4 pi * sum_k q_k phi_k, couleng = 332.0716 * sum;
// each thread sums a contiguous range of atoms, thread 0 adds the ranges in
// order (deterministic)
__global__ void energy_final_kernel(const double* __restrict__ part, int gy,
                                    const double* __restrict__ cou,
                                    const double* __restrict__ atmchr, int nchr,
                                    double* __restrict__ out) {
  __shared__ double ss[256], sc[256];
  const int per = (nchr + blockDim.x - 1) / blockDim.x;
  const int k0 = threadIdx.x * per, k1 = min(nchr, k0 + per);
  double se = 0.0, ce = 0.0;
  for (int k = k0; k < k1; ++k) {
    double p = 0.0;
    for (int y = 0; y < gy; ++y) p += part[(size_t)y * nchr + k];
    se = fma(atmchr[k], p, se);
    ce += cou[k];
  }
  ss[threadIdx.x] = se;
  sc[threadIdx.x] = ce;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      a += ss[t];
      b += sc[t];
    }
    const double para = 332.0716;
    out[0] = a * 0.5 * para * 4.0 * kPi;
    out[1] = b * para;
  }
}

}  // namespace

void energy_noalloc(int nface, const double* tr_xyz, const double* tr_q, const double* tr_area,
                    const double* x, int nchr, const double* chrpos, const double* atmchr,
                    double kappa, double eps0, double eps1, double* out, cudaStream_t s) {
  TABI_REQUIRE(nface > 0 && nchr > 0, TABI_ERR_ARG, "sizes must be positive");
  TABI_REQUIRE(tr_xyz && tr_q && tr_area && x && chrpos && atmchr && out, TABI_ERR_ARG,
               "null device pointer");
  TABI_REQUIRE(eps0 > 0.0 && eps1 > 0.0 && kappa >= 0.0, TABI_ERR_ARG, "bad physics constants");
  // scratch: gy rows of nchr partial potentials + nchr Coulomb partials
  TABI_REQUIRE((size_t)nchr * 2 <= kNoAllocScratch, TABI_ERR_LIMIT,
               "tabi_energy_noalloc: more than 524288 atoms (scratch of 2^20 doubles)");
  int dev = 0;
  TABI_CUDA(cudaGetDevice(&dev));
  double* scratch = scratch_for(dev);
  const int gx = ceil_div(nchr, kEA);
  int gy = std::max(1, std::min(64, 592 / std::max(gx, 1)));
  gy = (int)std::min<size_t>((size_t)gy, kNoAllocScratch / (size_t)nchr - 1);
  double* part = scratch;
  double* cou = scratch + (size_t)gy * nchr;
  energy_noalloc_kernel<<<dim3(gx, gy), kET, 0, s>>>(tr_xyz, tr_q, tr_area, x, nface, chrpos,
                                                      nchr, kappa, eps1 / eps0, part);
  coulomb_noalloc_kernel<<<nchr, 256, 0, s>>>(chrpos, atmchr, nchr, eps0, cou);
  energy_final_kernel<<<1, 256, 0, s>>>(part, gy, cou, atmchr, nchr, out);
  TABI_CUDA(cudaGetLastError());
}

}  // namespace tabi
