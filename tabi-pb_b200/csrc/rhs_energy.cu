// rhs_energy.cu -- the O(N*M) steps around the solve:
//   form_matrix  (main.f90:546-610): centroid, unit normal and Heron area per
//                face, then the RHS  b1 = sum_k q_k G0 / eps0,
//                b2 = sum_k q_k G1 / eps0  with G0 = 1/(4 pi rs),
//                G1 = cos / rs^2 / (4 pi).  Centroid, normal and area are
//                evaluated in the reference's operation order without
//                contraction, so the tree built on them is the reference's.
//   energy       (main.f90:144-157, 614-657): the reaction potential at every
//                atom  phi_k = sum_j A_j [(G1 - eps G2) x1_j + (G0 - Gk) x2_j]
//                and the pairwise Coulomb sum; the final sums over atoms are
//                done on the host in atom order, as the reference does.
#include <cmath>
#include <vector>

#include "tabi_impl.cuh"

namespace tabi {

namespace {

constexpr int kAtomTile = 256;

__device__ __forceinline__ double dot3_rn(const double* a, const double* b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}

__device__ __forceinline__ double dist_rn(const double* p, const double* q) {
  double d[3] = {__dsub_rn(p[0], q[0]), __dsub_rn(p[1], q[1]), __dsub_rn(p[2], q[2])};
  return __dsqrt_rn(dot3_rn(d, d));
}

// readin.f90:336-340 triangle_area (Heron)
__device__ __forceinline__ double heron(double aa, double bb, double cc) {
  double s = __dmul_rn(0.5, __dadd_rn(__dadd_rn(aa, bb), cc));
  double p = __dmul_rn(__dmul_rn(__dmul_rn(s, __dsub_rn(s, aa)), __dsub_rn(s, bb)),
                       __dsub_rn(s, cc));
  return __dsqrt_rn(p);
}

// atoms4: (x, y, z, q) per atom
__global__ void __launch_bounds__(256) form_matrix_kernel(
    const double* __restrict__ sptpos, const double* __restrict__ sptnrm,
    const int* __restrict__ nvert, int nface, const double* __restrict__ atoms4, int nchr,
    double eps0, double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz,
    double* __restrict__ onx, double* __restrict__ ony, double* __restrict__ onz,
    double* __restrict__ oarea, double* __restrict__ b) {
  __shared__ double4 sa[kAtomTile];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool own = i < nface;
  double r0[3] = {0, 0, 0}, v0[3] = {0, 0, 0};
  if (own) {
    const double third = 1.0 / 3.0;
    double r[3][3];
    for (int k = 0; k < 3; ++k) {
      int id = nvert[3 * i + k] - 1;
      for (int d = 0; d < 3; ++d) {
        double p = sptpos[3 * (size_t)id + d];
        r0[d] = __dadd_rn(r0[d], __dmul_rn(third, p));
        v0[d] = __dadd_rn(v0[d], __dmul_rn(third, sptnrm[3 * (size_t)id + d]));
        r[k][d] = p;
      }
    }
    double nv = __dsqrt_rn(dot3_rn(v0, v0));
    for (int d = 0; d < 3; ++d) v0[d] = __ddiv_rn(v0[d], nv);
    ox[i] = r0[0];
    oy[i] = r0[1];
    oz[i] = r0[2];
    onx[i] = v0[0];
    ony[i] = v0[1];
    onz[i] = v0[2];
    oarea[i] = heron(dist_rn(r[0], r[1]), dist_rn(r[0], r[2]), dist_rn(r[1], r[2]));
  }
  double b1 = 0.0, b2 = 0.0;
  const double inv4pi = kOneOver4Pi;
  for (int a0 = 0; a0 < nchr; a0 += kAtomTile) {
    int cnt = min(kAtomTile, nchr - a0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      const double* a = atoms4 + 4 * (size_t)(a0 + q);
      sa[q] = make_double4(a[0], a[1], a[2], a[3]);
    }
    __syncthreads();
    if (own)
      for (int q = 0; q < cnt; ++q) {
        double4 a = sa[q];
        double dx = a.x - r0[0], dy = a.y - r0[1], dz = a.z - r0[2];
        double rs2 = fma(dx, dx, fma(dy, dy, dz * dz));
        double inv = rsqrt(rs2);
        double G0 = inv4pi * inv;                                          // 1/(4 pi rs)
        double cosr = fma(v0[0], dx, fma(v0[1], dy, v0[2] * dz)) * inv;    // cos_theta
        double G1 = cosr * inv * inv * inv4pi;                             // cos/rs^2/(4 pi)
        b1 = fma(a.w, G0, b1);
        b2 = fma(a.w, G1, b2);
      }
  }
  if (own) {
    b[i] = b1 / eps0;
    b[nface + i] = b2 / eps0;
  }
}

// RHS only, surface already loaded (SoA)
__global__ void __launch_bounds__(256) rhs_kernel(const double* __restrict__ px,
                                                  const double* __restrict__ py,
                                                  const double* __restrict__ pz,
                                                  const double* __restrict__ nx,
                                                  const double* __restrict__ ny,
                                                  const double* __restrict__ nz, int nface,
                                                  const double* __restrict__ atoms4, int nchr,
                                                  double eps0, double* __restrict__ b) {
  __shared__ double4 sa[kAtomTile];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool own = i < nface;
  double r0[3] = {0, 0, 0}, v0[3] = {0, 0, 0};
  if (own) {
    r0[0] = px[i];
    r0[1] = py[i];
    r0[2] = pz[i];
    v0[0] = nx[i];
    v0[1] = ny[i];
    v0[2] = nz[i];
  }
  double b1 = 0.0, b2 = 0.0;
  for (int a0 = 0; a0 < nchr; a0 += kAtomTile) {
    int cnt = min(kAtomTile, nchr - a0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      const double* a = atoms4 + 4 * (size_t)(a0 + q);
      sa[q] = make_double4(a[0], a[1], a[2], a[3]);
    }
    __syncthreads();
    if (own)
      for (int q = 0; q < cnt; ++q) {
        double4 a = sa[q];
        double dx = a.x - r0[0], dy = a.y - r0[1], dz = a.z - r0[2];
        double inv = rsqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
        double cosr = fma(v0[0], dx, fma(v0[1], dy, v0[2] * dz)) * inv;
        b1 = fma(a.w, kOneOver4Pi * inv, b1);
        b2 = fma(a.w, cosr * inv * inv * kOneOver4Pi, b2);
      }
  }
  if (own) {
    b[i] = b1 / eps0;
    b[nface + i] = b2 / eps0;
  }
}

constexpr int kEA = 8;  // atoms per energy block
constexpr int kET = 256;

// potential_molecule (main.f90:614-657) for kEA atoms per block
__global__ void __launch_bounds__(kET) energy_kernel(
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
    const double* __restrict__ nx, const double* __restrict__ ny, const double* __restrict__ nz,
    const double* __restrict__ area, const double* __restrict__ x, int n,
    const double* __restrict__ atoms4, int nchr, double kappa, double eps,
    double* __restrict__ ptl) {
  int a0 = blockIdx.x * kEA;
  double ax[kEA], ay[kEA], az[kEA], acc[kEA];
#pragma unroll
  for (int k = 0; k < kEA; ++k) {
    int a = min(a0 + k, nchr - 1);
    ax[k] = atoms4[4 * (size_t)a];
    ay[k] = atoms4[4 * (size_t)a + 1];
    az[k] = atoms4[4 * (size_t)a + 2];
    acc[k] = 0.0;
  }
  for (int j = blockIdx.y * blockDim.x + threadIdx.x; j < n; j += gridDim.y * blockDim.x) {
    double rx = px[j], ry = py[j], rz = pz[j];
    double vx = nx[j], vy = ny[j], vz = nz[j];
    double A = area[j];
    double w1 = A * x[j], w2 = A * x[n + j];
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
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kEA; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (l == 0) s[k][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < kEA && a0 + (int)threadIdx.x < nchr) {
    double t = 0.0;
    for (int q = 0; q < kET / 32; ++q) t += s[threadIdx.x][q];
    ptl[(size_t)blockIdx.y * nchr + a0 + threadIdx.x] = t;
  }
}

// Coulomb: per atom k, sum_{l>k} q_k q_l / (eps0 dist)   (main.f90:149-155)
__global__ void coulomb_kernel(const double* __restrict__ atoms4, int nchr, double eps0,
                               double* __restrict__ out) {
  int k = blockIdx.x;
  double xk = atoms4[4 * (size_t)k], yk = atoms4[4 * (size_t)k + 1],
         zk = atoms4[4 * (size_t)k + 2], qk = atoms4[4 * (size_t)k + 3];
  double acc = 0.0;
  for (int l = k + 1 + threadIdx.x; l < nchr; l += blockDim.x) {
    double dx = xk - atoms4[4 * (size_t)l], dy = yk - atoms4[4 * (size_t)l + 1],
           dz = zk - atoms4[4 * (size_t)l + 2];
    double dist = sqrt(dx * dx + dy * dy + dz * dz);
    acc += 1.0 / eps0 / dist * qk * atoms4[4 * (size_t)l + 3];
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += s[q];
    out[k] = t;
  }
}

__global__ void pack_atoms_kernel(const double* __restrict__ chrpos,
                                  const double* __restrict__ atmchr, int nchr,
                                  double* __restrict__ atoms4) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nchr) return;
  atoms4[4 * (size_t)k] = chrpos[3 * (size_t)k];
  atoms4[4 * (size_t)k + 1] = chrpos[3 * (size_t)k + 1];
  atoms4[4 * (size_t)k + 2] = chrpos[3 * (size_t)k + 2];
  atoms4[4 * (size_t)k + 3] = atmchr[k];
}

}  // namespace

void pack_atoms_dev(Handle& H, int nchr, const double* chrpos_dev, const double* atmchr_dev,
                    cudaStream_t s) {
  H.d_atoms.alloc(4 * (size_t)std::max(nchr, 1));
  if (nchr > 0)
    { TABI_K(K_FORM, s); pack_atoms_kernel<<<ceil_div(nchr, 128), 128, 0, s>>>(chrpos_dev, atmchr_dev, nchr,
                                                          H.d_atoms.p); }
}

void launch_form_matrix(Handle& H, int nspt, const double* sptpos, const double* sptnrm,
                        int nface, const int* nvert, int nchr, const double* atoms4,
                        double* d_b, cudaStream_t s) {
  (void)nspt;
  { TABI_K(K_FORM, s); form_matrix_kernel<<<ceil_div(nface, 256), 256, 0, s>>>(
      sptpos, sptnrm, nvert, nface, atoms4, nchr, H.prm.eps0, H.d_x.p, H.d_y.p, H.d_z.p,
      H.d_nx.p, H.d_ny.p, H.d_nz.p, H.d_area.p, d_b); }
  TABI_CUDA(cudaGetLastError());
}

void launch_rhs(Handle& H, int nchr, const double* atoms4, double* d_b, cudaStream_t s) {
  { TABI_K(K_FORM, s); rhs_kernel<<<ceil_div(H.n, 256), 256, 0, s>>>(H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p,
                                                H.d_nz.p, H.n, atoms4, nchr, H.prm.eps0, d_b); }
  TABI_CUDA(cudaGetLastError());
}

// atoms must already be packed in H.d_atoms
void energy_dev(Handle& H, int nchr, const double* /*chrpos*/, const double* /*atmchr*/,
                const double* x, double* soleng, double* couleng, cudaStream_t s) {
  const int n = H.n;
  int gx = ceil_div(nchr, kEA);
  // face chunks per atom block: about six waves of the 2 x 148 resident
  // blocks, so the last partial wave costs little
  int gy = std::max(1, std::min(64, 296 * 6 / std::max(gx, 1)));
  H.d_ptl.alloc((size_t)gy * nchr + nchr);
  double eps = H.prm.eps1 / H.prm.eps0;
  { TABI_K(K_ENERGY, s); energy_kernel<<<dim3(gx, gy), kET, 0, s>>>(H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p,
                                             H.d_nz.p, H.d_area.p, x, n, H.d_atoms.p, nchr,
                                             H.prm.kappa, eps, H.d_ptl.p); }
  double* d_cou = H.d_ptl.p + (size_t)gy * nchr;
  { TABI_K(K_ENERGY, s); coulomb_kernel<<<nchr, 256, 0, s>>>(H.d_atoms.p, nchr, H.prm.eps0, d_cou); }
  std::vector<double> ptl((size_t)gy * nchr), cou(nchr), q(4 * (size_t)nchr);
  TABI_CUDA(cudaMemcpyAsync(ptl.data(), H.d_ptl.p, sizeof(double) * ptl.size(),
                            cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(cou.data(), d_cou, sizeof(double) * nchr, cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(q.data(), H.d_atoms.p, sizeof(double) * 4 * nchr,
                            cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  double se = 0.0, ce = 0.0;
  for (int k = 0; k < nchr; ++k) {
    double p = 0.0;
    for (int y = 0; y < gy; ++y) p += ptl[(size_t)y * nchr + k];
    se = se + q[4 * (size_t)k + 3] * p;
    ce = ce + cou[k];
  }
  const double para = 332.0716;
  *soleng = se * 0.5 * para * 4.0 * kPi;
  *couleng = ce * para;
}

}  // namespace tabi
