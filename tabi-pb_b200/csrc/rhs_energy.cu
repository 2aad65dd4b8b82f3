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
// One thread per face, every atom per thread: 64-thread blocks, so that the
// few hundred blocks a molecule needs spread evenly over the SMs (with
// 256-thread blocks the 363 of the benchmark molecule put three on some SMs
// and two on others, which bounded the launch by the busiest ones).
constexpr int kFaceThreads = 64;

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
__global__ void __launch_bounds__(kFaceThreads) form_matrix_kernel(
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
__global__ void __launch_bounds__(kFaceThreads) rhs_kernel(const double* __restrict__ px,
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

// ---- readin.f90:264-333 surface_area on the device.  A face is dropped when
// its Heron area is below 1e-5 or its centroid lies within sqrt(1e-5) of the
// centroid of any of the 10 faces before it in the ORIGINAL list (dropped
// ones included), so every face decides alone: one flag kernel (recomputing
// the 10 earlier centroids, with the reference's evaluation order), one
// prefix over the blocks' counts, one order-preserving compaction.
constexpr int kFFT = 256;  // faces per block

__device__ __forceinline__ void face_centroid(const double* __restrict__ sptpos,
                                              const int* __restrict__ nvert, int nspt, int f,
                                              double (&c)[3], double (&v)[3][3], bool& bad) {
  const double third = 1.0 / 3.0;
  c[0] = c[1] = c[2] = 0.0;
  for (int k = 0; k < 3; ++k) {
    int id = nvert[3 * (size_t)f + k] - 1;
    if (id < 0 || id >= nspt) {
      bad = true;
      id = 0;
    }
    for (int d = 0; d < 3; ++d) {
      const double p = sptpos[3 * (size_t)id + d];
      v[k][d] = p;
      c[d] = __dadd_rn(c[d], __dmul_rn(third, p));
    }
  }
}

__global__ void __launch_bounds__(kFFT) face_flag_kernel(
    const double* __restrict__ sptpos, int nspt, const int* __restrict__ nvert, int nface,
    unsigned char* __restrict__ keep, int* __restrict__ bcount, double* __restrict__ barea,
    int* __restrict__ bad_out) {
  const int i = blockIdx.x * kFFT + threadIdx.x;
  bool bad = false, k = false;
  double area = 0.0;
  if (i < nface) {
    double c[3], v[3][3];
    face_centroid(sptpos, nvert, nspt, i, c, v, bad);
    area = heron(dist_rn(v[0], v[1]), dist_rn(v[0], v[2]), dist_rn(v[1], v[2]));
    bool alert = false;
    for (int ii = max(0, i - 10); ii < i; ++ii) {
      double cc[3], vv[3][3];
      face_centroid(sptpos, nvert, nspt, ii, cc, vv, bad);
      double df[3] = {__dsub_rn(c[0], cc[0]), __dsub_rn(c[1], cc[1]), __dsub_rn(c[2], cc[2])};
      if (dot3_rn(df, df) < 1e-5) alert = true;
    }
    k = !(area < 1e-5 || alert);
    keep[i] = k ? 1 : 0;
  }
  if (bad) atomicExch(bad_out, 1);
  // the block's kept count and its area sum (fixed-order tree: deterministic)
  __shared__ double sa[kFFT];
  __shared__ int sc[kFFT];
  sa[threadIdx.x] = area;
  sc[threadIdx.x] = k ? 1 : 0;
  __syncthreads();
  for (int w = kFFT / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sc[threadIdx.x] += sc[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bcount[blockIdx.x] = sc[0];
    barea[blockIdx.x] = sa[0];
  }
}

// exclusive prefix of the block counts (one thread, blocks in order), the
// kept total and the total area
__global__ void face_scan_kernel(int* __restrict__ bcount, const double* __restrict__ barea,
                                 int nblk, int* __restrict__ total, double* __restrict__ s_area) {
  if (threadIdx.x != 0) return;
  int run = 0;
  double a = 0.0;
  for (int b = 0; b < nblk; ++b) {
    const int c = bcount[b];
    bcount[b] = run;
    run += c;
    a += barea[b];
  }
  *total = run;
  *s_area = a;
}

__global__ void __launch_bounds__(kFFT) face_compact_kernel(const int* __restrict__ nvert,
                                                           int nface,
                                                           const unsigned char* __restrict__ keep,
                                                           const int* __restrict__ boff,
                                                           int* __restrict__ out) {
  __shared__ int wsum[kFFT / 32];
  const int i = blockIdx.x * kFFT + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool k = i < nface && keep[i];
  const unsigned bal = __ballot_sync(0xffffffffu, k);
  if (lane == 0) wsum[warp] = __popc(bal);
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  if (k) {
    const int pos = boff[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u));
    out[3 * (size_t)pos] = nvert[3 * (size_t)i];
    out[3 * (size_t)pos + 1] = nvert[3 * (size_t)i + 1];
    out[3 * (size_t)pos + 2] = nvert[3 * (size_t)i + 2];
  }
}

void face_filter_dev(Handle& H, int nspt, const double* sptpos, int nface, const int* nvert,
                     int* nvert_out, int* nkept, double* s_area, cudaStream_t s) {
  const int nblk = ceil_div(nface, kFFT);
  H.ff_keep.alloc(nface);
  H.ff_cnt.alloc(nblk + 2);
  H.ff_area.alloc(nblk + 1);
  TABI_CUDA(cudaMemsetAsync(H.ff_cnt.p + nblk, 0, 2 * sizeof(int), s));
  { TABI_K(K_FORM, s);
    face_flag_kernel<<<nblk, kFFT, 0, s>>>(sptpos, nspt, nvert, nface, H.ff_keep.p, H.ff_cnt.p,
                                           H.ff_area.p, H.ff_cnt.p + nblk + 1); }
  { TABI_K(K_FORM, s);
    face_scan_kernel<<<1, 32, 0, s>>>(H.ff_cnt.p, H.ff_area.p, nblk, H.ff_cnt.p + nblk,
                                      H.ff_area.p + nblk); }
  { TABI_K(K_FORM, s);
    face_compact_kernel<<<nblk, kFFT, 0, s>>>(nvert, nface, H.ff_keep.p, H.ff_cnt.p,
                                              nvert_out); }
  int hb[2];
  TABI_CUDA(cudaMemcpyAsync(hb, H.ff_cnt.p + nblk, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(s_area, H.ff_area.p + nblk, sizeof(double), cudaMemcpyDeviceToHost,
                            s));
  TABI_CUDA(cudaStreamSynchronize(s));
  TABI_REQUIRE(hb[1] == 0, TABI_ERR_ARG, "face vertex index out of range");
  *nkept = hb[0];
}

void launch_form_matrix(Handle& H, int nspt, const double* sptpos, const double* sptnrm,
                        int nface, const int* nvert, int nchr, const double* atoms4,
                        double* d_b, cudaStream_t s) {
  (void)nspt;
  { TABI_K(K_FORM, s); form_matrix_kernel<<<ceil_div(nface, kFaceThreads), kFaceThreads, 0, s>>>(
      sptpos, sptnrm, nvert, nface, atoms4, nchr, H.prm.eps0, H.d_x.p, H.d_y.p, H.d_z.p,
      H.d_nx.p, H.d_ny.p, H.d_nz.p, H.d_area.p, d_b); }
  TABI_CUDA(cudaGetLastError());
}

void launch_rhs(Handle& H, int nchr, const double* atoms4, double* d_b, cudaStream_t s) {
  { TABI_K(K_FORM, s); rhs_kernel<<<ceil_div(H.n, kFaceThreads), kFaceThreads, 0, s>>>(H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p,
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
