// potential.cu -- output_potential (main.f90:226-326): the solution back in the
// original face order and the potential / normal derivative at the vertices.
//
// Per vertex, the faces that use it are recorded in face order, at most 14 of
// them (the reference's ind_vert table has nface_vert = 15 rows, the last one
// the count, main.f90:243,255-266); the vertex value is their average weighted
// by the inverse distance between the vertex and each face centroid
// (main.f90:268-281).  Both the face and the vertex values are then scaled by
// 332.0716 * 4 pi (main.f90:297-298).  A vertex no face uses divides 0 by 0,
// as in the reference.
//
// The table is built as a CSR: per (face, corner) one entry appended to its
// vertex's list (atomic cursor), each list then sorted by face index, so the
// first 14 entries are the ones the reference records.  The weighted sums run
// in that order with explicit round-to-nearest operations (no contraction),
// the reference's expression order.
#include <cstring>

#include "tabi_impl.cuh"

namespace tabi {

namespace {

constexpr int kMaxVertFaces = 14;  // nface_vert - 1 (main.f90:243)
constexpr int kScan = 1024;

// exclusive scan of in[0..m) into out[0..m], out[m] = total (block sums,
// their scan, add)
__global__ void vp_scan_block_kernel(const int* __restrict__ in, int m, int* __restrict__ out,
                                     int* __restrict__ bsum) {
  __shared__ int sh[kScan];
  const int i = blockIdx.x * kScan + threadIdx.x;
  const int v = i < m ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < kScan; o <<= 1) {
    const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < m) out[i] = sh[threadIdx.x] - v;
  if (threadIdx.x == kScan - 1) bsum[blockIdx.x] = sh[threadIdx.x];
}

__global__ void vp_scan_sums_kernel(int* __restrict__ bsum, int nb) {
  if (threadIdx.x != 0) return;
  int acc = 0;
  for (int k = 0; k < nb; ++k) {
    const int v = bsum[k];
    bsum[k] = acc;
    acc += v;
  }
  bsum[nb] = acc;
}

__global__ void vp_scan_add_kernel(int* __restrict__ out, int m, const int* __restrict__ bsum,
                                   int nb) {
  const int i = blockIdx.x * kScan + threadIdx.x;
  if (i < m) out[i] += bsum[blockIdx.x];
  if (i == 0) out[m] = bsum[nb];
}

__global__ void vp_unpermute_kernel(int n, const int* __restrict__ perm,
                                    const double* __restrict__ x, const double* __restrict__ px,
                                    const double* __restrict__ py, const double* __restrict__ pz,
                                    double* __restrict__ xo, double* __restrict__ cen) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int f = perm[t];
  xo[f] = x[t];
  xo[n + f] = x[n + t];
  cen[3 * (size_t)f] = px[t];
  cen[3 * (size_t)f + 1] = py[t];
  cen[3 * (size_t)f + 2] = pz[t];
}

__global__ void vp_count_kernel(int nface, int nspt, const int* __restrict__ nvert,
                                int* __restrict__ cnt, int* __restrict__ err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * nface) return;
  const int v = nvert[e] - 1;
  if (v < 0 || v >= nspt) {
    atomicExch(err, 1);
    return;
  }
  atomicAdd(&cnt[v], 1);
}

__global__ void vp_fill_kernel(int nface, const int* __restrict__ nvert, int* __restrict__ cursor,
                               int* __restrict__ list) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * nface) return;
  const int v = nvert[e] - 1;
  list[atomicAdd(&cursor[v], 1)] = e / 3;
}

// per vertex: sort its faces, then the inverse-distance weighted average of
// the first kMaxVertFaces
__global__ void vp_vertex_kernel(int nspt, int nface, const double* __restrict__ sptpos,
                                 const int* __restrict__ off, int* __restrict__ list,
                                 const double* __restrict__ xo, const double* __restrict__ cen,
                                 double scale, double* __restrict__ vert) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nspt) return;
  const int a = off[v], b = off[v + 1];
  for (int p = a + 1; p < b; ++p) {
    const int key = list[p];
    int q = p - 1;
    while (q >= a && list[q] > key) {
      list[q + 1] = list[q];
      --q;
    }
    list[q + 1] = key;
  }
  const double sx = sptpos[3 * (size_t)v], sy = sptpos[3 * (size_t)v + 1],
               sz = sptpos[3 * (size_t)v + 2];
  double s1 = 0.0, s2 = 0.0, tot = 0.0;
  const int e = min(b, a + kMaxVertFaces);
  for (int p = a; p < e; ++p) {
    const int f = list[p];
    const double dx = __dsub_rn(cen[3 * (size_t)f], sx);
    const double dy = __dsub_rn(cen[3 * (size_t)f + 1], sy);
    const double dz = __dsub_rn(cen[3 * (size_t)f + 2], sz);
    const double ll =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    const double w = __ddiv_rn(1.0, ll);
    s1 = __dadd_rn(s1, __dmul_rn(w, xo[f]));
    s2 = __dadd_rn(s2, __dmul_rn(w, xo[nface + f]));
    tot = __dadd_rn(tot, w);
  }
  vert[2 * (size_t)v] = __dmul_rn(__ddiv_rn(s1, tot), scale);
  vert[2 * (size_t)v + 1] = __dmul_rn(__ddiv_rn(s2, tot), scale);
}

__global__ void vp_scale_kernel(int n2, double scale, double* __restrict__ xo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n2) xo[i] = __dmul_rn(xo[i], scale);
}

}  // namespace

void output_potential_dev(Handle& H, int nspt, const double* sptpos, int nface, const int* nvert,
                          const double* x, double* x_orig, double* vert_ptl, cudaStream_t s) {
  TABI_REQUIRE(H.has_tree, TABI_ERR_STATE, "tabi_build_tree has not been called");
  TABI_REQUIRE(nface == H.n, TABI_ERR_ARG, "nface differs from the surface's");
  TABI_REQUIRE(nspt > 0 && sptpos && nvert && x && x_orig && vert_ptl, TABI_ERR_ARG,
               "null argument");
  const int n = H.n;
  H.vp_cen.alloc(3 * (size_t)n);
  H.vp_cnt.alloc(nspt + 1);
  H.vp_off.alloc(nspt + 1);
  H.vp_list.alloc(3 * (size_t)n);
  H.vp_err.alloc(1);
  H.vp_scan.alloc(ceil_div(nspt + 1, 1024) + 2);
  {
    TABI_K(K_ENERGY, s);
    vp_unpermute_kernel<<<ceil_div(n, 256), 256, 0, s>>>(n, H.d_perm.p, x, H.d_x.p, H.d_y.p,
                                                         H.d_z.p, x_orig, H.vp_cen.p);
  }
  TABI_CUDA(cudaMemsetAsync(H.vp_cnt.p, 0, sizeof(int) * (nspt + 1), s));
  TABI_CUDA(cudaMemsetAsync(H.vp_err.p, 0, sizeof(int), s));
  {
    TABI_K(K_ENERGY, s);
    vp_count_kernel<<<ceil_div(3 * (int64_t)n, 256), 256, 0, s>>>(n, nspt, nvert, H.vp_cnt.p,
                                                                   H.vp_err.p);
  }
  int bad = 0;
  TABI_CUDA(cudaMemcpyAsync(H.h_pinned, H.vp_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  std::memcpy(&bad, H.h_pinned, sizeof(int));
  TABI_REQUIRE(bad == 0, TABI_ERR_ARG, "a face refers to a vertex outside 1..nspt");
  {
    const int nb = ceil_div(nspt, kScan);
    { TABI_K(K_ENERGY, s); vp_scan_block_kernel<<<nb, kScan, 0, s>>>(H.vp_cnt.p, nspt, H.vp_off.p, H.vp_scan.p); }
    { TABI_K(K_ENERGY, s); vp_scan_sums_kernel<<<1, 32, 0, s>>>(H.vp_scan.p, nb); }
    { TABI_K(K_ENERGY, s); vp_scan_add_kernel<<<nb, kScan, 0, s>>>(H.vp_off.p, nspt, H.vp_scan.p, nb); }
  }
  TABI_CUDA(cudaMemcpyAsync(H.vp_cnt.p, H.vp_off.p, sizeof(int) * nspt, cudaMemcpyDeviceToDevice,
                            s));
  {
    TABI_K(K_ENERGY, s);
    vp_fill_kernel<<<ceil_div(3 * (int64_t)n, 256), 256, 0, s>>>(n, nvert, H.vp_cnt.p,
                                                                  H.vp_list.p);
  }
  const double scale = 332.0716 * 4 * kPi;
  {
    TABI_K(K_ENERGY, s);
    vp_vertex_kernel<<<ceil_div(nspt, 128), 128, 0, s>>>(nspt, n, sptpos, H.vp_off.p,
                                                         H.vp_list.p, x_orig, H.vp_cen.p, scale,
                                                         vert_ptl);
  }
  {
    TABI_K(K_ENERGY, s);
    vp_scale_kernel<<<ceil_div(2 * (int64_t)n, 256), 256, 0, s>>>(2 * n, scale, x_orig);
  }
  TABI_CUDA(cudaGetLastError());
}

}  // namespace tabi
