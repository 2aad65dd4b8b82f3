// matvec.cu -- the treecode operator y = A x (TREE_COMPP_PB,
// treecode3d_pb.f:1130-1189) as four device steps:
//
//  1. moments   COMP_MS (treecode3d_pb.f:859-916) for every cluster some
//               target accepts.  The 16 source charges of pb_kernel
//               (main.f90:664-694) reduce to 4 distinct ones -- A*x2 and
//               (n_d*A)*x1 -- so 4 raw moment sets are summed, then
//               weighted by the integer part of der_cof (main.f90:380-399)
//               into the 16 per-index sets the contraction reads.
//  2. far       one thread per (target, accepted cluster): the generated
//               COMP_TCOEFF + COMPP_TREE_PB evaluation (taylor_gen.cuh),
//               cluster moments staged in shared memory.
//  3. near      one thread per (target, near leaf): COMPP_DIRECT_PB
//               (treecode3d_pb.f:919-1008) over the leaf's faces staged in
//               shared memory; the target's own face is skipped, which is what
//               the reference's shift-and-zero-area trick (:1169-1172) amounts
//               to.
//  4. reduce    per target, the interaction results summed in traversal order:
//               y1 = pre1*x1 - peng1, y2 = pre2*x2 - peng2 (:1177-1178).
// All results are written to per-(target, interaction) slots fixed by the
// traversal, so the sums are deterministic.
#include <algorithm>

#include "bie_kernels.cuh"
#include "reduce.cuh"
#include "taylor_gen.cuh"
#include "tabi_impl.cuh"

namespace tabi {

namespace {

// ---- moments
template <int P>
__global__ void mom_partial_kernel(const int4* __restrict__ chunks,
                                   const int* __restrict__ mslot_node,
                                   const double* __restrict__ nd_mid,
                                   const double* __restrict__ px, const double* __restrict__ py,
                                   const double* __restrict__ pz, const double* __restrict__ nx,
                                   const double* __restrict__ ny, const double* __restrict__ nz,
                                   const double* __restrict__ area,
                                   const double* __restrict__ x, int n,
                                   double* __restrict__ mraw) {
  constexpr int NT = tabi_nterms(P);
  constexpr int TILE = 128;
  constexpr int W = 3 * (P + 1) + 4;
  __shared__ double st[TILE][W];
  int4 ch = chunks[blockIdx.x];
  int node = mslot_node[ch.x];
  double mx = nd_mid[3 * node], my = nd_mid[3 * node + 1], mz = nd_mid[3 * node + 2];
  int t = threadIdx.x;
  int set = t / NT, term = t - set * NT;
  bool own = t < 4 * NT;
  int k1 = 0, k2 = 0, k3 = 0;
  if (own) {
    const signed char(*tt)[3] = tabi_terms<P>();
    k1 = tt[term][0];
    k2 = tt[term][1];
    k3 = tt[term][2];
  }
  double acc = 0.0;
  for (int base = 0; base < ch.z; base += TILE) {
    int cnt = min(TILE, ch.z - base);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      int i = ch.y + base + q;
      // COMP_MS :876-889: dx = x - mid, powers by repeated multiplication
      double dx = px[i] - mx, dy = py[i] - my, dz = pz[i] - mz;
      double a = 1.0, b = 1.0, c = 1.0;
#pragma unroll
      for (int p = 0; p <= P; ++p) {
        st[q][p] = a;
        st[q][P + 1 + p] = b;
        st[q][2 * (P + 1) + p] = c;
        a *= dx;
        b *= dy;
        c *= dz;
      }
      double A = area[i], x1 = x[i], x2 = x[n + i];
      // pb_kernel (main.f90:673-681): A*x2 and (n_d*A)*x1
      st[q][3 * (P + 1) + 0] = A * x2;
      st[q][3 * (P + 1) + 1] = (nx[i] * A) * x1;
      st[q][3 * (P + 1) + 2] = (ny[i] * A) * x1;
      st[q][3 * (P + 1) + 3] = (nz[i] * A) * x1;
    }
    __syncthreads();
    if (own)
      for (int q = 0; q < cnt; ++q) {
        double txyz = st[q][k1] * st[q][P + 1 + k2] * st[q][2 * (P + 1) + k3];
        acc = fma(st[q][3 * (P + 1) + set], txyz, acc);
      }
  }
  if (own) mraw[((size_t)ch.w * 4 + set) * NT + term] = acc;
}

template <int P, typename TO>
__global__ void mom_final_kernel(const int2* __restrict__ mslot_chunks,
                                 const double* __restrict__ mraw, TO* __restrict__ mw) {
  constexpr int NT = tabi_nterms(P);
  int slot = blockIdx.x;
  int2 cr = mslot_chunks[slot];
  const signed char(*tt)[3] = tabi_terms<P>();
  // kk (main.f90:358-376) and the source set / sign of each of the 16 indices
  const int kk[16][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 0}, {0, 1, 0},
                         {0, 0, 1}, {2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 1, 0}, {0, 2, 0},
                         {0, 1, 1}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};
  for (int q = threadIdx.x; q < 16 * NT; q += blockDim.x) {
    int idx = q / NT, term = q - idx * NT;
    int set = (idx == 0) ? 0 : (idx <= 3) ? idx : (idx <= 6) ? 0 : 1 + (idx - 7) / 3;
    double sgn = (idx >= 7) ? -1.0 : 1.0;
    double raw = 0.0;
    for (int c = 0; c < cr.y; ++c) raw += mraw[((size_t)(cr.x + c) * 4 + set) * NT + term];
    int kv[3] = {tt[term][0], tt[term][1], tt[term][2]};
    double w = 1.0;
    for (int m = 0; m < 3; ++m)
      for (int j = 1; j <= kk[idx][m]; ++j) w *= (double)(kv[m] + j);
    mw[(size_t)slot * 16 * NT + q] = (TO)(sgn * w * raw);
  }
}

// ---- far field
// T = double: the reference's arithmetic.  T = float (mixed precision): the
// target-to-centre offset is formed in FP64 and rounded once, the Taylor
// recurrences and the contraction run in FP32, the result is widened to FP64
// for the per-target sum.  Order 3 is capped at 128 registers (8 blocks per
// SM instead of 6 in FP64, for a few bytes of spill).
template <int P, typename T>
__global__ void __launch_bounds__(64, P == 3 ? 8 : 1) far_kernel(const WorkItem* __restrict__ work,
                                                 const int2* __restrict__ ent,
                                                 const T* __restrict__ mw,
                                                 const double* __restrict__ nd_mid,
                                                 const double* __restrict__ px,
                                                 const double* __restrict__ py,
                                                 const double* __restrict__ pz,
                                                 const double* __restrict__ nx,
                                                 const double* __restrict__ ny,
                                                 const double* __restrict__ nz, T kappa,
                                                 T eps, double2* __restrict__ res) {
  constexpr int NT = tabi_nterms(P);
  __shared__ T smw[16 * NT];
  WorkItem wi = work[blockIdx.x];
  const T* src = mw + (size_t)wi.mslot * 16 * NT;
  for (int q = threadIdx.x; q < 16 * NT; q += blockDim.x) smw[q] = src[q];
  __syncthreads();
  if ((int)threadIdx.x >= wi.count) return;
  int2 e = ent[wi.start + threadIdx.x];
  int t = e.x;
  // COMP_TCOEFF :707-709: dx = target - mid
  T dx = (T)(px[t] - nd_mid[3 * wi.node]);
  T dy = (T)(py[t] - nd_mid[3 * wi.node + 1]);
  T dz = (T)(pz[t] - nd_mid[3 * wi.node + 2]);
  T o1, o2;
  far_eval<P, T>(dx, dy, dz, kappa, smw, (T)nx[t], (T)ny[t], (T)nz[t], eps, T(1) / eps, o1, o2);
  res[e.y] = make_double2((double)o1 * kOneOver4Pi, (double)o2 * kOneOver4Pi);
}

// ---- near field
constexpr int kNearThreads = 128;
constexpr int kNearTile = 512;

__global__ void __launch_bounds__(kNearThreads) near_kernel(
    const WorkItem* __restrict__ work, const int2* __restrict__ ent,
    const int* __restrict__ nd_ibeg, const int* __restrict__ nd_num,
    const double* __restrict__ px, const double* __restrict__ py,
    const double* __restrict__ pz, const double* __restrict__ nx,
    const double* __restrict__ ny, const double* __restrict__ nz,
    const double* __restrict__ area, const double* __restrict__ x, int n, double kappa,
    double eps, double2* __restrict__ res) {
  __shared__ double s_x[kNearTile], s_y[kNearTile], s_z[kNearTile];
  __shared__ double s_nx[kNearTile], s_ny[kNearTile], s_nz[kNearTile];
  __shared__ double s_w1[kNearTile], s_w2[kNearTile];
  WorkItem wi = work[blockIdx.x];
  int ib = nd_ibeg[wi.node], nsrc = nd_num[wi.node];
  bool own = (int)threadIdx.x < wi.count;
  int t = 0, slot = 0;
  double tx = 0, ty = 0, tz = 0, vx = 0, vy = 0, vz = 0;
  if (own) {
    int2 e = ent[wi.start + threadIdx.x];
    t = e.x;
    slot = e.y;
    tx = px[t];
    ty = py[t];
    tz = pz[t];
    vx = nx[t];
    vy = ny[t];
    vz = nz[t];
  }
  const double inv_eps = 1.0 / eps;
  double p1 = 0.0, p2 = 0.0;
  for (int b0 = 0; b0 < nsrc; b0 += kNearTile) {
    int cnt = min(kNearTile, nsrc - b0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      int j = ib + b0 + q;
      s_x[q] = px[j];
      s_y[q] = py[j];
      s_z[q] = pz[j];
      s_nx[q] = nx[j];
      s_ny[q] = ny[j];
      s_nz[q] = nz[j];
      double A = area[j];
      s_w1[q] = A * x[j];
      s_w2[q] = A * x[n + j];
    }
    __syncthreads();
    if (own) {
      int self = t - (ib + b0);
#pragma unroll 2
      for (int q = 0; q < cnt; ++q) {
        bool skip = (q == self);
        double dx = s_x[q] - tx, dy = s_y[q] - ty, dz = s_z[q] - tz;
        if (skip) dx = 1.0;  // keeps the skipped pair finite
        double K1, K2, K3, K4;
        bie4<double>(dx, dy, dz, vx, vy, vz, s_nx[q], s_ny[q], s_nz[q], kappa, eps, inv_eps, K1,
                     K2, K3, K4);
        double w1 = skip ? 0.0 : s_w1[q], w2 = skip ? 0.0 : s_w2[q];
        p1 = fma(K1, w1, fma(K2, w2, p1));
        p2 = fma(K3, w1, fma(K4, w2, p2));
      }
    }
  }
  if (own) res[slot] = make_double2(p1, p2);
}

// Mixed-precision near field.  Each face's position relative to the centre of
// its leaf is kept as an unevaluated FP32 sum hi + lo (to ~2^-48 of the leaf
// size), with its area and its normal in FP32 (leaf_rel_kernel, once per tree);
// the target is split the same way against the same centre.  r - s is then
// (hi_s - hi_t) + (lo_s - lo_t), accurate to FP32 rounding of |r - s| itself:
// with one rounded FP32 coordinate, n.(r - s) of adjacent panels (a few
// hundredths of an Angstrom on a curved surface) would carry the 1e-6 A
// rounding of leaf-sized coordinates, an error of ~1e-4 relative in K1 and K4.
// The four kernels and the per-(target, leaf) sum run in FP32; the per-target
// sum over leaves stays FP64 (reduce_kernel).
__global__ void leaf_rel_kernel(const int* __restrict__ leaves, const int* __restrict__ nd_ibeg,
                                const int* __restrict__ nd_num, const double* __restrict__ nd_mid,
                                const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, const double* __restrict__ nx,
                                const double* __restrict__ ny, const double* __restrict__ nz,
                                const double* __restrict__ area, float4* __restrict__ lpos,
                                float4* __restrict__ llo, float4* __restrict__ lnrm) {
  const int node = leaves[blockIdx.x];
  const int ib = nd_ibeg[node], m = nd_num[node];
  const double mx = nd_mid[3 * node], my = nd_mid[3 * node + 1], mz = nd_mid[3 * node + 2];
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    const int j = ib + q;
    const double rx = px[j] - mx, ry = py[j] - my, rz = pz[j] - mz;
    const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
    lpos[j] = make_float4(hx, hy, hz, (float)area[j]);
    llo[j] = make_float4((float)(rx - hx), (float)(ry - hy), (float)(rz - hz), 0.f);
    lnrm[j] = make_float4((float)nx[j], (float)ny[j], (float)nz[j], 0.f);
  }
}

constexpr int kNearTileF = 512;

__global__ void __launch_bounds__(kNearThreads) near_kernel_f32(
    const WorkItem* __restrict__ work, const int2* __restrict__ ent,
    const int* __restrict__ nd_ibeg, const int* __restrict__ nd_num,
    const double* __restrict__ nd_mid, const double* __restrict__ px,
    const double* __restrict__ py, const double* __restrict__ pz,
    const float4* __restrict__ lpos, const float4* __restrict__ llo,
    const float4* __restrict__ lnrm, const double* __restrict__ x, int n, float kappa,
    float eps, double2* __restrict__ res) {
  __shared__ float4 s_p[kNearTileF];  // relative position (hi), A * x1
  __shared__ float4 s_l[kNearTileF];  // relative position (lo)
  __shared__ float4 s_n[kNearTileF];  // normal, A * x2
  WorkItem wi = work[blockIdx.x];
  const int ib = nd_ibeg[wi.node], nsrc = nd_num[wi.node];
  const bool own = (int)threadIdx.x < wi.count;
  int t = 0, slot = 0;
  float tx = 0.f, ty = 0.f, tz = 0.f, lx = 0.f, ly = 0.f, lz = 0.f;
  float vx = 0.f, vy = 0.f, vz = 0.f;
  if (own) {
    int2 e = ent[wi.start + threadIdx.x];
    t = e.x;
    slot = e.y;
    const double rx = px[t] - nd_mid[3 * wi.node];
    const double ry = py[t] - nd_mid[3 * wi.node + 1];
    const double rz = pz[t] - nd_mid[3 * wi.node + 2];
    tx = (float)rx;
    ty = (float)ry;
    tz = (float)rz;
    lx = (float)(rx - tx);
    ly = (float)(ry - ty);
    lz = (float)(rz - tz);
    float4 nv = lnrm[t];
    vx = nv.x;
    vy = nv.y;
    vz = nv.z;
  }
  const float inv_eps = 1.f / eps;
  float p1 = 0.f, p2 = 0.f;
  for (int b0 = 0; b0 < nsrc; b0 += kNearTileF) {
    const int cnt = min(kNearTileF, nsrc - b0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      const int j = ib + b0 + q;
      float4 a = lpos[j], b = lnrm[j];
      const double A = (double)a.w;
      a.w = (float)(A * x[j]);
      b.w = (float)(A * x[n + j]);
      s_p[q] = a;
      s_l[q] = llo[j];
      s_n[q] = b;
    }
    __syncthreads();
    if (own) {
      const int self = t - (ib + b0);
#pragma unroll 4
      for (int q = 0; q < cnt; ++q) {
        const float4 a = s_p[q], l = s_l[q], b = s_n[q];
        const bool skip = (q == self);
        float dx = (a.x - tx) + (l.x - lx), dy = (a.y - ty) + (l.y - ly),
              dz = (a.z - tz) + (l.z - lz);
        if (skip) dx = 1.f;  // keeps the skipped pair finite
        float K1, K2, K3, K4;
        bie4(dx, dy, dz, vx, vy, vz, b.x, b.y, b.z, kappa, eps, inv_eps, K1, K2, K3, K4);
        const float w1 = skip ? 0.f : a.w, w2 = skip ? 0.f : b.w;
        p1 = fmaf(K1, w1, fmaf(K2, w2, p1));
        p2 = fmaf(K3, w1, fmaf(K4, w2, p2));
      }
    }
  }
  if (own) res[slot] = make_double2((double)p1, (double)p2);
}

__global__ void reduce_kernel(const int64_t* __restrict__ slot_off,
                              const double2* __restrict__ res, const double* __restrict__ x,
                              int n, int t0, int t1, double pre1, double pre2,
                              double* __restrict__ y) {
  int t = t0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= t1) return;
  double s1 = 0.0, s2 = 0.0;
  for (int64_t k = slot_off[t]; k < slot_off[t + 1]; ++k) {
    double2 r = res[k];
    s1 += r.x;
    s2 += r.y;
  }
  y[t] = pre1 * x[t] - s1;
  y[n + t] = pre2 * x[n + t] - s2;
}

template <int P>
void launch_moments(Handle& H, const double* x, bool f32, cudaStream_t s) {
  Tree& T = H.tree;
  constexpr int NT = tabi_nterms(P);
  if (T.nmslot == 0) return;
  int nch = 0;
  for (int k = 0; k < T.nmslot; ++k) nch += T.mslot_nchunk[k];
  int threads = ((4 * NT + 31) / 32) * 32;
  {
    TABI_K(K_MOMENTS, s);
    mom_partial_kernel<P><<<nch, threads, 0, s>>>(T.d_mchunks.p, T.d_mslot_node.p, T.d_mid.p,
                                                  H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p,
                                                  H.d_nz.p, H.d_area.p, x, H.n, H.d_mraw.p);
  }
  TABI_K(K_MOMENTS, s);
  if (f32)
    mom_final_kernel<P, float><<<T.nmslot, 256, 0, s>>>(T.d_mslot_chunks.p, H.d_mraw.p,
                                                          H.d_mwf.p);
  else
    mom_final_kernel<P, double><<<T.nmslot, 256, 0, s>>>(T.d_mslot_chunks.p, H.d_mraw.p,
                                                           H.d_mw.p);
}

template <int P>
void launch_far(Handle& H, bool f32, cudaStream_t s) {
  Tree& T = H.tree;
  const int nw = (int)(T.ranged ? T.r_far_work.size() : T.far_work.size());
  const WorkItem* fw = T.ranged ? T.d_r_far_work.p : T.d_far_work.p;
  const int2* fe = T.ranged ? T.d_r_far_ent.p : T.d_far_ent.p;
  if (nw == 0) return;
  const double eps = H.prm.eps1 / H.prm.eps0;
  TABI_K(K_FAR, s);
  if (f32)
    far_kernel<P, float><<<nw, 64, 0, s>>>(
        fw, fe, H.d_mwf.p, T.d_mid.p, H.d_x.p, H.d_y.p, H.d_z.p,
        H.d_nx.p, H.d_ny.p, H.d_nz.p, (float)H.prm.kappa, (float)eps, H.d_res.p);
  else
    far_kernel<P, double><<<nw, 64, 0, s>>>(
        fw, fe, H.d_mw.p, T.d_mid.p, H.d_x.p, H.d_y.p, H.d_z.p,
        H.d_nx.p, H.d_ny.p, H.d_nz.p, H.prm.kappa, eps, H.d_res.p);
}

// FP32 copies of the faces relative to their leaf centres (once per tree)
void prepare_f32(Handle& H, cudaStream_t s) {
  Tree& T = H.tree;
  if (T.lrel_ready) return;
  T.d_leaves.alloc(std::max(T.nleaf, 1));
  TABI_CUDA(cudaMemcpyAsync(T.d_leaves.p, T.leaves.data(), sizeof(int) * T.nleaf,
                            cudaMemcpyHostToDevice, s));
  T.d_lpos.alloc(std::max(H.n, 1));
  T.d_llo.alloc(std::max(H.n, 1));
  T.d_lnrm.alloc(std::max(H.n, 1));
  {
    TABI_K(K_TREE, s);
    leaf_rel_kernel<<<T.nleaf, 256, 0, s>>>(T.d_leaves.p, T.d_ibeg.p, T.d_num.p, T.d_mid.p,
                                            H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p,
                                            H.d_nz.p, H.d_area.p, T.d_lpos.p, T.d_llo.p,
                                            T.d_lnrm.p);
  }
  TABI_CUDA(cudaGetLastError());
  T.lrel_ready = true;
}

}  // namespace

double reduce_dev(Handle& H, int op, const double* a, const double* b, int n, cudaStream_t s) {
  H.d_red.alloc(kRedBlocks + 8);
  int nb = std::min(kRedBlocks, ceil_div(n, kRedThreads));
  if (nb < 1) nb = 1;
  if (op == 0)
    { TABI_K(K_VEC, s); reduce_partial_kernel<0><<<nb, kRedThreads, 0, s>>>(a, b, n, H.d_red.p); }
  else if (op == 1)
    { TABI_K(K_VEC, s); reduce_partial_kernel<1><<<nb, kRedThreads, 0, s>>>(a, b, n, H.d_red.p); }
  else
    { TABI_K(K_VEC, s); reduce_partial_kernel<2><<<nb, kRedThreads, 0, s>>>(a, b, n, H.d_red.p); }
  { TABI_K(K_VEC, s); reduce_final_kernel<<<1, 256, 0, s>>>(H.d_red.p, nb, H.d_red.p + kRedBlocks); }
  TABI_CUDA(cudaMemcpyAsync(H.h_pinned, H.d_red.p + kRedBlocks, sizeof(double),
                            cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  return H.h_pinned[0];
}

double asum_dev(Handle& H, const double* x, int n, cudaStream_t s) {
  return reduce_dev(H, 0, x, nullptr, n, s);
}
double dot_dev(Handle& H, const double* a, const double* b, int n, cudaStream_t s) {
  return reduce_dev(H, 1, a, b, n, s);
}
double nrm2_dev(Handle& H, const double* a, int n, cudaStream_t s) {
  return sqrt(reduce_dev(H, 2, a, nullptr, n, s));
}

void matvec_dev(Handle& H, const double* x, double* y, cudaStream_t s, bool check_zero) {
  const int n = H.n;
  if (check_zero) {
    // MATVECmain (main.f90:478-479): sum|x| < 1e-10 gives y = x
    double a = asum_dev(H, x, 2 * n, s);
    if (a < 1e-10) {
      if (y != x)
        TABI_CUDA(cudaMemcpyAsync(y, x, sizeof(double) * 2 * n, cudaMemcpyDeviceToDevice, s));
      return;
    }
  }
  Tree& T = H.tree;
  const bool f32 = H.mv_prec == TABI_PREC_MIXED;
  if (f32) {
    prepare_f32(H, s);
    if (T.nmslot > 0) H.d_mwf.alloc(H.d_mw.n);
  }
  TABI_PHASE(K_PHASE_MATVEC, s);
  // the near field runs on the handle's side stream, concurrently with the
  // moments + far field on s; both write disjoint result slots
  const int nnw = (int)(T.ranged ? T.r_near_work.size() : T.near_work.size());
  const WorkItem* nwk = T.ranged ? T.d_r_near_work.p : T.d_near_work.p;
  const int2* nent = T.ranged ? T.d_r_near_ent.p : T.d_near_ent.p;
  const bool fork = nnw > 0 && H.side != nullptr;
  cudaStream_t sn = fork ? H.side : s;
  if (fork) {
    TABI_CUDA(cudaEventRecord(H.ev_fork, s));
    TABI_CUDA(cudaStreamWaitEvent(sn, H.ev_fork, 0));
  }
  // moments first (small, needed by the far field), then the near field on
  // the side stream and the far field on s
  switch (H.prm.order) {
    case 1: launch_moments<1>(H, x, f32, s); break;
    case 2: launch_moments<2>(H, x, f32, s); break;
    case 3: launch_moments<3>(H, x, f32, s); break;
    case 4: launch_moments<4>(H, x, f32, s); break;
    case 5: launch_moments<5>(H, x, f32, s); break;
    case 6: launch_moments<6>(H, x, f32, s); break;
    case 7: launch_moments<7>(H, x, f32, s); break;
    case 8: launch_moments<8>(H, x, f32, s); break;
    default: throw Error(TABI_ERR_ARG, "order must be 1..8");
  }
  if (nnw > 0 && f32) {
    TABI_K(K_NEAR, sn);
    near_kernel_f32<<<nnw, kNearThreads, 0, sn>>>(
        nwk, nent, T.d_ibeg.p, T.d_num.p, T.d_mid.p, H.d_x.p, H.d_y.p,
        H.d_z.p, T.d_lpos.p, T.d_llo.p, T.d_lnrm.p, x, n, (float)H.prm.kappa,
        (float)(H.prm.eps1 / H.prm.eps0), H.d_res.p);
  } else if (nnw > 0) {
    TABI_K(K_NEAR, sn);
    near_kernel<<<nnw, kNearThreads, 0, sn>>>(
        nwk, nent, T.d_ibeg.p, T.d_num.p, H.d_x.p, H.d_y.p, H.d_z.p,
        H.d_nx.p, H.d_ny.p, H.d_nz.p, H.d_area.p, x, n, H.prm.kappa, H.prm.eps1 / H.prm.eps0,
        H.d_res.p);
  }
  switch (H.prm.order) {
    case 1: launch_far<1>(H, f32, s); break;
    case 2: launch_far<2>(H, f32, s); break;
    case 3: launch_far<3>(H, f32, s); break;
    case 4: launch_far<4>(H, f32, s); break;
    case 5: launch_far<5>(H, f32, s); break;
    case 6: launch_far<6>(H, f32, s); break;
    case 7: launch_far<7>(H, f32, s); break;
    case 8: launch_far<8>(H, f32, s); break;
    default: break;
  }
  if (fork) {
    TABI_CUDA(cudaEventRecord(H.ev_join, sn));
    TABI_CUDA(cudaStreamWaitEvent(s, H.ev_join, 0));
  }
  double eps = H.prm.eps1 / H.prm.eps0;
  const int t0 = T.ranged ? T.rt0 : 0, t1 = T.ranged ? T.rt1 : n;
  { TABI_K(K_REDUCE, s); reduce_kernel<<<ceil_div(t1 - t0, 256), 256, 0, s>>>(T.d_slot_off.p, H.d_res.p, x, n, t0, t1,
                                                 0.5 * (1.0 + eps), 0.5 * (1.0 + 1.0 / eps), y); }
  TABI_CUDA(cudaGetLastError());
}

namespace {

// FP64 direct sum of the operator for selected targets (the accuracy
// reference of the treecode): y_t = pre x_t - sum_{j != t} (K(t, j) A_j x_j),
// every source evaluated exactly (COMPP_DIRECT_PB's kernels,
// treecode3d_pb.f:919-1008).  Grid: x = chunks of kDirT targets (one per
// thread), y = chunks of kDirS sources staged through shared memory;
// partials per (target, source chunk) are summed in chunk order afterwards.
constexpr int kDirT = 128, kDirS = 8192, kDirTile = 256;

__global__ void __launch_bounds__(kDirT) direct_kernel(
    int n, const int* __restrict__ targets, int nt, const double* __restrict__ px,
    const double* __restrict__ py, const double* __restrict__ pz,
    const double* __restrict__ nx, const double* __restrict__ ny,
    const double* __restrict__ nz, const double* __restrict__ area,
    const double* __restrict__ x, double kappa, double eps, double2* __restrict__ part) {
  __shared__ double s_x[kDirTile], s_y[kDirTile], s_z[kDirTile];
  __shared__ double s_nx[kDirTile], s_ny[kDirTile], s_nz[kDirTile];
  __shared__ double s_w1[kDirTile], s_w2[kDirTile];
  const int k = blockIdx.x * kDirT + threadIdx.x;
  const bool own = k < nt;
  const int t = own ? targets[k] : 0;
  const double tx = px[t], ty = py[t], tz = pz[t], vx = nx[t], vy = ny[t], vz = nz[t];
  const double inv_eps = 1.0 / eps;
  const int j0 = blockIdx.y * kDirS, j1 = min(n, j0 + kDirS);
  double p1 = 0.0, p2 = 0.0;
  for (int b0 = j0; b0 < j1; b0 += kDirTile) {
    const int cnt = min(kDirTile, j1 - b0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += kDirT) {
      const int j = b0 + q;
      s_x[q] = px[j];
      s_y[q] = py[j];
      s_z[q] = pz[j];
      s_nx[q] = nx[j];
      s_ny[q] = ny[j];
      s_nz[q] = nz[j];
      s_w1[q] = area[j] * x[j];
      s_w2[q] = area[j] * x[n + j];
    }
    __syncthreads();
    if (own)
      for (int q = 0; q < cnt; ++q) {
        const bool skip = (b0 + q == t);
        double dx = s_x[q] - tx, dy = s_y[q] - ty, dz = s_z[q] - tz;
        if (skip) dx = 1.0;
        double K1, K2, K3, K4;
        bie4<double>(dx, dy, dz, vx, vy, vz, s_nx[q], s_ny[q], s_nz[q], kappa, eps, inv_eps, K1,
                     K2, K3, K4);
        const double w1 = skip ? 0.0 : s_w1[q], w2 = skip ? 0.0 : s_w2[q];
        p1 = fma(K1, w1, fma(K2, w2, p1));
        p2 = fma(K3, w1, fma(K4, w2, p2));
      }
  }
  if (own) part[(size_t)k * gridDim.y + blockIdx.y] = make_double2(p1, p2);
}

__global__ void direct_final_kernel(int n, const int* __restrict__ targets, int nt, int nchunk,
                                    const double2* __restrict__ part,
                                    const double* __restrict__ x, double pre1, double pre2,
                                    double* __restrict__ y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const int t = targets[k];
  double s1 = 0.0, s2 = 0.0;
  for (int c = 0; c < nchunk; ++c) {
    const double2 r = part[(size_t)k * nchunk + c];
    s1 += r.x;
    s2 += r.y;
  }
  y[k] = pre1 * x[t] - s1;
  y[nt + k] = pre2 * x[n + t] - s2;
}

}  // namespace

void direct_targets_dev(Handle& H, int nt, const int* targets, const double* x, double* y,
                        cudaStream_t s) {
  TABI_REQUIRE(H.has_surface, TABI_ERR_STATE, "no surface");
  const int n = H.n;
  const int nchunk = ceil_div(n, kDirS);
  H.d_dirpart.alloc((size_t)std::max(nt, 1) * nchunk);
  const double eps = H.prm.eps1 / H.prm.eps0;
  {
    TABI_K(K_NEAR, s);
    direct_kernel<<<dim3(ceil_div(nt, kDirT), nchunk), kDirT, 0, s>>>(
        n, targets, nt, H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p, H.d_nz.p, H.d_area.p, x,
        H.prm.kappa, eps, H.d_dirpart.p);
  }
  {
    TABI_K(K_REDUCE, s);
    direct_final_kernel<<<ceil_div(nt, 256), 256, 0, s>>>(n, targets, nt, nchunk,
                                                          H.d_dirpart.p, x, 0.5 * (1.0 + eps),
                                                          0.5 * (1.0 + 1.0 / eps), y);
  }
  TABI_CUDA(cudaGetLastError());
}

void set_target_range(Handle& H, int t0, int t1, cudaStream_t s) {
  Tree& T = H.tree;
  const int n = H.n;
  TABI_REQUIRE(H.has_tree, TABI_ERR_STATE, "tabi_build_tree has not been called");
  TABI_REQUIRE(0 <= t0 && t0 < t1 && t1 <= n, TABI_ERR_ARG, "target range must be within 0..nface");
  T.ranged = false;
  if (t0 == 0 && t1 == n) return;
  // leaf-aligned: the shard owns whole leaves (so the preconditioner, which is
  // leaf-local, splits with it)
  std::vector<int> starts;
  for (int c : T.leaves) starts.push_back(T.ibeg[c]);
  std::sort(starts.begin(), starts.end());
  auto boundary = [&](int t) {
    return t == n || std::binary_search(starts.begin(), starts.end(), t);
  };
  TABI_REQUIRE(boundary(t0) && boundary(t1), TABI_ERR_ARG,
               "target range must start and end on leaf boundaries (tree order)");
  // the interaction entries of targets in range, item by item
  auto restrict_list = [&](const PinVec<WorkItem>& work, const DBuf<int2>& ent,
                           std::vector<WorkItem>& rwork, DBuf<WorkItem>& d_rwork,
                           DBuf<int2>& d_rent) {
    size_t total = 0;
    for (const WorkItem& w : work) total = std::max(total, (size_t)w.start + w.count);
    std::vector<int2> h(total), out;
    if (total)
      TABI_CUDA(cudaMemcpyAsync(h.data(), ent.p, sizeof(int2) * total, cudaMemcpyDeviceToHost,
                                s));
    TABI_CUDA(cudaStreamSynchronize(s));
    rwork.clear();
    for (const WorkItem& w : work) {
      const int start = (int)out.size();
      for (int k = 0; k < w.count; ++k) {
        const int2 e = h[(size_t)w.start + k];
        if (e.x >= t0 && e.x < t1) out.push_back(e);
      }
      const int cnt = (int)out.size() - start;
      if (cnt > 0) rwork.push_back(WorkItem{w.node, start, cnt, w.mslot});
    }
    d_rwork.alloc(std::max<size_t>(rwork.size(), 1));
    d_rent.alloc(std::max<size_t>(out.size(), 1));
    if (!rwork.empty())
      TABI_CUDA(cudaMemcpyAsync(d_rwork.p, rwork.data(), sizeof(WorkItem) * rwork.size(),
                                cudaMemcpyHostToDevice, s));
    if (!out.empty())
      TABI_CUDA(cudaMemcpyAsync(d_rent.p, out.data(), sizeof(int2) * out.size(),
                                cudaMemcpyHostToDevice, s));
  };
  restrict_list(T.far_work, T.d_far_ent, T.r_far_work, T.d_r_far_work, T.d_r_far_ent);
  restrict_list(T.near_work, T.d_near_ent, T.r_near_work, T.d_r_near_work, T.d_r_near_ent);
  // the preconditioner's leaves in range, in the apply's big / small classes
  std::vector<int> big, small;
  for (int l = 0; l < T.nleaf; ++l) {
    const int c = T.leaves[l], b0 = T.ibeg[c], nm = T.num[c];
    if (b0 >= t0 && b0 + nm <= t1) (2 * nm > 512 ? big : small).push_back(l);
  }
  auto by_size = [&](int a, int b) { return T.num[T.leaves[a]] > T.num[T.leaves[b]]; };
  std::sort(big.begin(), big.end(), by_size);
  std::sort(small.begin(), small.end(), by_size);
  T.r_solve_big = (int)big.size();
  T.r_solve_small = (int)small.size();
  big.insert(big.end(), small.begin(), small.end());
  T.d_r_solve_list.alloc(std::max<size_t>(big.size(), 1));
  if (!big.empty())
    TABI_CUDA(cudaMemcpyAsync(T.d_r_solve_list.p, big.data(), sizeof(int) * big.size(),
                              cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  T.ranged = true;
  T.rt0 = t0;
  T.rt1 = t1;
}

}  // namespace tabi
