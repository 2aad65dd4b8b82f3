// precond.cu -- the leaf-block-diagonal preconditioner (LEAFMATVECpara,
// treecode3d_pb.f:1393-1542) and the diagonal one (MSOLVEprec, main.f90:532-542).
//
// Per leaf of n faces the reference assembles the 2n x 2n column-major block
//   row i, col j      : -A_j (G1 - eps G2)      (j != i)       = -A_j K1
//   row i+n, col j    : -A_j (G0 - Gk)                         = -A_j K2
//   row i, col j+n    : -A_j (G4 - G3)                         = -A_j K3
//   row i+n, col j+n  : -A_j (G10 - G20/eps)                   = -A_j K4
//   diagonal          : pre1 (rows 1..n), pre2 (rows n+1..2n)
// (K2 and K3 sit in the transposed block positions relative to the matvec
// operator -- reproduced as is), then calls DGETRF (which, with the vendored
// testing ILAENV, is the unblocked recursive DGETRF2: partial pivoting on the
// largest |a|, first index on ties) and DGETRS, on EVERY call.  The block
// never changes, so here it is assembled and factored once per tree
// (right-looking LU with partial pivoting, the same pivot rule; one CTA per
// leaf) and every apply is a blocked forward/back substitution.
#include <algorithm>

#include "bie_kernels.cuh"
#include "tabi_impl.cuh"

namespace tabi {

namespace {

constexpr int kAsmCols = 8;

// grid: one block per (leaf, 8-column tile); tiles given as (leaf, j0)
__global__ void __launch_bounds__(256) assemble_kernel(
    const int2* __restrict__ tiles, const int2* __restrict__ leaf_rng,
    const int64_t* __restrict__ blk_off, const double* __restrict__ px,
    const double* __restrict__ py, const double* __restrict__ pz, const double* __restrict__ nx,
    const double* __restrict__ ny, const double* __restrict__ nz,
    const double* __restrict__ area, double kappa, double eps, double* __restrict__ lu) {
  int2 tl = tiles[blockIdx.x];
  int2 lr = leaf_rng[tl.x];
  int ib = lr.x, n = lr.y, m = 2 * n;
  double* A = lu + blk_off[tl.x];
  const double pre1 = 0.5 * (1.0 + eps), pre2 = 0.5 * (1.0 + 1.0 / eps);
  const double inv_eps = 1.0 / eps;
  for (int jj = 0; jj < kAsmCols; ++jj) {
    int j = tl.y + jj;
    if (j >= n) break;
    double sx = px[ib + j], sy = py[ib + j], sz = pz[ib + j];
    double vx = nx[ib + j], vy = ny[ib + j], vz = nz[ib + j];
    double Aj = area[ib + j];
    double* c1 = A + (size_t)j * m;        // column j
    double* c2 = A + (size_t)(j + n) * m;  // column j + n
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      if (i == j) {
        c1[i] = pre1;
        c1[i + n] = 0.0;
        c2[i] = 0.0;
        c2[i + n] = pre2;
        continue;
      }
      int t = ib + i;
      double K1, K2, K3, K4;
      bie4<double>(sx - px[t], sy - py[t], sz - pz[t], nx[t], ny[t], nz[t], vx, vy, vz, kappa,
                   eps, inv_eps, K1, K2, K3, K4);
      c1[i] = -K1 * Aj;
      c1[i + n] = -K2 * Aj;
      c2[i] = -K3 * Aj;
      c2[i + n] = -K4 * Aj;
    }
  }
}

constexpr int kLuThreads = 256;
constexpr int kNB = 32;   // panel width
constexpr int kTM = 64;   // trailing-update tile

__device__ __forceinline__ void argmax_merge(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// Right-looking blocked LU with partial pivoting of one leaf block per CTA.
__global__ void __launch_bounds__(kLuThreads) lu_kernel(const int2* __restrict__ leaf_rng,
                                                        const int64_t* __restrict__ blk_off,
                                                        double* __restrict__ lu,
                                                        int* __restrict__ piv,
                                                        int* __restrict__ info) {
  int leaf = blockIdx.x;
  int2 lr = leaf_rng[leaf];
  int m = 2 * lr.y;
  double* A = lu + blk_off[leaf];
  int* ip = piv + 2 * lr.x;
  __shared__ double s_v[kLuThreads / 32];
  __shared__ int s_i[kLuThreads / 32];
  __shared__ int s_p;
  __shared__ double sL[kTM][kNB + 1];
  __shared__ double sU[kNB][kTM + 1];
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int my_info = 0;
  for (int k0 = 0; k0 < m; k0 += kNB) {
    int nb = min(kNB, m - k0);
    // ---- panel factorization (columns k0 .. k0+nb-1)
    for (int kk = k0; kk < k0 + nb; ++kk) {
      double* col = A + (size_t)kk * m;
      double bv = -1.0;
      int bi = m;
      for (int i = kk + tid; i < m; i += blockDim.x) argmax_merge(bv, bi, fabs(col[i]), i);
      for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        argmax_merge(bv, bi, v2, i2);
      }
      if (lane == 0) {
        s_v[warp] = bv;
        s_i[warp] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double v = s_v[0];
        int i = s_i[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) argmax_merge(v, i, s_v[w], s_i[w]);
        s_p = i;
        ip[kk] = i + 1;  // 1-based like LAPACK
      }
      __syncthreads();
      int p = s_p;
      double pv = col[p];
      if (pv == 0.0) {
        if (my_info == 0) my_info = kk + 1;
        __syncthreads();
        continue;  // DGETRF2: no swap, no scaling, INFO set
      }
      if (p != kk)
        for (int c = tid; c < m; c += blockDim.x) {
          double* cc = A + (size_t)c * m;
          double t = cc[kk];
          cc[kk] = cc[p];
          cc[p] = t;
        }
      __syncthreads();
      pv = col[kk];
      if (fabs(pv) >= 2.2250738585072014e-308) {
        double r = 1.0 / pv;
        for (int i = kk + 1 + tid; i < m; i += blockDim.x) col[i] *= r;
      } else {
        for (int i = kk + 1 + tid; i < m; i += blockDim.x) col[i] /= pv;
      }
      __syncthreads();
      // rank-1 update of the rest of the panel
      int ncol = k0 + nb - kk - 1;
      int nrow = m - kk - 1;
      for (int q = tid; q < ncol * nrow; q += blockDim.x) {
        int c = kk + 1 + q / nrow;
        int i = kk + 1 + q % nrow;
        double* cc = A + (size_t)c * m;
        cc[i] = fma(-col[i], cc[kk], cc[i]);
      }
      __syncthreads();
    }
    int c1 = k0 + nb;
    if (c1 >= m) break;
    // ---- U12 = L11^{-1} A12 (unit lower), one column per thread
    for (int c = c1 + tid; c < m; c += blockDim.x) {
      double* cc = A + (size_t)c * m;
      double xv[kNB];
#pragma unroll
      for (int r = 0; r < kNB; ++r) xv[r] = (r < nb) ? cc[k0 + r] : 0.0;
#pragma unroll
      for (int r = 1; r < kNB; ++r) {
        if (r < nb) {
          double s = xv[r];
#pragma unroll
          for (int q = 0; q < kNB; ++q)
            if (q < r) s = fma(-A[(size_t)(k0 + q) * m + k0 + r], xv[q], s);
          xv[r] = s;
        }
      }
#pragma unroll
      for (int r = 0; r < kNB; ++r)
        if (r < nb) cc[k0 + r] = xv[r];
    }
    __syncthreads();
    // ---- A22 -= L21 * U12, 64x64 tiles, 4x4 per thread
    int rows = m - c1;
    int ntr = (rows + kTM - 1) / kTM;
    int tr = tid / 16, tc = tid % 16;  // 16 x 16 thread grid
    for (int tile = 0; tile < ntr * ntr; ++tile) {
      int r0 = c1 + (tile / ntr) * kTM;
      int cb = c1 + (tile % ntr) * kTM;
      // load L21 tile (kTM x nb) and U12 tile (nb x kTM)
      for (int q = tid; q < kTM * kNB; q += blockDim.x) {
        int r = q % kTM, k = q / kTM;
        int gr = r0 + r;
        sL[r][k] = (gr < m && k < nb) ? A[(size_t)(k0 + k) * m + gr] : 0.0;
      }
      for (int q = tid; q < kNB * kTM; q += blockDim.x) {
        int k = q % kNB, c = q / kNB;
        int gc = cb + c;
        sU[k][c] = (gc < m && k < nb) ? A[(size_t)gc * m + k0 + k] : 0.0;
      }
      __syncthreads();
      double acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
#pragma unroll 8
      for (int k = 0; k < kNB; ++k) {
        double lv[4], uv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) lv[a] = sL[tr + 16 * a][k];
#pragma unroll
        for (int b = 0; b < 4; ++b) uv[b] = sU[k][tc + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fma(lv[a], uv[b], acc[a][b]);
      }
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        int gc = cb + tc + 16 * b;
        if (gc >= m) continue;
        double* cc = A + (size_t)gc * m;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          int gr = r0 + tr + 16 * a;
          if (gr < m) cc[gr] -= acc[a][b];
        }
      }
      __syncthreads();
    }
  }
  if (tid == 0) info[leaf] = my_info;
}

constexpr int kSolveThreads = 256;

// Forward/back substitution with the factored block (DGETRS 'N').
__global__ void __launch_bounds__(kSolveThreads) solve_kernel(
    const int2* __restrict__ leaf_rng, const int64_t* __restrict__ blk_off,
    const double* __restrict__ lu, const int* __restrict__ piv, int N,
    const double* __restrict__ r, double* __restrict__ z) {
  extern __shared__ double xs[];
  int leaf = blockIdx.x;
  int2 lr = leaf_rng[leaf];
  int n = lr.y, m = 2 * n, ib = lr.x;
  const double* A = lu + blk_off[leaf];
  const int* ip = piv + 2 * ib;
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < n; i += blockDim.x) {
    xs[i] = r[ib + i];
    xs[n + i] = r[N + ib + i];
  }
  __syncthreads();
  if (tid == 0)  // DLASWP, increasing k
    for (int k = 0; k < m; ++k) {
      int p = ip[k] - 1;
      if (p != k) {
        double t = xs[k];
        xs[k] = xs[p];
        xs[p] = t;
      }
    }
  __syncthreads();
  // L y = P r (unit lower)
  for (int k0 = 0; k0 < m; k0 += 32) {
    int nb = min(32, m - k0);
    if (warp == 0) {
      double v = (lane < nb) ? xs[k0 + lane] : 0.0;
      for (int kk = 0; kk < nb; ++kk) {
        double xk = __shfl_sync(0xffffffffu, v, kk);
        if (lane > kk && lane < nb) v = fma(-A[(size_t)(k0 + kk) * m + k0 + lane], xk, v);
      }
      if (lane < nb) xs[k0 + lane] = v;
    }
    __syncthreads();
    for (int i = k0 + nb + tid; i < m; i += blockDim.x) {
      double s = xs[i];
      for (int q = 0; q < nb; ++q) s = fma(-A[(size_t)(k0 + q) * m + i], xs[k0 + q], s);
      xs[i] = s;
    }
    __syncthreads();
  }
  // U x = y
  for (int kend = m; kend > 0; kend -= 32) {
    int k0 = max(0, kend - 32);
    int nb = kend - k0;
    if (warp == 0) {
      double v = (lane < nb) ? xs[k0 + lane] : 0.0;
      for (int kk = nb - 1; kk >= 0; --kk) {
        if (lane == kk) v = v / A[(size_t)(k0 + kk) * m + k0 + kk];
        double xk = __shfl_sync(0xffffffffu, v, kk);
        if (lane < kk) v = fma(-A[(size_t)(k0 + kk) * m + k0 + lane], xk, v);
      }
      if (lane < nb) xs[k0 + lane] = v;
    }
    __syncthreads();
    for (int i = tid; i < k0; i += blockDim.x) {
      double s = xs[i];
      for (int q = 0; q < nb; ++q) s = fma(-A[(size_t)(k0 + q) * m + i], xs[k0 + q], s);
      xs[i] = s;
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += blockDim.x) {
    z[ib + i] = xs[i];
    z[N + ib + i] = xs[n + i];
  }
}

__global__ void diag_kernel(const double* r, double* z, int n, double s1, double s2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = r[i] / s1;
  else if (i < 2 * n) z[i] = r[i] / s2;
}

}  // namespace

void build_precond(Handle& H, cudaStream_t s) {
  Tree& T = H.tree;
  if (H.prm.iprcd != 1) {
    H.has_precond = true;
    return;
  }
  const int nl = T.nleaf;
  std::vector<int2> rng(nl);
  T.blk_off.resize(nl);
  int64_t off = 0;
  std::vector<int2> tiles;
  for (int l = 0; l < nl; ++l) {
    int c = T.leaves[l];
    rng[l] = make_int2(T.ibeg[c], T.num[c]);
    T.blk_off[l] = off;
    off += 4LL * T.num[c] * T.num[c];
    for (int j = 0; j < T.num[c]; j += kAsmCols) tiles.push_back(make_int2(l, j));
  }
  T.d_lu.alloc(std::max<int64_t>(off, 1));
  T.d_piv.alloc(2 * (size_t)H.n);
  T.d_blk_off.alloc(nl);
  T.d_leaf_rng.alloc(nl);
  DBuf<int2> d_tiles;
  d_tiles.alloc(tiles.size());
  DBuf<int> d_info;
  d_info.alloc(nl);
  TABI_CUDA(cudaMemcpyAsync(T.d_blk_off.p, T.blk_off.data(), sizeof(int64_t) * nl,
                            cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(T.d_leaf_rng.p, rng.data(), sizeof(int2) * nl, cudaMemcpyHostToDevice,
                            s));
  TABI_CUDA(cudaMemcpyAsync(d_tiles.p, tiles.data(), sizeof(int2) * tiles.size(),
                            cudaMemcpyHostToDevice, s));
  double eps = H.prm.eps1 / H.prm.eps0;
  { TABI_K(K_ASSEMBLE, s); assemble_kernel<<<(int)tiles.size(), 256, 0, s>>>(d_tiles.p, T.d_leaf_rng.p, T.d_blk_off.p,
                                                    H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p,
                                                    H.d_ny.p, H.d_nz.p, H.d_area.p,
                                                    H.prm.kappa, eps, T.d_lu.p); }
  { TABI_K(K_LU, s); lu_kernel<<<nl, kLuThreads, 0, s>>>(T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p, T.d_piv.p,
                                      d_info.p); }
  std::vector<int> info(nl);
  TABI_CUDA(cudaMemcpyAsync(info.data(), d_info.p, sizeof(int) * nl, cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  for (int l = 0; l < nl; ++l)
    if (info[l] != 0)
      throw Error(TABI_ERR_SINGULAR, "leaf block " + std::to_string(l) +
                                         " is singular (DGETRF info " +
                                         std::to_string(info[l]) + ")");
  H.has_precond = true;
}

void msolve_dev(Handle& H, const double* r, double* z, cudaStream_t s) {
  Tree& T = H.tree;
  const int n = H.n;
  double eps = H.prm.eps1 / H.prm.eps0;
  if (H.prm.iprcd != 1) {
    { TABI_K(K_SOLVE, s); diag_kernel<<<ceil_div(2 * n, 256), 256, 0, s>>>(r, z, n, 0.5 * (1.0 + eps),
                                                     0.5 * (1.0 + 1.0 / eps)); }
    TABI_CUDA(cudaGetLastError());
    return;
  }
  size_t smem = sizeof(double) * 2 * (size_t)T.max_leaf;
  TABI_REQUIRE(smem <= 200 * 1024, TABI_ERR_LIMIT, "leaf too large for the block solve");
  if (smem > 48 * 1024)
    TABI_CUDA(cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  { TABI_K(K_SOLVE, s); solve_kernel<<<T.nleaf, kSolveThreads, smem, s>>>(T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p,
                                                    T.d_piv.p, n, r, z); }
  TABI_CUDA(cudaGetLastError());
}

}  // namespace tabi
