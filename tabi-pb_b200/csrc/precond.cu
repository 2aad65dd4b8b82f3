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
// (right-looking LU with partial pivoting, the same pivot rule, batched over
// all leaves) and every apply is a blocked forward/back substitution.
#include <algorithm>
#include <optional>
#include <climits>

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

// Right-looking blocked LU with partial pivoting of one leaf block per CTA,
// panel in global memory (used for blocks too large for the shared-memory
// panel of the batched kernels).
__global__ void __launch_bounds__(kLuThreads) lu_kernel(const int* __restrict__ leaves,
                                                        const int2* __restrict__ leaf_rng,
                                                        const int64_t* __restrict__ blk_off,
                                                        double* __restrict__ lu,
                                                        int* __restrict__ piv,
                                                        int* __restrict__ info,
                                                        int skip_max_m) {
  int leaf = leaves[blockIdx.x];
  int2 lr = leaf_rng[leaf];
  int m = 2 * lr.y;
  if (m <= skip_max_m) return;  // factored by the batched kernels
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
      // a column of NaNs offers no candidate: the diagonal row stays the pivot
      double bv = -1.0;
      int bi = kk;
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


// Batched, level-synchronous right-looking LU with partial pivoting for all
// leaf blocks of order m <= kPanelMaxM at once, in outer blocks of kOB columns
// (the plan is built in build_precond).  Inside an outer block, panel step s
// (k0 = 32 s) is three launches over every block that still has columns left:
//   lu_panel_reg_kernel / lu_panel_kernel  one CTA per block: the 32-column
//                    panel (rows k0..m-1) as two 16-column halves -- pivot
//                    search (largest |a|, first index on ties, as IDAMAX), row
//                    swap, scaling, rank-1 updates; the second half first takes
//                    the first half's swaps, TRSM and GEMM update (DGETRF2's
//                    recursion, one level);
//   lu_strip_kernel  one CTA per 128-column strip of the outer block: the
//                    panel's row swaps, and for strips right of the panel
//                    U12 = L11^{-1} A12; strips left of the panel only take
//                    swaps (LAPACK applies every pivot to the L columns too);
//   lu_gemm_kernel   one CTA per 64 x 64 tile of the outer block right of the
//                    panel: A22 -= L21 U12 with k = 32.
// After the outer block, its row interchanges reach the columns left and right
// of it at once (lu_swapmap_kernel + lu_rowswap_kernel), U12 of the columns
// right of it follows by 32-row TRSM + small GEMM steps, and the trailing
// matrix takes one kOB-deep lu_gemm_kernel update.  The trailing updates of
// all blocks run concurrently across the GPU.
constexpr int kBP = 32;            // panel width
constexpr int kSP = 16;            // panel half held in shared memory
constexpr int kPanelMaxM = 1536;   // half panel of 1536 x 16 doubles = 192 KB
constexpr int kPT = 256;           // panel kernel threads
constexpr int kUT = 256;           // strip / gemm kernel threads
constexpr int kUC = 128;           // strip width
constexpr int kGT = 64;            // gemm tile
constexpr int kOB = 256;           // outer block: columns right of it are updated once per block
constexpr int kLuSmallBlock = 512; // blocks up to this order factor on the side stream

// Factor columns [c0l, c0l + nb) of the panel held in P (local column c of
// the half is P + c * mr, local row r = global row k0 + r) starting at local
// row r0; records 1-based global pivots.
__device__ void panel_factor(double* P, int mr, int r0, int nb, int k0, int* ip, int* info,
                             int leaf, double* s_v, int* s_i, int* s_p) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = 0; j < nb; ++j) {
    const int lr0 = r0 + j;  // local row of the diagonal
    double* col = P + (size_t)j * mr;
    // a column of NaNs offers no candidate: the diagonal row stays the pivot
    double bv = -1.0;
    int bi = lr0;
    for (int i = lr0 + tid; i < mr; i += kPT) argmax_merge(bv, bi, fabs(col[i]), i);
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
    if (warp == 0) {
      double v = (lane < kPT / 32) ? s_v[lane] : -1.0;
      int i = (lane < kPT / 32) ? s_i[lane] : mr;
      for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        argmax_merge(v, i, v2, i2);
      }
      if (lane == 0) *s_p = i;
    }
    __syncthreads();
    const int p = *s_p;
    const double pv = col[p];
    if (pv == 0.0) {  // DGETRF2: INFO set, no swap, no scaling
      if (tid == 0) {
        atomicCAS(&info[leaf], 0, k0 + lr0 + 1);
        ip[k0 + lr0] = k0 + lr0 + 1;
      }
      __syncthreads();
      continue;
    }
    if (tid == 0) ip[k0 + lr0] = k0 + p + 1;  // 1-based, like LAPACK
    if (p != lr0 && tid < nb) {
      double* cc = P + (size_t)tid * mr;
      double t = cc[lr0];
      cc[lr0] = cc[p];
      cc[p] = t;
    }
    __syncthreads();
    const double pk = col[lr0];
    const bool recip = fabs(pk) >= 2.2250738585072014e-308;
    const double rcp = 1.0 / pk;
    for (int i = lr0 + 1 + tid; i < mr; i += kPT) {
      double l = recip ? col[i] * rcp : col[i] / pk;
      col[i] = l;
      for (int c = j + 1; c < nb; ++c) {
        double* cc = P + (size_t)c * mr;
        cc[i] = fma(-l, cc[lr0], cc[i]);
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kPT) lu_panel_kernel(const int* __restrict__ items, int k0,
                                                       const int2* __restrict__ leaf_rng,
                                                       const int64_t* __restrict__ blk_off,
                                                       double* __restrict__ lu,
                                                       int* __restrict__ piv,
                                                       int* __restrict__ info) {
  extern __shared__ double P[];
  __shared__ double s_v[kPT / 32];
  __shared__ int s_i[kPT / 32];
  __shared__ int s_p;
  __shared__ double sL11[kSP][kSP + 1];
  __shared__ int s_rows[2 * kSP], s_src[2 * kSP];
  const int leaf = items[blockIdx.x];
  const int2 lr = leaf_rng[leaf];
  const int m = 2 * lr.y;
  const int nb = min(kBP, m - k0), mr = m - k0;
  const int nb1 = min(kSP, nb), nb2 = nb - nb1;
  double* A = lu + blk_off[leaf];
  int* ip = piv + 2 * lr.x;
  const int tid = threadIdx.x;
  // ---- first half
  for (int q = tid; q < nb1 * mr; q += kPT) {
    int c = q / mr, r = q - c * mr;
    P[q] = A[(size_t)(k0 + c) * m + k0 + r];
  }
  __syncthreads();
  panel_factor(P, mr, 0, nb1, k0, ip, info, leaf, s_v, s_i, &s_p);
  for (int q = tid; q < nb1 * mr; q += kPT) {
    int c = q / mr, r = q - c * mr;
    A[(size_t)(k0 + c) * m + k0 + r] = P[q];
  }
  if (nb2 == 0) return;
  for (int q = tid; q < nb1 * nb1; q += kPT) {
    int c = q / nb1, r = q - c * nb1;
    sL11[r][c] = P[(size_t)c * mr + r];
  }
  __syncthreads();
  // ---- second half: load, first half's swaps, TRSM, GEMM update, factor
  const int c2 = k0 + kSP;
  for (int q = tid; q < nb2 * mr; q += kPT) {
    int c = q / mr, r = q - c * mr;
    P[q] = A[(size_t)(c2 + c) * m + k0 + r];
  }
  __syncthreads();
  if (tid < nb2) {
    double* cc = P + (size_t)tid * mr;
    for (int j = 0; j < nb1; ++j) {
      int p = ip[k0 + j] - 1 - k0;
      if (p != j) {
        double t = cc[j];
        cc[j] = cc[p];
        cc[p] = t;
      }
    }
    double x[kSP];
#pragma unroll
    for (int r = 0; r < kSP; ++r) x[r] = (r < nb1) ? cc[r] : 0.0;
#pragma unroll
    for (int r = 1; r < kSP; ++r) {
      double acc = x[r];
#pragma unroll
      for (int q = 0; q < kSP; ++q)
        if (q < r) acc = fma(-sL11[r][q], x[q], acc);
      x[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < kSP; ++r)
      if (r < nb1) cc[r] = x[r];
  }
  __syncthreads();
  // rows kSP.. of the second half -= L21 (first half, global) * U (rows 0..15 of P)
  for (int i = kSP + tid; i < mr; i += kPT) {
    double l[kSP];
#pragma unroll
    for (int q = 0; q < kSP; ++q) l[q] = A[(size_t)(k0 + q) * m + k0 + i];
    for (int c = 0; c < nb2; ++c) {
      double* cc = P + (size_t)c * mr;
      double acc = cc[i];
#pragma unroll
      for (int q = 0; q < kSP; ++q) acc = fma(-l[q], cc[q], acc);
      cc[i] = acc;
    }
  }
  __syncthreads();
  panel_factor(P, mr, kSP, nb2, k0, ip, info, leaf, s_v, s_i, &s_p);
  for (int q = tid; q < nb2 * mr; q += kPT) {
    int c = q / mr, r = q - c * mr;
    A[(size_t)(c2 + c) * m + k0 + r] = P[q];
  }
  // the second half's swaps on the first half's columns (gathered through
  // shared memory: rows touched and, for each, the row its value comes from)
  __syncthreads();
  if (tid == 0) {
    int nr = 0;
    for (int j = kSP; j < nb; ++j) s_rows[nr++] = k0 + j;
    for (int j = kSP; j < nb; ++j) {
      int p = ip[k0 + j] - 1;
      bool have = false;
      for (int q = 0; q < nr; ++q) have |= (s_rows[q] == p);
      if (!have) s_rows[nr++] = p;
    }
    for (int q = 0; q < nr; ++q) s_src[q] = s_rows[q];
    for (int j = kSP; j < nb; ++j) {
      int p = ip[k0 + j] - 1, a = -1, b = -1;
      for (int q = 0; q < nr; ++q) {
        if (s_rows[q] == k0 + j) a = q;
        if (s_rows[q] == p) b = q;
      }
      int t = s_src[a];
      s_src[a] = s_src[b];
      s_src[b] = t;
    }
    s_p = nr;
  }
  __syncthreads();
  const int nr = s_p;
  for (int q = tid; q < nr * nb1; q += kPT) {
    int row = q / nb1, c = q - row * nb1;
    P[q] = A[(size_t)(k0 + c) * m + s_src[row]];
  }
  __syncthreads();
  for (int q = tid; q < nr * nb1; q += kPT) {
    int row = q / nb1, c = q - row * nb1;
    A[(size_t)(k0 + c) * m + s_rows[row]] = P[q];
  }
}

// The same panel step with the panel half held in registers: thread t owns
// the local rows t + NT q (q < R), all 16 columns of the half.  Per column a
// single CTA barrier: before it, every warp publishes its best candidate
// (|value|, row) and that row's 16 values, and the owner of the diagonal row
// publishes it; after it, every warp reduces the candidates itself, takes the
// winner's row as the pivot row, and each thread swaps, scales and updates its
// own rows.  Candidates are double-buffered by step parity, so a fast warp's
// writes of step j+1 cannot meet a slow warp's reads of step j.  The column
// in work is always register 0: after each step a thread rotates its rows'
// 16 registers left by one, so the column loop needs no unrolling (an
// unrolled loop overflowed the instruction cache) and after 16 steps the
// registers are back in column order.  The operations and their order equal
// lu_panel_kernel's, so the factors are the same bit for bit.
constexpr int kRegMaxRows = 2;  // rows per thread of the register panel

struct PanelShared {
  static constexpr int kMaxW = 16;
  double cand[2][kMaxW][kSP];  // each warp's best row (rotated order)
  double cv[2][kMaxW];         // its |value|
  int ci[2][kMaxW];            // its local row
  double lrow[2][kSP];         // the diagonal row before the swap
  int piv[kBP];                // local pivot rows of the panel's columns
  double u12[kSP][kSP + 1];    // second half: U12 after the TRSM
};

template <int NT, int R>
__device__ __forceinline__ void panel_half_reg(double (&a)[R][kSP], int mr, int rbase, int nbh,
                                               int k0, int& st, int* ip, int* info, int leaf,
                                               PanelShared& S) {
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll 1
  for (int j = 0; j < kSP; ++j) {  // nbh pivot steps, then rotations only
    if (j < nbh) {                 // uniform over the CTA
      const int lr0 = rbase + j, b = st & 1, rem = nbh - j;
      double bv = -1.0;
      int bi = INT_MAX;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int r = tid + NT * q;
        if (r >= lr0 && r < mr) argmax_merge(bv, bi, fabs(a[q][0]), r);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        argmax_merge(bv, bi, v2, i2);
      }
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int r = tid + NT * q;
        if (r == bi) {
#pragma unroll
          for (int c = 0; c < kSP; ++c) S.cand[b][warp][c] = a[q][c];
        }
        if (r == lr0) {
#pragma unroll
          for (int c = 0; c < kSP; ++c) S.lrow[b][c] = a[q][c];
        }
      }
      if (lane == 0) {
        S.cv[b][warp] = bv;
        S.ci[b][warp] = bi;
      }
      __syncthreads();
      double v = lane < NW ? S.cv[b][lane] : -1.0;
      int p = lane < NW ? S.ci[b][lane] : INT_MAX;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, p, o);
        argmax_merge(v, p, v2, i2);
      }
      // no candidate at all (a column of NaNs): keep the diagonal row
      const double* urow = p == INT_MAX ? S.lrow[b] : S.cand[b][(p % NT) >> 5];
      if (p == INT_MAX) p = lr0;
      const double pv = urow[0];
      if (pv == 0.0) p = lr0;  // a zero column: no interchange
      if (tid == 0) {
        S.piv[lr0] = p;
        ip[k0 + lr0] = k0 + p + 1;  // 1-based, like LAPACK
      }
      if (pv != 0.0) {
        const bool recip = fabs(pv) >= 2.2250738585072014e-308;
        const double rcp = 1.0 / pv;
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int r = tid + NT * q;
          if (p != lr0) {
            if (r == p) {
#pragma unroll
              for (int c = 0; c < kSP; ++c) a[q][c] = S.lrow[b][c];
            } else if (r == lr0) {
#pragma unroll
              for (int c = 0; c < kSP; ++c) a[q][c] = urow[c];
            }
          }
          if (r > lr0 && r < mr) {
            const double l = recip ? a[q][0] * rcp : a[q][0] / pv;
            a[q][0] = l;
#pragma unroll
            for (int c = 1; c < kSP; ++c)
              if (c < rem) a[q][c] = fma(-l, urow[c], a[q][c]);
          }
        }
      } else if (tid == 0) {  // DGETRF2: INFO set, no swap, no scaling
        atomicCAS(&info[leaf], 0, k0 + lr0 + 1);
      }
      ++st;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const double t0 = a[q][0];
#pragma unroll
      for (int c = 0; c < kSP - 1; ++c) a[q][c] = a[q][c + 1];
      a[q][kSP - 1] = t0;
    }
  }
}

// Source row of local row r after the row interchanges (j, piv[j]) for
// j = j0 .. j1-1 were applied in order: the swaps replayed backwards.
__device__ __forceinline__ int swapped_source(int r, const int* piv, int j0, int j1) {
  for (int j = j1 - 1; j >= j0; --j) {
    const int pj = piv[j];
    if (r == j) r = pj;
    else if (r == pj) r = j;
  }
  return r;
}

template <int NT, int R>
__global__ void __launch_bounds__(NT, 512 / NT) lu_panel_reg_kernel(
    const int* __restrict__ items, int k0, const int2* __restrict__ leaf_rng,
    const int64_t* __restrict__ blk_off, double* __restrict__ lu, int* __restrict__ piv,
    int* __restrict__ info) {
  static_assert(NT / 32 <= PanelShared::kMaxW, "too many warps");
  __shared__ PanelShared S;
  const int leaf = items[blockIdx.x];
  const int2 lr = leaf_rng[leaf];
  const int m = 2 * lr.y;
  const int nb = min(kBP, m - k0), mr = m - k0;
  const int nb1 = min(kSP, nb), nb2 = nb - nb1;
  double* A = lu + blk_off[leaf];
  int* ip = piv + 2 * lr.x;
  const int tid = threadIdx.x;
  int st = 0;
  double a[R][kSP];
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {  // the two 16-column halves
    const int nbh = h == 0 ? nb1 : nb2, cb = k0 + kSP * h;
    if (nbh == 0) break;
    if (h == 0) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int r = tid + NT * q;
#pragma unroll
        for (int c = 0; c < kSP; ++c)
          a[q][c] = (r < mr && c < nb1) ? A[(size_t)(k0 + c) * m + k0 + r] : 0.0;
      }
    } else {
      // load through the first half's swaps, TRSM, GEMM update
      __syncthreads();  // pivots and the stored first half visible to all
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int r = tid + NT * q;
        const int src = r < mr ? swapped_source(r, S.piv, 0, kSP) : r;
#pragma unroll
        for (int c = 0; c < kSP; ++c)
          a[q][c] = (r < mr && c < nb2) ? A[(size_t)(cb + c) * m + k0 + src] : 0.0;
      }
      if (tid < 32) {  // U12 = L11^{-1} A12: rows 0..15 are lanes 0..15, q = 0
        const int lane = tid;
        double l11[kSP];
#pragma unroll
        for (int q = 0; q < kSP; ++q)
          l11[q] = lane < kSP ? A[(size_t)(k0 + q) * m + k0 + lane] : 0.0;
#pragma unroll
        for (int q = 0; q < kSP - 1; ++q)
#pragma unroll
          for (int c = 0; c < kSP; ++c) {
            const double x = __shfl_sync(0xffffffffu, a[0][c], q);
            if (lane > q && lane < kSP) a[0][c] = fma(-l11[q], x, a[0][c]);
          }
        if (lane < kSP)
#pragma unroll
          for (int c = 0; c < kSP; ++c) S.u12[lane][c] = a[0][c];
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < R; ++q) {  // rows 16.. -= L21 U12 (per element k = 0..15 in order)
        const int r = tid + NT * q;
        if (r >= kSP && r < mr) {
          const double* lrow = A + (size_t)k0 * m + k0 + r;
#pragma unroll 1
          for (int k = 0; k < kSP; ++k) {
            const double l = lrow[(size_t)k * m];
#pragma unroll
            for (int c = 0; c < kSP; ++c) a[q][c] = fma(-l, S.u12[k][c], a[q][c]);
          }
        }
      }
    }
    panel_half_reg<NT, R>(a, mr, kSP * h, nbh, k0, st, ip, info, leaf, S);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int r = tid + NT * q;
      if (r < mr) {
#pragma unroll
        for (int c = 0; c < kSP; ++c)
          if (c < nbh) A[(size_t)(cb + c) * m + k0 + r] = a[q][c];
      }
    }
  }
  if (nb2 == 0) return;
  __syncthreads();
  // the second half's swaps on the first half's columns: slot s < 16 is the
  // diagonal row 16 + s, slot 16 + j the pivot row of column 16 + j when it is
  // below the panel's diagonal rows and not named by an earlier column
  constexpr int kPer = (2 * kSP * kSP + NT - 1) / NT;
  double v[kPer];
  int dst[kPer];
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int u = tid + NT * e, s = u / kSP, c = u - s * kSP;
    int t = -1;
    if (s < kSP) {
      if (s < nb2) t = kSP + s;
    } else if (s - kSP < nb2) {
      const int j = s - kSP, pj = S.piv[kSP + j];
      t = pj;
      if (pj < nb) t = -1;
      for (int j2 = 0; j2 < j; ++j2)
        if (S.piv[kSP + j2] == pj) t = -1;
    }
    dst[e] = -1;
    if (u < 2 * kSP * kSP && t >= 0) {
      const int src = swapped_source(t, S.piv, kSP, kSP + nb2);
      if (src != t) {
        v[e] = A[(size_t)(k0 + c) * m + k0 + src];
        dst[e] = t;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int u = tid + NT * e, c = u % kSP;
    if (dst[e] >= 0) A[(size_t)(k0 + c) * m + k0 + dst[e]] = v[e];
  }
}

// item = (leaf, c0, c1, mode): columns [c0, c1) of the leaf block.
// mode 0: left of the panel, the panel's swaps; 1: right of the panel, the
// panel's swaps then U12 = L11^{-1} A12; 3: U12 = L11^{-1} A12 only (columns
// right of an outer block, whose swaps were applied by lu_rowswap_kernel).
__global__ void __launch_bounds__(kUT) lu_strip_kernel(const int4* __restrict__ items, int k0,
                                                       const int2* __restrict__ leaf_rng,
                                                       const int64_t* __restrict__ blk_off,
                                                       double* __restrict__ lu,
                                                       const int* __restrict__ piv) {
  __shared__ double sL11[kBP][kBP + 1];
  __shared__ double sV[2 * kBP][kUC / 4];
  __shared__ int s_rows[2 * kBP], s_src[2 * kBP];
  __shared__ int s_idx[kPanelMaxM];
  __shared__ int s_nr;
  const int4 it = items[blockIdx.x];
  const int leaf = it.x, c0 = it.y, c1 = it.z, mode = it.w;
  const int2 lr = leaf_rng[leaf];
  const int m = 2 * lr.y;
  const int nb = min(kBP, m - k0);
  double* A = lu + blk_off[leaf];
  const int* ip = piv + 2 * lr.x;
  const int tid = threadIdx.x;
  const int ncol = c1 - c0;
  if (mode != 3) {
    // the panel's swaps replayed on the row indices k0..m-1, then the rows
    // whose content moved listed with the row their value comes from
    const int mr = m - k0;
    for (int i = tid; i < mr; i += kUT) s_idx[i] = k0 + i;
    if (tid == 0) s_nr = 0;
    __syncthreads();
    if (tid == 0)
      for (int j = 0; j < nb; ++j) {
        const int p = ip[k0 + j] - 1 - k0;
        const int t = s_idx[j];
        s_idx[j] = s_idx[p];
        s_idx[p] = t;
      }
    __syncthreads();
    for (int i = tid; i < mr; i += kUT)
      if (s_idx[i] != k0 + i) {
        const int q = atomicAdd(&s_nr, 1);  // at most 2 nb rows move
        s_rows[q] = k0 + i;
        s_src[q] = s_idx[i];
      }
    __syncthreads();
    const int nr = s_nr;
    for (int cs = 0; cs < ncol; cs += kUC / 4) {
      const int nc = min(kUC / 4, ncol - cs);
      for (int q = tid; q < nr * nc; q += kUT) {
        int row = q / nc, c = q - row * nc;
        sV[row][c] = A[(size_t)(c0 + cs + c) * m + s_src[row]];
      }
      __syncthreads();
      for (int q = tid; q < nr * nc; q += kUT) {
        int row = q / nc, c = q - row * nc;
        A[(size_t)(c0 + cs + c) * m + s_rows[row]] = sV[row][c];
      }
      __syncthreads();
    }
  }
  if (mode != 1 && mode != 3) return;
  for (int q = tid; q < nb * nb; q += kUT) {
    int c = q / nb, r = q - c * nb;
    sL11[r][c] = A[(size_t)(k0 + c) * m + k0 + r];
  }
  __syncthreads();
  if (tid < ncol) {  // U12 = L11^{-1} A12 (unit lower), one column per thread
    double* cc = A + (size_t)(c0 + tid) * m;
    double x[kBP];
#pragma unroll
    for (int r = 0; r < kBP; ++r) x[r] = (r < nb) ? cc[k0 + r] : 0.0;
#pragma unroll
    for (int r = 1; r < kBP; ++r) {
      double acc = x[r];
#pragma unroll
      for (int q = 0; q < kBP; ++q)
        if (q < r) acc = fma(-sL11[r][q], x[q], acc);
      x[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < kBP; ++r)
      if (r < nb) cc[k0 + r] = x[r];
  }
}

// item = (leaf, r0, c0, ends): C[r0:r0+64, c0:c0+64] -= L[r0:, k0:k0+kd] U[k0:k0+kd, c0:]
// with kd = min(kdepth, m - k0) (32 inside a panel step, kOB for the update
// right of an outer block), staged 32 deep; rows are clipped at re and columns
// at ce, packed as ends = (re << 16) | ce (0: both m).  The C tile is read and
// written once per launch, so a 256-deep update moves an eighth of the bytes
// of eight 32-deep ones.
//
// The 32-deep slices of L and U are copied into shared memory with cp.async
// (16-byte chunks, zero-filled outside the tile), double-buffered: slice k+1
// is in flight while slice k is multiplied.  Every address is 16-byte
// aligned: blocks start at multiples of 4 doubles, m and all row and column
// offsets are even, and a slice's depth is even, so a chunk (two doubles) is
// either wholly inside the tile or wholly outside it.
constexpr int kUPitch = kBP + 2;  // U slice stored by column, 16-byte aligned rows
constexpr size_t kGemmSmem = sizeof(double) * 2 * (kBP * kGT + kGT * kUPitch);

__device__ __forceinline__ void cp_async16(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 16 : 0));
}

__global__ void __launch_bounds__(kUT, 2) lu_gemm_kernel(const int4* __restrict__ items, int k0,
                                                         int kdepth,
                                                         const int2* __restrict__ leaf_rng,
                                                         const int64_t* __restrict__ blk_off,
                                                         double* __restrict__ lu) {
  extern __shared__ double gsm[];
  double* sLb = gsm;                      // [2][kBP][kGT]: L slice, k-major
  double* sUb = gsm + 2 * kBP * kGT;      // [2][kGT][kUPitch]: U slice, by column
  const int4 it = items[blockIdx.x];
  const int leaf = it.x, r0 = it.y, c0 = it.z;
  const int m = 2 * leaf_rng[leaf].y;
  const int re = it.w ? min(m, it.w >> 16) : m, ce = it.w ? min(m, it.w & 0xffff) : m;
  const int kd = min(kdepth, m - k0);
  double* A = lu + blk_off[leaf];
  const int tid = threadIdx.x, tr = tid & 15, tc = tid >> 4;
  // issue the copies of the slice starting at column k0 + kc into buffer buf
  auto load_slice = [&](int kc, int buf) {
    const int nbk = min(kBP, kd - kc), kb = k0 + kc;
    double* sL = sLb + buf * kBP * kGT;
    double* sU = sUb + buf * kGT * kUPitch;
#pragma unroll
    for (int e = 0; e < (kBP * kGT / 2) / kUT; ++e) {
      const int q = tid + kUT * e;
      const int k = q / (kGT / 2), rr = 2 * (q % (kGT / 2));
      const bool ok = k < nbk && r0 + rr < re;
      cp_async16(sL + k * kGT + rr, ok ? A + (size_t)(kb + k) * m + r0 + rr : A, ok);
    }
#pragma unroll
    for (int e = 0; e < (kGT * kBP / 2) / kUT; ++e) {
      const int q = tid + kUT * e;
      const int cc = q / (kBP / 2), kk = 2 * (q % (kBP / 2));
      const bool ok = kk < nbk && c0 + cc < ce;
      cp_async16(sU + cc * kUPitch + kk, ok ? A + (size_t)(c0 + cc) * m + kb + kk : A, ok);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  load_slice(0, 0);
  // C values first (independent of the tiles)
  double cv[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = c0 + tc + 16 * b;
    const double* cc = A + (size_t)c * m;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tr + 16 * a;
      cv[a][b] = (c < ce && r < re) ? cc[r] : 0.0;
    }
  }
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int kc = 0, buf = 0; kc < kd; kc += kBP, buf ^= 1) {
    if (kc + kBP < kd) {
      load_slice(kc + kBP, buf ^ 1);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
    const double* sL = sLb + buf * kBP * kGT;
    const double* sU = sUb + buf * kGT * kUPitch;
#pragma unroll 8
    for (int k = 0; k < kBP; ++k) {
      double lv[4], uv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) lv[a] = sL[k * kGT + tr + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) uv[b] = sU[(tc + 16 * b) * kUPitch + k];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(lv[a], uv[b], acc[a][b]);
    }
    __syncthreads();  // buffer buf is refilled two slices on
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = c0 + tc + 16 * b;
    if (c >= ce) continue;
    double* cc = A + (size_t)c * m;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = r0 + tr + 16 * a;
      if (r < re) cc[r] = cv[a][b] - acc[a][b];
    }
  }
}

// Row interchanges of an outer block (pivots K0 .. K0+nb-1, in order) as one
// gather: per leaf (one CTA), the swaps are replayed on an index array of the
// rows K0.. in shared memory, then the rows whose content moved are listed
// with the row their value comes from (map row of the leaf: 2 kOB rows, 2 kOB
// sources, count; stride 4 kOB + 1 ints).
__global__ void __launch_bounds__(256) lu_swapmap_kernel(const int* __restrict__ leaves, int K0,
                                                         const int2* __restrict__ leaf_rng,
                                                         const int* __restrict__ piv,
                                                         int* __restrict__ map) {
  __shared__ int idx[kPanelMaxM];
  __shared__ int cnt;
  const int leaf = leaves[blockIdx.x];
  const int2 lr = leaf_rng[leaf];
  const int m = 2 * lr.y, nb = min(kOB, m - K0), mr = m - K0;
  const int* ip = piv + 2 * lr.x;
  int* rows = map + (size_t)blockIdx.x * (4 * kOB + 1);
  int* src = rows + 2 * kOB;
  for (int i = threadIdx.x; i < mr; i += blockDim.x) idx[i] = K0 + i;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int j = 0; j < nb; ++j) {
      const int p = ip[K0 + j] - 1 - K0;
      const int t = idx[j];
      idx[j] = idx[p];
      idx[p] = t;
    }
  __syncthreads();
  for (int i = threadIdx.x; i < mr; i += blockDim.x)
    if (idx[i] != K0 + i) {
      const int q = atomicAdd(&cnt, 1);  // at most 2 nb rows move
      rows[q] = K0 + i;
      src[q] = idx[i];
    }
  __syncthreads();
  if (threadIdx.x == 0) rows[4 * kOB] = cnt;
}

// item = (slot, c0, c1, leaf): the outer block's row interchanges on columns
// [c0, c1), through the map of lu_swapmap_kernel (slot = the leaf's map row)
constexpr int kRC = 8;  // columns per pass
__global__ void __launch_bounds__(kUT) lu_rowswap_kernel(const int4* __restrict__ items,
                                                         const int2* __restrict__ leaf_rng,
                                                         const int64_t* __restrict__ blk_off,
                                                         const int* __restrict__ map,
                                                         double* __restrict__ lu) {
  __shared__ double sV[2 * kOB][kRC];
  const int4 it = items[blockIdx.x];
  const int* rows = map + (size_t)it.x * (4 * kOB + 1);
  const int* src = rows + 2 * kOB;
  const int nr = rows[4 * kOB];
  const int m = 2 * leaf_rng[it.w].y;
  double* A = lu + blk_off[it.w];
  for (int cs = it.y; cs < it.z; cs += kRC) {
    const int nc = min(kRC, it.z - cs);
    for (int q = threadIdx.x; q < nr * nc; q += kUT) {
      const int row = q / nc, c = q - row * nc;
      sV[row][c] = A[(size_t)(cs + c) * m + src[row]];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr * nc; q += kUT) {
      const int row = q / nc, c = q - row * nc;
      A[(size_t)(cs + c) * m + rows[row]] = sV[row][c];
    }
    __syncthreads();
  }
}

// After the factorisation, per leaf: the row permutation of all its pivots
// (DLASWP applied to the index vector, so an apply gathers in one parallel
// step) and the inverses of the 32 x 32 diagonal blocks of L (unit lower) and
// U (upper), so that each step of the blocked substitutions is a small GEMV
// instead of a 32-step serial recurrence.
constexpr int kDB = 32;

__global__ void lu_perm_kernel(const int2* __restrict__ leaf_rng, const int* __restrict__ piv,
                               int nleaf, int* __restrict__ perm) {
  int leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= nleaf) return;
  int2 lr = leaf_rng[leaf];
  int m = 2 * lr.y;
  const int* ip = piv + 2 * lr.x;
  int* pm = perm + 2 * lr.x;
  for (int i = 0; i < m; ++i) pm[i] = i;
  for (int k = 0; k < m; ++k) {
    int p = ip[k] - 1;
    if (p != k) {
      int t = pm[k];
      pm[k] = pm[p];
      pm[p] = t;
    }
  }
}

// one warp per (leaf, diagonal block): lane j computes column j of L^{-1} and
// U^{-1} of the block (identity padding past the end of the matrix)
__global__ void lu_diaginv_kernel(const int2* __restrict__ blocks,  // (leaf, k0)
                                  const int2* __restrict__ leaf_rng,
                                  const int64_t* __restrict__ blk_off,
                                  const int64_t* __restrict__ dinv_off,
                                  const double* __restrict__ lu, double* __restrict__ dinv,
                                  int* __restrict__ info) {
  __shared__ double D[4][kDB][kDB + 1];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int2 bk = blocks[blockIdx.x * 4 + w];
  if (bk.x < 0) return;
  int2 lr = leaf_rng[bk.x];
  int m = 2 * lr.y, k0 = bk.y, nb = min(kDB, m - k0);
  const double* A = lu + blk_off[bk.x];
  for (int c = 0; c < kDB; ++c)
    D[w][lane][c] = (c < nb && lane < nb) ? A[(size_t)(k0 + c) * m + k0 + lane]
                                          : (c == lane ? 1.0 : 0.0);
  __syncwarp();
  // a NaN or Inf pivot (coincident faces give a non-finite kernel value) is
  // recorded as -(its 1-based row); DGETRF's exact-zero info takes precedence
  if (lane < nb && !isfinite(D[w][lane][lane])) atomicCAS(&info[bk.x], 0, -(k0 + lane + 1));
  double* Li = dinv + dinv_off[bk.x] + (size_t)(k0 / kDB) * 2 * kDB * kDB;
  double* Ui = Li + kDB * kDB;
  // L^{-1} e_j (unit lower)
  double x[kDB];
#pragma unroll
  for (int i = 0; i < kDB; ++i) {
    double v = (i == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int q = 0; q < kDB; ++q)
      if (q < i) v = fma(-D[w][i][q], x[q], v);
    x[i] = v;
  }
#pragma unroll
  for (int i = 0; i < kDB; ++i) Li[(size_t)lane * kDB + i] = x[i];  // column lane
  // U^{-1} e_j (upper, non-unit)
#pragma unroll
  for (int i = kDB - 1; i >= 0; --i) {
    double v = (i == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int q = 0; q < kDB; ++q)
      if (q > i) v = fma(-D[w][i][q], x[q], v);
    x[i] = v / D[w][i][i];
  }
#pragma unroll
  for (int i = 0; i < kDB; ++i) Ui[(size_t)lane * kDB + i] = x[i];
}

// Forward/back substitution with the factored block (DGETRS 'N') in 32-row
// steps: gather through the pivot permutation, then per step every warp
// applies the diagonal block's precomputed inverse to the step's 32 running
// values (a 32 x 32 GEMV, redundant per warp, so no warp waits for another)
// and updates its rows below (above) with a 32-wide GEMV.  The finalised
// values go to a second array, so one barrier per step suffices: running
// values r (xs in the forward sweep, fin in the backward one) and results are
// never the same words within a step.  No L2 prefetch of the coming steps'
// panels: with all large blocks prefetching at once, one step ahead measured
// 203 us per apply of the bench molecule, two 225 us, four 263 us, and none
// 188 us; the prefetches compete for DRAM and L2 with the loads the steps
// wait for.  Large blocks run with 512 threads; leaf_list selects the
// launch's leaves.  Shared memory: 2 m + NT doubles.
template <int NT>
__global__ void __launch_bounds__(NT, (NT <= 256 ? 4 : 1)) solve_kernel(
    const int2* __restrict__ leaf_rng, const int64_t* __restrict__ blk_off,
    const int64_t* __restrict__ dinv_off, const int* __restrict__ leaf_list,
    const double* __restrict__ lu, const double* __restrict__ dinv,
    const int* __restrict__ perm, int N, const double* __restrict__ r,
    double* __restrict__ z) {
  extern __shared__ double sm[];
  int leaf = leaf_list[blockIdx.x];
  int2 lr = leaf_rng[leaf];
  const int n = lr.y, m = 2 * n, ib = lr.x;
  double* xs = sm;             // forward sweep: running; backward: results
  double* fin = sm + m;        // forward sweep: results; backward: running
  double* ys = sm + 2 * m;     // per warp: the step's 32 diagonal results
  const double* A = lu + blk_off[leaf];
  const double* Di = dinv + dinv_off[leaf];
  const int* pm = perm + 2 * ib;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < m; i += NT) {
    int src = pm[i];
    xs[i] = (src < n) ? r[ib + src] : r[N + ib + src - n];
  }
  // the inverse diagonal block of sweep step t (L blocks 0..nblk-1, then U
  // blocks nblk-1..0), staged into shared memory one step ahead by cp.async
  const int nblk = (m + kDB - 1) / kDB;
  double* dbuf = ys + 32 * (NT / 32);  // [2][kDB * kDB]
  auto stage = [&](int t, int buf) {
    if (t >= 2 * nblk) return;
    const int b = t < nblk ? t : 2 * nblk - 1 - t;
    const double* src = Di + (size_t)b * 2 * kDB * kDB + (t < nblk ? 0 : kDB * kDB);
    for (int e = 2 * tid; e < kDB * kDB; e += 2 * NT) {
      const unsigned d = (unsigned)__cvta_generic_to_shared(dbuf + buf * kDB * kDB + e);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + e));
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  // step t: y = Dinv * run[k0 .. k0+nb), res[k0 ..] = y, run[i] -= A[i, k0 ..
  // k0+nb) y for the rows [i0, i1); the next step's block is copied while the
  // rows are updated.  Four partial sums per dot product keep the dependent
  // FMA chains 8 deep.
  // y = Dinv * run[k0 .. k0+nb) for lane `lane`, four partial sums
  auto diag = [&](int t, int k0, int nb, const double* run) {
    const double* Dblk = dbuf + (t & 1) * kDB * kDB;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    if (nb == kDB) {  // run + k0 is 16-byte aligned: paired loads
      const double2* r2 = reinterpret_cast<const double2*>(run + k0);
#pragma unroll
      for (int q = 0; q < kDB; q += 4) {
        const double2 ra = r2[q / 2], rb = r2[q / 2 + 1];
        v0 = fma(Dblk[q * kDB + lane], ra.x, v0);
        v1 = fma(Dblk[(q + 1) * kDB + lane], ra.y, v1);
        v2 = fma(Dblk[(q + 2) * kDB + lane], rb.x, v2);
        v3 = fma(Dblk[(q + 3) * kDB + lane], rb.y, v3);
      }
    } else {
      for (int q = 0; q < nb; ++q) v0 = fma(Dblk[q * kDB + lane], run[k0 + q], v0);
    }
    return (v0 + v1) + (v2 + v3);
  };
  // run[i] -= A[i, k0 .. k0+nb) y for row i, tq preloaded when `have`
  auto row = [&](int k0, int nb, int i, const double* y, double (&tq)[kDB], bool have,
                 double* run) {
    const double* a = A + (size_t)k0 * m + i;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    if (nb == kDB) {
      if (!have) {
#pragma unroll
        for (int q = 0; q < kDB; ++q) tq[q] = a[(size_t)q * m];
      }
      const double2* y2 = reinterpret_cast<const double2*>(y);
#pragma unroll
      for (int q = 0; q < kDB; q += 4) {
        const double2 ya = y2[q / 2], yb = y2[q / 2 + 1];
        s0 = fma(tq[q], ya.x, s0);
        s1 = fma(tq[q + 1], ya.y, s1);
        s2 = fma(tq[q + 2], yb.x, s2);
        s3 = fma(tq[q + 3], yb.y, s3);
      }
    } else {
      for (int q = 0; q < nb; ++q) s0 = fma(a[(size_t)q * m], y[q], s0);
    }
    run[i] -= (s0 + s1) + (s2 + s3);
  };
  auto step = [&](int t, int k0, int nb, double* run, double* res, int i0, int i1) {
    double tq[kDB];
    if constexpr (NT >= 512) {
      // warp 0 forms y and shares it through shared memory (one more barrier,
      // against 16 warps each reading the 8 KB block); the first row's panel
      // values are loaded meanwhile
      const int ifirst = i0 + tid;
      const bool pre = ifirst < i1 && nb == kDB;
      if (pre) {
        const double* a = A + (size_t)k0 * m + ifirst;
#pragma unroll
        for (int q = 0; q < kDB; ++q) tq[q] = a[(size_t)q * m];
      }
      if (warp == 0) {
        const double v = diag(t, k0, nb, run);
        ys[lane] = v;
        if (lane < nb) res[k0 + lane] = v;
      }
      stage(t + 1, (t + 1) & 1);
      __syncthreads();
      for (int i = ifirst; i < i1; i += NT) row(k0, nb, i, ys, tq, pre && i == ifirst, run);
    } else {
      // every warp forms y itself (no barrier before the rows)
      double* yw = ys + 32 * warp;
      const double v = diag(t, k0, nb, run);
      yw[lane] = v;
      if (warp == 0 && lane < nb) res[k0 + lane] = v;
      __syncwarp();
      stage(t + 1, (t + 1) & 1);
      for (int i = i0 + tid; i < i1; i += NT) row(k0, nb, i, yw, tq, false, run);
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
  };
  stage(0, 0);
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  // L y = P r: running values in xs, y in fin
  for (int k0 = 0, t = 0; k0 < m; k0 += kDB, ++t) {
    const int nb = min(kDB, m - k0);
    step(t, k0, nb, xs, fin, k0 + nb, m);
  }
  // U x = y: running values in fin, x in xs
  for (int b = nblk - 1, t = nblk; b >= 0; --b, ++t) {
    const int k0 = b * kDB;
    const int nb = min(kDB, m - k0);
    step(t, k0, nb, fin, xs, 0, k0);
  }
  for (int i = tid; i < n; i += NT) {
    z[ib + i] = xs[i];
    z[N + ib + i] = xs[n + i];
  }
}

// ---------------------------------------------------------------------------
// Unpivoted blocked LU with a certificate of partial pivoting.
//
// DGETRF2 swaps rows only where a column holds an entry larger in magnitude
// than its diagonal after elimination (IDAMAX, first index on ties).  The leaf
// blocks of a well-resolved surface are strongly diagonal (the 2n x 2n blocks
// of the benchmark molecule have condition numbers near 100 and no row
// interchange at all), so the factorisation runs first without pivot
// searches, as a right-looking blocked LU in 64-column steps:
//   lu_np_diag_kernel   the 64 x 64 diagonal block of every leaf, factored in
//                       shared memory, with the inverses of its L and U
//                       (kept for the panels, and their 32 x 32 diagonal
//                       blocks for the applies);
//   lu_np_panel_kernel  L21 = A21 U11^{-1} by 64-row chunks and
//                       U12 = L11^{-1} A12 by 64-column chunks;
//   lu_gemm2_kernel     A22 -= L21 U12, 64 deep.
// Every multiplier l is checked: |l| <= 1 - 2^-20 for all of them certifies
// that partial pivoting (on these values or on the reference's, which differ
// by rounding only) keeps the diagonal row at every column, so the factors
// are DGETRF's.  A leaf whose certificate fails anywhere (a larger entry, a
// near tie, a zero or non-finite pivot) is re-assembled and factored again by
// the pivoted kernels above.
constexpr int kNP = 64;    // step width
constexpr int kNPT = 256;  // threads of the diagonal and panel kernels
constexpr int kNPPitch = kNP + 1;
constexpr double kNoPivBound = 1.0 - 1.0 / 1048576.0;
constexpr size_t kNPDiagSmem = sizeof(double) * 3 * kNP * kNPPitch;
constexpr size_t kNPPanelSmem = sizeof(double) * 2 * kNP * kNPPitch;

// Per leaf (leaves[blockIdx.x]) with m > k0: D = A[k0:k0+d, k0:k0+d], d =
// min(64, m - k0), factored in place without interchanges (DGETRF2's scaling:
// multipliers times the pivot's reciprocal); scr receives L^{-1} (unit lower,
// column-major) and U^{-1} (row-major) of D, 64 x 64 each with zeros outside
// the triangle and from d on, and dinv the 32 x 32 diagonal blocks of both
// (identity padded, the layout lu_diaginv_kernel writes).  The block, L^{-1}
// and U^{-1} live in registers on a 16 x 16 thread grid; one loop of d
// steps with one barrier each factors the block and forms both inverses
// (the loop's comment gives the scheme).  Every entry of the factors takes
// the same sequence of updates as in a column-by-column DGETF2 order.
// one double into shared memory, asynchronously (zero when !valid)
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 8 : 0));
}

__global__ void __launch_bounds__(kNPT) lu_np_diag_kernel(
    const int* __restrict__ leaves, int k0, const int2* __restrict__ leaf_rng,
    const int64_t* __restrict__ blk_off, const int64_t* __restrict__ dinv_off,
    double* __restrict__ lu, double* __restrict__ dinv, double* __restrict__ scr,
    int* __restrict__ fail) {
  extern __shared__ double nsm[];
  chain_wait();  // the previous launch of the chain has finished
  chain_signal();
  double(*D)[kNPPitch] = reinterpret_cast<double(*)[kNPPitch]>(nsm);
  double(*Li)[kNPPitch] = reinterpret_cast<double(*)[kNPPitch]>(nsm + kNP * kNPPitch);
  double(*Ui)[kNPPitch] = reinterpret_cast<double(*)[kNPPitch]>(nsm + 2 * kNP * kNPPitch);
  const int leaf = leaves[blockIdx.x];
  const int m = 2 * leaf_rng[leaf].y;
  const int d = min(kNP, m - k0);
  double* A = lu + blk_off[leaf];
  const int tid = threadIdx.x;
  for (int e = tid; e < kNP * kNP; e += kNPT) {
    const int c = e >> 6, r = e & 63;
    cp_async8(&D[r][c], A + (size_t)(k0 + min(c, d - 1)) * m + k0 + min(r, d - 1),
              r < d && c < d);
  }
  asm volatile("cp.async.commit_group;\n" ::);
  __shared__ double s_rcp[kNP];  // reciprocal of each pivot
  __shared__ double s_row[2][kNP], s_col[2][kNP], s_xrow[2][kNP], s_zcol[2][kNP];
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  // Thread (tx, ty) of a 16 x 16 grid holds rows ty + 16p and columns
  // tx + 16q (p, q < 4) of the block in registers, and of X = L^{-1} and
  // Z = U^{-1}.  The column loop runs as four rolled loops of 16 (one per
  // band jp), so every register index and every band range is a compile-time
  // constant; a short rolled loop also keeps the code that this
  // once-per-launch kernel fetches small.  Entries of finished rows and
  // columns within a band take a zero multiplier or row entry, which leaves
  // them unchanged, so the updates need no predicates.
  //
  // Step j, one barrier (published vectors double-buffered by parity):
  //  * the factorisation (DGETRF2's scaling): row j and column j, unscaled,
  //    are published; every thread forms its rows' multipliers with the
  //    pivot's reciprocal and updates its entries right of and below the
  //    pivot.  The reciprocal of pivot j + 1 is formed during step j by the
  //    thread that holds that entry, right after its update, and stored for
  //    step j + 1.  A pivot that is zero, subnormal (where DGETRF2 divides
  //    instead) or not finite fails the certificate, and the leaf goes to
  //    the pivoted kernels, which follow DGETRF2 there.
  //  * X by forward row operations, row i -= L[i][j] (row j of X), with row j
  //    final at step j and L[i][j] the step's multiplier;
  //  * Z by column operations, column j times the pivot's reciprocal, then
  //    column c -= U[j][c] (column j of Z), with U[j][c] the step's row.
  // X is lower and Z upper triangular, so step j changes X in rows of bands
  // >= jp and columns of bands <= jp, Z the other way round.
  const int tx = tid & 15, ty = tid >> 4;
  bool bad = false;
  double a[4][4], x[4][4], z[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = ty + 16 * p, c = tx + 16 * q;
      a[p][q] = D[i][c];
      x[p][q] = z[p][q] = (i == c && i < d) ? 1.0 : 0.0;
    }
  auto pivot_rcp = [&](int j, double pk) {  // by the holder of entry (j, j)
    if (!(fabs(pk) >= 2.2250738585072014e-308 && fabs(pk) <= 1.7976931348623157e308)) bad = true;
    s_rcp[j] = 1.0 / pk;
  };
  if (tid == 0) pivot_rcp(0, a[0][0]);
#pragma unroll
  for (int jp = 0; jp < 4; ++jp) {
#pragma unroll 1
    for (int jt = 0; jt < 16; ++jt) {
      const int j = 16 * jp + jt, b = j & 1;
      if (j >= d) break;
      if (ty == jt) {
#pragma unroll
        for (int q = jp; q < 4; ++q) s_row[b][tx + 16 * q] = a[jp][q];
#pragma unroll
        for (int q = 0; q <= jp; ++q) s_xrow[b][tx + 16 * q] = x[jp][q];
      }
      if (tx == jt) {
#pragma unroll
        for (int p = jp; p < 4; ++p) s_col[b][ty + 16 * p] = a[p][jp];
#pragma unroll
        for (int p = 0; p <= jp; ++p) s_zcol[b][ty + 16 * p] = z[p][jp];
      }
      __syncthreads();
      const double rcp = s_rcp[j];
      double l[4], u[4], ux[4], zc[4];
#pragma unroll
      for (int p = jp; p < 4; ++p) {
        const int i = ty + 16 * p;
        l[p] = i > j ? s_col[b][i] * rcp : 0.0;
      }
#pragma unroll
      for (int q = jp; q < 4; ++q) {
        const int c = tx + 16 * q;
        u[q] = c > j ? s_row[b][c] : 0.0;
      }
#pragma unroll
      for (int q = 0; q <= jp; ++q) ux[q] = s_xrow[b][tx + 16 * q];
#pragma unroll
      for (int p = 0; p <= jp; ++p) zc[p] = s_zcol[b][ty + 16 * p] * rcp;
      if (tx == jt) {  // the holders of column j: its multipliers, column j of Z scaled
#pragma unroll
        for (int p = jp; p < 4; ++p)
          if (ty + 16 * p > j) {
            if (!(fabs(l[p]) <= kNoPivBound)) bad = true;
            a[p][jp] = l[p];
          }
#pragma unroll
        for (int p = 0; p <= jp; ++p) z[p][jp] = zc[p];
      }
#pragma unroll
      for (int p = jp; p < 4; ++p)
#pragma unroll
        for (int q = jp; q < 4; ++q) a[p][q] = fma(-l[p], u[q], a[p][q]);
      // the next pivot's reciprocal, by its holder
      if (tx == ty && tx == ((j + 1) & 15) && j + 1 < d) {
        if (jt < 15)
          pivot_rcp(j + 1, a[jp][jp]);
        else if (jp < 3)
          pivot_rcp(j + 1, a[jp < 3 ? jp + 1 : 3][jp < 3 ? jp + 1 : 3]);
      }
#pragma unroll
      for (int p = jp; p < 4; ++p)
#pragma unroll
        for (int q = 0; q <= jp; ++q) x[p][q] = fma(-l[p], ux[q], x[p][q]);
#pragma unroll
      for (int p = 0; p <= jp; ++p)
#pragma unroll
        for (int q = jp; q < 4; ++q) z[p][q] = fma(-zc[p], u[q], z[p][q]);
    }
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = ty + 16 * p, c = tx + 16 * q;
      D[i][c] = a[p][q];
      Li[i][c] = x[p][q];
      Ui[i][c] = z[p][q];
    }
  __syncthreads();
  // factors back
  for (int e = tid; e < d * d; e += kNPT) {
    const int c = e / d, r = e - c * d;
    A[(size_t)(k0 + c) * m + k0 + r] = D[r][c];
  }
  if (__syncthreads_or(bad) && tid == 0) fail[leaf] = 1;
  double* S = scr + (size_t)blockIdx.x * 2 * kNP * kNP;
  for (int e = tid; e < kNP * kNP; e += kNPT) {
    const int hi = e / kNP, lo = e - hi * kNP;
    S[e] = Li[lo][hi];            // column-major L^{-1}
    S[kNP * kNP + e] = Ui[hi][lo];  // row-major U^{-1}
  }
  double* Di = dinv + dinv_off[leaf] + (size_t)(k0 / kDB) * 2 * kDB * kDB;
  for (int b = 0; b * kDB < d; ++b) {
    const int nb = min(kDB, d - b * kDB), o = b * kDB;
    double* Lb = Di + (size_t)b * 2 * kDB * kDB;
    double* Ub = Lb + kDB * kDB;
    for (int e = tid; e < kDB * kDB; e += kNPT) {
      const int c = e / kDB, r = e - c * kDB;
      const double id = r == c ? 1.0 : 0.0;
      Lb[e] = (r < nb && c < nb) ? Li[o + r][o + c] : id;
      Ub[e] = (r < nb && c < nb) ? Ui[o + r][o + c] : id;
    }
  }
}

// item = (leaf, slot, kind, off): kind 0, rows [off, off + 64) of the step's
// column panel: L21 = A21 U11^{-1}, each multiplier checked; kind 1, columns
// [off, off + 64) of its row panel: U12 = L11^{-1} A12.  slot = the leaf's
// row in the diagonal kernel's launch (its scratch).  A 64 x 64 x 64 product
// out = P Q from shared memory, 4 x 4 outputs per thread (rows tr + 16 a,
// columns tc + 16 b: P loads on 16 consecutive rows, Q loads broadcast).
__global__ void __launch_bounds__(kNPT) lu_np_panel_kernel(
    const int4* __restrict__ items, int k0, const int2* __restrict__ leaf_rng,
    const int64_t* __restrict__ blk_off, double* __restrict__ lu,
    const double* __restrict__ scr, int* __restrict__ fail) {
  extern __shared__ double nsm[];
  chain_wait();  // the previous launch of the chain has finished
  chain_signal();
  double(*X)[kNPPitch] = reinterpret_cast<double(*)[kNPPitch]>(nsm);
  double(*V)[kNPPitch] = reinterpret_cast<double(*)[kNPPitch]>(nsm + kNP * kNPPitch);
  const int4 it = items[blockIdx.x];
  const int leaf = it.x, kind = it.z, off = it.w;
  const int m = 2 * leaf_rng[leaf].y;
  const int d = min(kNP, m - k0);
  const int cnt = min(kNP, m - off);
  double* A = lu + blk_off[leaf];
  const double* S = scr + (size_t)it.y * 2 * kNP * kNP + (kind == 0 ? kNP * kNP : 0);
  const int tid = threadIdx.x, tr = tid & 15, tc = tid >> 4;
  // V = the inverse as [row][col]: U^{-1} (row-major in scr) for kind 0,
  // L^{-1} (column-major in scr) for kind 1; zeros outside d x d
  for (int e = tid; e < kNP * kNP; e += kNPT) {
    const int hi = e >> 6, lo = e & 63;
    cp_async8(kind == 0 ? &V[hi][lo] : &V[lo][hi], S + e, true);
  }
  if (kind == 0) {  // X[i][q] = A[off + i, k0 + q]
    for (int e = tid; e < kNP * kNP; e += kNPT) {
      const int q = e >> 6, i = e & 63;
      const bool ok = i < cnt && q < d;
      cp_async8(&X[i][q], ok ? A + (size_t)(k0 + q) * m + off + i : A, ok);
    }
  } else {          // X[q][c] = A[k0 + q, off + c]
    for (int e = tid; e < kNP * kNP; e += kNPT) {
      const int c = e >> 6, q = e & 63;
      const bool ok = c < cnt && q < d;
      cp_async8(&X[q][c], ok ? A + (size_t)(off + c) * m + k0 + q : A, ok);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  // kind 0: out = X V (P = X, Q = V); kind 1: out = V X (P = V, Q = X)
  const double(*P)[kNPPitch] = kind == 0 ? X : V;
  const double(*Q)[kNPPitch] = kind == 0 ? V : X;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
#pragma unroll 4
  for (int q = 0; q < d; ++q) {
    double pv[4], qv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) pv[a] = P[tr + 16 * a][q];
#pragma unroll
    for (int b = 0; b < 4; ++b) qv[b] = Q[q][tc + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(pv[a], qv[b], acc[a][b]);
  }
  bool bad = false;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = tr + 16 * a, c = tc + 16 * b;
      if (kind == 0) {
        if (r < cnt && c < d) {
          if (!(fabs(acc[a][b]) <= kNoPivBound)) bad = true;
          A[(size_t)(k0 + c) * m + off + r] = acc[a][b];
        }
      } else if (c < cnt && r < d) {
        A[(size_t)(off + c) * m + k0 + r] = acc[a][b];
      }
    }
  if (__syncthreads_or(bad) && tid == 0) fail[leaf] = 1;
}

// Updates of the unpivoted factorisation: item = (leaf, r0, c0, ends):
// C = A[r0:r0+128, c0:c0+64] -= A[r0:, k0:k0+kd] A[k0:k0+kd, c0:] with
// kd = min(kdepth, m - k0) (64 inside an outer block of kOB2 columns, kOB2
// for the trailing matrix right of it), rows clipped at re and columns at ce,
// packed as ends = (re << 16) | ce (0: both m).  256 threads, 8 x 4
// outputs each: rows 2 tr + 32 a + {0, 1} (a = 0..3; each pair one 16-byte
// shared load, eight lanes of a load phase on 32 distinct banks) and columns
// 4 tc .. 4 tc + 3 (two 16-byte loads, broadcast within a phase).  C is loaded
// into the accumulators and the products subtracted one k at a time
// (fma(-l, u, c)), the order of the reference's DGEMM (C := C - A B,
// dgetrf_dep.f), while the 32-deep slices of L (k-major) and U (by column,
// pitch 34: conflict-free 16-byte stores, broadcast loads) arrive by cp.async
// (zero-filled outside the tile: m, r0, c0, k0 and the depth are even, so a
// 16-byte chunk is wholly inside or outside).
constexpr int kG2M = 128, kG2N = 64, kG2K = 32;
constexpr int kG2UP = kG2K + 2;  // U slice by column: pitch of 34 doubles
constexpr int kOB2 = 256;  // outer block of the unpivoted factorisation
constexpr size_t kGemm2Smem = sizeof(double) * 2 * (kG2K * kG2M + kG2N * kG2UP);

__global__ void __launch_bounds__(256, 2) lu_gemm2_kernel(const int4* __restrict__ items, int k0,
                                                          int kdepth,
                                                          const int2* __restrict__ leaf_rng,
                                                          const int64_t* __restrict__ blk_off,
                                                          double* __restrict__ lu) {
  extern __shared__ double gsm2[];
  chain_wait();  // the previous launch of the chain has finished
  chain_signal();
  double* sL = gsm2;                      // [2][kG2K][kG2M]  L slice, k-major
  double* sU = gsm2 + 2 * kG2K * kG2M;    // [2][kG2N][kG2UP] U slice, by column
  const int4 it = items[blockIdx.x];
  const int leaf = it.x, r0 = it.y, c0 = it.z;
  const int m = 2 * leaf_rng[leaf].y;
  const int re = it.w ? min(m, it.w >> 16) : m, ce = it.w ? min(m, it.w & 0xffff) : m;
  const int kd = min(kdepth, m - k0);
  double* A = lu + blk_off[leaf];
  const int tid = threadIdx.x;
  const int tr = tid & 15, tc = tid >> 4;
  auto row_of = [&](int a) { return 2 * tr + 32 * (a >> 1) + (a & 1); };
  auto load_slice = [&](int kc, int buf) {
    const int nbk = min(kG2K, kd - kc), kb = k0 + kc;
    double* L = sL + buf * kG2K * kG2M;
    double* U = sU + buf * kG2N * kG2UP;
#pragma unroll
    for (int e = 0; e < (kG2K * kG2M / 2) / 256; ++e) {
      const int q = tid + 256 * e;
      const int k = q / (kG2M / 2), rr = 2 * (q % (kG2M / 2));
      const bool ok = k < nbk && r0 + rr < re;
      cp_async16(L + k * kG2M + rr, ok ? A + (size_t)(kb + k) * m + r0 + rr : A, ok);
    }
    // U by column (the source's own layout): 16-byte chunks of 2 k
#pragma unroll
    for (int e = 0; e < (kG2K * kG2N / 2) / 256; ++e) {
      const int q = tid + 256 * e;
      const int c = q / (kG2K / 2), kk = 2 * (q % (kG2K / 2));
      const bool ok = kk < nbk && c0 + c < ce;
      cp_async16(U + c * kG2UP + kk, ok ? A + (size_t)(c0 + c) * m + kb + kk : A, ok);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  load_slice(0, 0);
  if (kG2K < kd) load_slice(kG2K, 1);
  // C by row pairs: 16 lanes read 256 contiguous bytes of a column (rows and
  // m are even, so a pair is wholly inside or outside)
  double acc[8][4];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = c0 + 4 * tc + b;
    const double* cc = A + (size_t)min(c, m - 1) * m;
#pragma unroll
    for (int a = 0; a < 8; a += 2) {
      const int r = r0 + row_of(a);
      const double2 v = (c < ce && r < re) ? *reinterpret_cast<const double2*>(cc + r)
                                           : make_double2(0.0, 0.0);
      acc[a][b] = v.x;
      acc[a + 1][b] = v.y;
    }
  }
  for (int kc = 0, buf = 0; kc < kd; kc += kG2K, buf ^= 1) {
    if (kc + kG2K < kd) {
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
    // all 32 k of the slice (zero-filled past the depth: fma(-0, 0, c) = c),
    // the next k's operands loaded while this k's products run
    const double* L = sL + buf * kG2K * kG2M + 2 * tr;
    const double* U = sU + buf * kG2N * kG2UP + 4 * tc * kG2UP;
    double2 lc[4];
    double uc[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) lc[a] = *reinterpret_cast<const double2*>(L + 32 * a);
#pragma unroll
    for (int b = 0; b < 4; ++b) uc[b] = U[b * kG2UP];
#pragma unroll
    for (int k = 0; k < kG2K; ++k) {
      double2 ln[4];
      double un[4];
      if (k + 1 < kG2K) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
          ln[a] = *reinterpret_cast<const double2*>(L + (k + 1) * kG2M + 32 * a);
#pragma unroll
        for (int b = 0; b < 4; ++b) un[b] = U[b * kG2UP + k + 1];
      }
      const double lv[8] = {lc[0].x, lc[0].y, lc[1].x, lc[1].y,
                            lc[2].x, lc[2].y, lc[3].x, lc[3].y};
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(-lv[a], uc[b], acc[a][b]);
      if (k + 1 < kG2K) {
#pragma unroll
        for (int a = 0; a < 4; ++a) lc[a] = ln[a];
#pragma unroll
        for (int b = 0; b < 4; ++b) uc[b] = un[b];
      }
    }
    if (kc + 2 * kG2K < kd) {  // buffer buf takes the slice two on
      __syncthreads();
      load_slice(kc + 2 * kG2K, buf);
    }
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int c = c0 + 4 * tc + b;
    if (c >= ce) continue;
    double* cc = A + (size_t)c * m;
#pragma unroll
    for (int a = 0; a < 8; a += 2) {
      const int r = r0 + row_of(a);
      if (r < re) *reinterpret_cast<double2*>(cc + r) = make_double2(acc[a][b], acc[a + 1][b]);
    }
  }
}

// every leaf: no interchange (1-based local pivots i + 1) and the identity
// row permutation of the applies
__global__ void lu_np_identity_kernel(const int2* __restrict__ leaf_rng, int* __restrict__ piv,
                                      int* __restrict__ perm) {
  const int2 lr = leaf_rng[blockIdx.x];
  const int m = 2 * lr.y;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    piv[2 * lr.x + i] = i + 1;
    perm[2 * lr.x + i] = i;
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
  PinVec<int2>& tiles = H.pc_h_tiles;
  tiles.restart();
  for (int l = 0; l < nl; ++l) {
    int c = T.leaves[l];
    rng[l] = make_int2(T.ibeg[c], T.num[c]);
    T.blk_off[l] = off;
    off += 4LL * T.num[c] * T.num[c];
    for (int j = 0; j < T.num[c]; j += kAsmCols) tiles.push(make_int2(l, j));
  }
  T.d_lu.alloc(std::max<int64_t>(off, 1));
  T.d_piv.alloc(2 * (size_t)H.n);
  T.d_blk_off.alloc(nl);
  T.d_leaf_rng.alloc(nl);
  DBuf<int2>& d_tiles = H.pc_tiles;
  d_tiles.alloc(tiles.len);
  DBuf<int>& d_info = H.pc_info;
  d_info.alloc(nl);
  H.pc_h_blk_off.assign(T.blk_off.data(), nl);
  H.pc_h_blk_off.upload(T.d_blk_off, s);
  H.pc_h_rng.assign(rng.data(), nl);
  H.pc_h_rng.upload(T.d_leaf_rng, s);
  tiles.upload(d_tiles, s);
  double eps = H.prm.eps1 / H.prm.eps0;
  { TABI_K(K_ASSEMBLE, s); assemble_kernel<<<(int)tiles.len, 256, 0, s>>>(d_tiles.p, T.d_leaf_rng.p, T.d_blk_off.p,
                                                    H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p,
                                                    H.d_ny.p, H.d_nz.p, H.d_area.p,
                                                    H.prm.kappa, eps, T.d_lu.p); }
  TABI_CUDA(cudaMemsetAsync(d_info.p, 0, sizeof(int) * nl, s));
  // apply lists (they depend on the leaf sizes only, so they are built while
  // the assembly runs): blocks of order > 512 get 512 threads (one wave on the GPU),
  // the others 256 threads on the side stream; largest first in each
  {
    std::vector<int> big, small;
    for (int l = 0; l < nl; ++l) (2 * rng[l].y > 512 ? big : small).push_back(l);
    std::sort(big.begin(), big.end(), [&](int a, int b) { return rng[a].y > rng[b].y; });
    std::sort(small.begin(), small.end(), [&](int a, int b) { return rng[a].y > rng[b].y; });
    T.n_solve_big = (int)big.size();
    T.n_solve_small = (int)small.size();
    big.insert(big.end(), small.begin(), small.end());
    H.pc_h_solve_list.assign(big.data(), big.size());
    H.pc_h_solve_list.upload(T.d_solve_list, s);
  }
  // ---- unpivoted factorisation of every leaf, certified (see lu_np_diag_kernel)
  H.pc_lu_phase.emplace(H.prof, K_PHASE_LU, s);
  const bool try_np = (H.prm.flags & TABI_FLAG_PIVOTED_LU) == 0;
  if (try_np) {
    DBuf<int>& d_fail = H.pc_fail;
    d_fail.alloc(nl);
    TABI_CUDA(cudaMemsetAsync(d_fail.p, 0, sizeof(int) * nl, s));
    T.d_lu_perm.alloc(2 * (size_t)H.n);
    { TABI_K(K_LU_POST, s); lu_np_identity_kernel<<<nl, 256, 0, s>>>(T.d_leaf_rng.p, T.d_piv.p, T.d_lu_perm.p); }
    // the inverse diagonal blocks are written by the diagonal kernel
    T.dinv_off.resize(nl);
    int64_t doff = 0;
    for (int l = 0; l < nl; ++l) {
      T.dinv_off[l] = doff;
      doff += (int64_t)ceil_div(2 * rng[l].y, kDB) * 2 * kDB * kDB;
    }
    T.d_dinv.alloc(std::max<int64_t>(doff, 1));
    T.d_dinv_off.alloc(nl);
    H.pc_h_dinv_off.assign(T.dinv_off.data(), nl);
    H.pc_h_dinv_off.upload(T.d_dinv_off, s);
    raise_smem_limit((const void*)lu_np_diag_kernel, kNPDiagSmem);
    raise_smem_limit((const void*)lu_np_panel_kernel, kNPPanelSmem);
    raise_smem_limit((const void*)lu_gemm2_kernel, kGemm2Smem);
    std::vector<int> grp[2];
    for (int l = 0; l < nl; ++l) grp[2 * rng[l].y > kLuSmallBlock ? 0 : 1].push_back(l);
    for (auto& g : grp)
      std::sort(g.begin(), g.end(), [&](int a, int b) { return rng[a].y > rng[b].y; });
    // both groups on the handle's high-priority LU streams, forked from s
    TABI_CUDA(cudaEventRecord(H.ev_fork, s));
    TABI_CUDA(cudaStreamWaitEvent(H.lu_hi, H.ev_fork, 0));
    TABI_CUDA(cudaStreamWaitEvent(H.lu_small, H.ev_fork, 0));
    // Two-level right-looking order (outer blocks of kOB2 columns, inner steps
    // of 64).  Inside an outer block: the diagonal block of each inner step,
    // its L21 for every row below and its U12 for the block's own columns, and
    // the update of the block's own columns.  Then the columns right of the
    // block: U12 = L11^{-1} A12 in four 64-row sub-steps (each applies the
    // inner step's L^{-1}, then updates the block's rows below it), and the
    // trailing matrix takes one kOB2-deep update.
    //
    // Look-ahead (the large-block group): the trailing update of an outer
    // block is split by columns.  The next outer block's kOB2 columns, which
    // its steps factor, are updated on the group's stream; the columns beyond
    // it on the low-priority auxiliary stream, beside the next
    // block's diagonal, panel and update launches, which touch only rows and
    // columns of that block or its own columns below it.  The next block's
    // columns right of it (rows of the block, columns beyond) wait for the
    // auxiliary stream.  Every entry is updated by the same tile in the same
    // k order as without the split, so the factors are the same bit for bit.
    struct Launch {
      // 0 diagonal, 1 panel, 2 update, 3 fork to the auxiliary stream,
      // 4 wait for the auxiliary stream, 5 update on the auxiliary stream
      int kind;
      int k0, depth, off, cnt, scr_slot0;
    };
    // one group's plan: item lists (uploaded on st) and its launches
    auto plan_np = [&](const std::vector<int>& order, Handle::NpPlan& B, cudaStream_t st,
                       bool la) {
      int gmax = 0;
      for (int l : order) gmax = std::max(gmax, 2 * rng[l].y);
      std::vector<Launch> plan;
      PinVec<int>& dl = B.h_dleaves;
      PinVec<int4>& pit = B.h_pitems;
      PinVec<int4>& git = B.h_gitems;
      dl.restart();
      pit.restart();
      git.restart();
      const auto pack = [](int re, int ce) { return (re << 16) | ce; };
      int max_slots = 1;
      auto emit = [&](int kind, int k0, int depth, size_t before, size_t after, int slot0) {
        if (after > before)
          plan.push_back({kind, k0, depth, (int)before, (int)(after - before), slot0});
      };
      bool rest_pending = false;  // an update on the auxiliary stream not yet waited for
      for (int K0 = 0; K0 < gmax; K0 += kOB2) {
        int nact = 0;
        for (int l : order) nact += 2 * rng[l].y > K0;
        max_slots = std::max(max_slots, nact);
        // the leaves' rows in this outer block's diagonal launches: slot index
        // = inner step * nact + position
        for (int k0 = K0; k0 < std::min(gmax, K0 + kOB2); k0 += kNP) {
          const int j = (k0 - K0) / kNP;
          size_t d0 = dl.len, p0 = pit.len, g0 = git.len;
          int slot = 0;
          for (int l : order) {
            const int m = 2 * rng[l].y;
            if (m <= k0) continue;
            dl.push(l);
            const int d = std::min(kNP, m - k0), ce = std::min(m, K0 + kOB2);
            for (int off = k0 + d; off < m; off += kNP)
              pit.push(make_int4(l, j * nact + slot, 0, off));
            for (int off = k0 + d; off < ce; off += kNP)
              pit.push(make_int4(l, j * nact + slot, 1, off));
            for (int r0 = k0 + d; r0 < m; r0 += kG2M)
              for (int c0 = k0 + d; c0 < ce; c0 += kG2N)
                git.push(make_int4(l, r0, c0, pack(m, ce)));
            ++slot;
          }
          emit(0, k0, 0, d0, dl.len, j * nact);
          emit(1, k0, 0, p0, pit.len, 0);
          emit(2, k0, kNP, g0, git.len, 0);
        }
        // the columns right of the block (leaves with m > K0 + kOB2 have all
        // four inner steps; their slot in inner step j is j * nact + the
        // leaf's position among the active leaves)
        const int Kend = K0 + kOB2;
        if (rest_pending) {
          plan.push_back({4, K0, 0, 0, 0, 0});
          rest_pending = false;
        }
        for (int j = 0; j < kOB2 / kNP; ++j) {
          const int k0 = K0 + j * kNP;
          size_t p0 = pit.len, g0 = git.len;
          int pos = 0;
          for (int l : order) {
            const int m = 2 * rng[l].y;
            if (m <= K0) continue;
            if (m > Kend) {
              for (int off = Kend; off < m; off += kNP)
                pit.push(make_int4(l, j * nact + pos, 1, off));
              for (int r0 = k0 + kNP; r0 < Kend; r0 += kG2M)
                for (int c0 = Kend; c0 < m; c0 += kG2N)
                  git.push(make_int4(l, r0, c0, pack(Kend, m)));
            }
            ++pos;
          }
          emit(1, k0, 0, p0, pit.len, 0);
          emit(2, k0, kNP, g0, git.len, 0);
        }
        // the trailing update: columns [Kend, Knext) here, the rest on the
        // auxiliary stream (all of it here without look-ahead)
        const int Knext = la ? Kend + kOB2 : INT_MAX;
        size_t g0 = git.len;
        for (int l : order) {
          const int m = 2 * rng[l].y;
          if (m <= Kend) continue;
          for (int r0 = Kend; r0 < m; r0 += kG2M)
            for (int c0 = Kend; c0 < std::min(m, Knext); c0 += kG2N)
              git.push(make_int4(l, r0, c0, 0));
        }
        const size_t g1 = git.len;
        for (int l : order) {
          const int m = 2 * rng[l].y;
          if (m <= Knext) continue;
          for (int r0 = Kend; r0 < m; r0 += kG2M)
            for (int c0 = Knext; c0 < m; c0 += kG2N) git.push(make_int4(l, r0, c0, 0));
        }
        // the fork before the look-ahead columns' launch (the auxiliary stream
        // must not wait for it), the rest launched after it (earlier launches
        // are dispatched first)
        const bool rest = git.len > g1;
        if (rest) plan.push_back({3, K0, 0, 0, 0, 0});
        emit(2, K0, kOB2, g0, g1, 0);
        if (rest) {
          emit(5, K0, kOB2, g1, git.len, 0);
          rest_pending = true;
        }
      }
      if (rest_pending) plan.push_back({4, gmax, 0, 0, 0, 0});
      dl.upload(B.dleaves, st);
      pit.upload(B.pitems, st);
      git.upload(B.gitems, st);
      B.scr.alloc((size_t)max_slots * (kOB2 / kNP) * 2 * kNP * kNP);
      return plan;
    };
    // Issues launch `at` of a group's plan.  Kernels follow kernels on the
    // group's stream as a programmatic chain; the first one after the uploads
    // or a cross-stream event starts the ordinary way.
    struct Issuer {
      std::vector<Launch> plan;
      Handle::NpPlan* B;
      cudaStream_t st;
      size_t at = 0;
      bool chain = false;
    };
    auto issue_one = [&](Issuer& is) {
      const Launch& q = is.plan[is.at++];
      Handle::NpPlan& B = *is.B;
      cudaStream_t st = is.st;
      bool& chain = is.chain;
      {
        if (q.kind == 0) {
          TABI_K(K_LU, st);
          launch_chained(chain, lu_np_diag_kernel, dim3(q.cnt), dim3(kNPT), kNPDiagSmem, st,
                         B.dleaves.p + q.off, q.k0, T.d_leaf_rng.p, T.d_blk_off.p,
                         T.d_dinv_off.p, T.d_lu.p, T.d_dinv.p,
                         B.scr.p + (size_t)q.scr_slot0 * 2 * kNP * kNP, d_fail.p);
          chain = true;
        } else if (q.kind == 1) {
          TABI_K(K_LU_STRIP, st);
          launch_chained(chain, lu_np_panel_kernel, dim3(q.cnt), dim3(kNPT), kNPPanelSmem, st,
                         B.pitems.p + q.off, q.k0, T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p,
                         B.scr.p, d_fail.p);
          chain = true;
        } else if (q.kind == 3) {
          TABI_CUDA(cudaEventRecord(H.ev_la, st));
          TABI_CUDA(cudaStreamWaitEvent(H.aux, H.ev_la, 0));
          chain = false;
        } else if (q.kind == 4) {
          TABI_CUDA(cudaStreamWaitEvent(st, H.ev_rest, 0));
          chain = false;
        } else {
          cudaStream_t gs = q.kind == 5 ? H.aux : st;
          TABI_K(K_LU_UPDATE, gs);
          launch_chained(chain && q.kind == 2, lu_gemm2_kernel, dim3(q.cnt), dim3(256),
                         kGemm2Smem, gs,
                         B.gitems.p + q.off, q.k0, q.depth, T.d_leaf_rng.p, T.d_blk_off.p,
                         T.d_lu.p);
          if (q.kind == 5) TABI_CUDA(cudaEventRecord(H.ev_rest, H.aux));
          else chain = true;
        }
      }
    };
    // both plans first, then their launches interleaved, so that both chains
    // start at once (the host issues far faster than the GPU runs them)
    Issuer big{}, small{};
    big.B = &H.pc_np[0];
    big.st = H.lu_hi;
    small.B = &H.pc_np[1];
    small.st = H.lu_small;
    if (!grp[0].empty()) big.plan = plan_np(grp[0], H.pc_np[0], H.lu_hi, true);
    if (!grp[1].empty()) small.plan = plan_np(grp[1], H.pc_np[1], H.lu_small, false);
    while (big.at < big.plan.size() || small.at < small.plan.size()) {
      if (big.at < big.plan.size()) issue_one(big);
      if (small.at < small.plan.size()) issue_one(small);
    }
  }
}

void finish_precond(Handle& H, cudaStream_t s) {
  if (H.prm.iprcd != 1 || H.has_precond) return;
  Tree& T = H.tree;
  const int nl = T.nleaf;
  std::vector<int2> rng(nl);
  for (int l = 0; l < nl; ++l) {
    const int c = T.leaves[l];
    rng[l] = make_int2(T.ibeg[c], T.num[c]);
  }
  const double eps = H.prm.eps1 / H.prm.eps0;
  DBuf<int>& d_info = H.pc_info;
  const bool try_np = (H.prm.flags & TABI_FLAG_PIVOTED_LU) == 0;
  // Two leaf groups with plans of their own: blocks of order above
  // kLuSmallBlock and the others, so the many short factorisations of small
  // leaves run beside the long chain of steps of the large ones instead of
  // inside its launches.  The unpivoted factorisation runs them on the
  // handle's LU streams (see below); the pivoted one on the caller's stream
  // and the side stream, with one fork after the assembly and one join at
  // the end (fork / join).
  auto fork = [&](bool split) {
    if (!split) return;
    TABI_CUDA(cudaEventRecord(H.ev_fork, s));
    TABI_CUDA(cudaStreamWaitEvent(H.side, H.ev_fork, 0));
  };
  auto join = [&](bool split) {
    if (!split) return;
    TABI_CUDA(cudaEventRecord(H.ev_join, H.side));
    TABI_CUDA(cudaStreamWaitEvent(s, H.ev_join, 0));
  };
  std::vector<int> pv_leaves;  // leaves factored with partial pivoting
  if (try_np) {
    DBuf<int>& d_fail = H.pc_fail;
    TABI_CUDA(cudaEventRecord(H.ev_join, H.lu_small));
    TABI_CUDA(cudaStreamWaitEvent(s, H.ev_join, 0));
    TABI_CUDA(cudaEventRecord(H.ev_lu_join, H.lu_hi));
    TABI_CUDA(cudaStreamWaitEvent(s, H.ev_lu_join, 0));
    std::vector<int> failed(nl);
    TABI_CUDA(cudaMemcpyAsync(failed.data(), d_fail.p, sizeof(int) * nl, cudaMemcpyDeviceToHost,
                              s));
    TABI_CUDA(cudaStreamSynchronize(s));
    for (int l = 0; l < nl; ++l)
      if (failed[l]) pv_leaves.push_back(l);
    if (!pv_leaves.empty()) {
      // those blocks again from their kernel values
      std::vector<int2> ptiles;
      for (int l : pv_leaves)
        for (int j = 0; j < rng[l].y; j += kAsmCols) ptiles.push_back(make_int2(l, j));
      H.pc_tiles2.alloc(ptiles.size());
      TABI_CUDA(cudaMemcpyAsync(H.pc_tiles2.p, ptiles.data(), sizeof(int2) * ptiles.size(),
                                cudaMemcpyHostToDevice, s));
      TABI_K(K_ASSEMBLE, s);
      assemble_kernel<<<(int)ptiles.size(), 256, 0, s>>>(H.pc_tiles2.p, T.d_leaf_rng.p,
                                                         T.d_blk_off.p, H.d_x.p, H.d_y.p,
                                                         H.d_z.p, H.d_nx.p, H.d_ny.p, H.d_nz.p,
                                                         H.d_area.p, H.prm.kappa, eps, T.d_lu.p);
    }
  } else {
    for (int l = 0; l < nl; ++l) pv_leaves.push_back(l);
  }
  H.pc_pv_leaves = (int)pv_leaves.size();
  if (!pv_leaves.empty()) {
    // batched LU for blocks with m <= kPanelMaxM; the global-memory kernel for
    // larger ones
    int mmax = 0;
    bool any_big = false;
    std::vector<int> big_leaves;
    for (int l : pv_leaves) {
      int m = 2 * rng[l].y;
      if (m <= kPanelMaxM) mmax = std::max(mmax, m);
      else {
        any_big = true;
        big_leaves.push_back(l);
      }
    }
    if (mmax > 0) {
      size_t smem = sizeof(double) * (size_t)mmax * kSP;
      raise_smem_limit((const void*)lu_panel_kernel, std::max<size_t>(smem, 48 * 1024));
    }
    raise_smem_limit((const void*)lu_gemm_kernel, kGemmSmem);
    // Two leaf groups with plans of their own: blocks of order above
    // kLuSmallBlock on the handle's stream, the others on its side stream, so
    // the many short factorisations of small leaves run beside the long
    // panel chain of the large ones instead of inside its launches; one fork
    // after the assembly, one join at the end.
    std::vector<int> grp[2];
    for (int l : pv_leaves) {
      const int m = 2 * rng[l].y;
      if (m <= kPanelMaxM) grp[m > kLuSmallBlock ? 0 : 1].push_back(l);
    }
    for (auto& g : grp)
      std::sort(g.begin(), g.end(), [&](int a, int b) { return rng[a].y > rng[b].y; });
    const bool split = H.side != nullptr && !grp[0].empty() && !grp[1].empty();
    fork(split);
    // Two-level right-looking LU (LAPACK DGETRF order) of one group.  Outer
    // blocks of kOB columns; inside one, 32-column panel steps update only
    // the block's own columns (and swap the columns left of the panel).  After
    // the block its kOB row interchanges are applied at once to the columns
    // right of it, U12 follows by 32-row TRSM + small GEMM steps, and the
    // trailing matrix gets one kOB-deep update.
    auto run_group = [&](const std::vector<int>& order, Handle::LuPlan& B, cudaStream_t st) {
      int gmax = 0;
      for (int l : order) gmax = std::max(gmax, 2 * rng[l].y);
      struct Launch {
        int kind;  // 0 panel, 1 strip, 2 gemm, 3 swap map, 4 row swap
        int k0, kdepth, off, cnt;
      };
      std::vector<Launch> plan;
      std::vector<int> pitems, mleaves;
      std::vector<int4> sitems, gitems, ritems;
      auto emit = [&](int kind, int k0, int kdepth, size_t before, size_t after) {
        if (after > before) plan.push_back({kind, k0, kdepth, (int)before, (int)(after - before)});
      };
      const auto pack = [](int re, int ce) { return (re << 16) | ce; };
      for (int K0 = 0; K0 < gmax; K0 += kOB) {
        for (int k0 = K0; k0 < std::min(gmax, K0 + kOB); k0 += kBP) {
          size_t p0 = pitems.size(), s0 = sitems.size(), g0 = gitems.size();
          for (int l : order) {
            const int m = 2 * rng[l].y;
            if (m <= k0) continue;
            pitems.push_back(l);
            const int nb = std::min(kBP, m - k0), ce = std::min(m, K0 + kOB);
            // left of the panel inside the outer block (the columns left of
            // the block get the block's swaps at its end)
            for (int c0 = K0; c0 < k0; c0 += kUC)
              sitems.push_back(make_int4(l, c0, std::min(c0 + kUC, k0), 0));
            for (int c0 = k0 + nb; c0 < ce; c0 += kUC)
              sitems.push_back(make_int4(l, c0, std::min(c0 + kUC, ce), 1));
            for (int r0 = k0 + nb; r0 < m; r0 += kGT)
              for (int c0 = k0 + nb; c0 < ce; c0 += kGT)
                gitems.push_back(make_int4(l, r0, c0, pack(m, ce)));
          }
          emit(0, k0, 0, p0, pitems.size());
          emit(1, k0, 0, s0, sitems.size());
          emit(2, k0, kBP, g0, gitems.size());
        }
        // the block's row interchanges on the columns left of it and right of it
        const int Kend = K0 + kOB;
        size_t m0 = mleaves.size(), r0i = ritems.size();
        for (int l : order) {
          const int m = 2 * rng[l].y;
          if (m <= K0 || (K0 == 0 && m <= Kend)) continue;
          const int slot = (int)(mleaves.size() - m0);
          mleaves.push_back(l);
          for (int c0 = 0; c0 < K0; c0 += kUC)
            ritems.push_back(make_int4(slot, c0, std::min(c0 + kUC, K0), l));
          for (int c0 = Kend; c0 < m; c0 += kUC)
            ritems.push_back(make_int4(slot, c0, std::min(c0 + kUC, m), l));
        }
        emit(3, K0, 0, m0, mleaves.size());
        emit(4, K0, 0, r0i, ritems.size());
        for (int kb = K0; kb < Kend; kb += kBP) {
          size_t s0 = sitems.size(), g0 = gitems.size();
          for (int l : order) {
            const int m = 2 * rng[l].y;
            if (m <= Kend) continue;
            for (int c0 = Kend; c0 < m; c0 += kUC)
              sitems.push_back(make_int4(l, c0, std::min(c0 + kUC, m), 3));
            for (int rr = kb + kBP; rr < Kend; rr += kGT)
              for (int c0 = Kend; c0 < m; c0 += kGT)
                gitems.push_back(make_int4(l, rr, c0, pack(Kend, m)));
          }
          emit(1, kb, 0, s0, sitems.size());
          emit(2, kb, kBP, g0, gitems.size());
        }
        size_t g0 = gitems.size();
        for (int l : order) {
          const int m = 2 * rng[l].y;
          if (m <= Kend) continue;
          for (int rr = Kend; rr < m; rr += kGT)
            for (int c0 = Kend; c0 < m; c0 += kGT) gitems.push_back(make_int4(l, rr, c0, 0));
        }
        emit(2, K0, kOB, g0, gitems.size());
      }
      auto up = [&](auto& buf, const auto& v) {
        buf.alloc(std::max<size_t>(v.size(), 1));
        if (!v.empty())
          TABI_CUDA(cudaMemcpyAsync(buf.p, v.data(), sizeof(v[0]) * v.size(),
                                    cudaMemcpyHostToDevice, st));
      };
      up(B.list, pitems);
      up(B.items, sitems);
      up(B.gitems, gitems);
      up(B.mleaves, mleaves);
      up(B.ritems, ritems);
      size_t maxm = 1;
      for (const Launch& L : plan)
        if (L.kind == 3) maxm = std::max<size_t>(maxm, (size_t)L.cnt);
      B.map.alloc(maxm * (4 * kOB + 1));
      for (const Launch& L : plan) {
        switch (L.kind) {
          case 0: {
            // the register-resident panel up to 512 x kRegMaxRows rows left
            // (the fewest warps that hold the rows, one row per thread below
            // 257 rows), the shared-memory one above; a launch is sized by its
            // first (largest) block
            const int mr = 2 * rng[pitems[L.off]].y - L.k0;
            const int* list = B.list.p + L.off;
            TABI_K(K_LU, st);
            if (mr <= 256)
              lu_panel_reg_kernel<256, 1><<<L.cnt, 256, 0, st>>>(
                  list, L.k0, T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p, T.d_piv.p, d_info.p);
            else if (mr <= 512)
              lu_panel_reg_kernel<256, 2><<<L.cnt, 256, 0, st>>>(
                  list, L.k0, T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p, T.d_piv.p, d_info.p);
            else if (mr <= 512 * kRegMaxRows)
              lu_panel_reg_kernel<512, kRegMaxRows><<<L.cnt, 512, 0, st>>>(
                  list, L.k0, T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p, T.d_piv.p, d_info.p);
            else
              lu_panel_kernel<<<L.cnt, kPT, sizeof(double) * (size_t)mr * kSP, st>>>(
                  list, L.k0, T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p, T.d_piv.p, d_info.p);
            break;
          }
          case 1: {
            TABI_K(K_LU_STRIP, st);
            lu_strip_kernel<<<L.cnt, kUT, 0, st>>>(B.items.p + L.off, L.k0, T.d_leaf_rng.p,
                                                   T.d_blk_off.p, T.d_lu.p, T.d_piv.p);
            break;
          }
          case 2: {
            TABI_K(K_LU_UPDATE, st);
            lu_gemm_kernel<<<L.cnt, kUT, kGemmSmem, st>>>(B.gitems.p + L.off, L.k0, L.kdepth,
                                                          T.d_leaf_rng.p, T.d_blk_off.p,
                                                          T.d_lu.p);
            break;
          }
          case 3: {
            TABI_K(K_LU_SWAP, st);
            lu_swapmap_kernel<<<L.cnt, 256, 0, st>>>(B.mleaves.p + L.off, L.k0,
                                                     T.d_leaf_rng.p, T.d_piv.p, B.map.p);
            break;
          }
          case 4: {
            TABI_K(K_LU_SWAP, st);
            lu_rowswap_kernel<<<L.cnt, kUT, 0, st>>>(B.ritems.p + L.off, T.d_leaf_rng.p,
                                                     T.d_blk_off.p, B.map.p, T.d_lu.p);
            break;
          }
        }
      }
    };
    if (!grp[0].empty()) run_group(grp[0], H.pc_plan[0], s);
    if (!grp[1].empty()) run_group(grp[1], H.pc_plan[1], split ? H.side : s);
    join(split);
    if (any_big) {
      H.pc_big.alloc(big_leaves.size());
      TABI_CUDA(cudaMemcpyAsync(H.pc_big.p, big_leaves.data(), sizeof(int) * big_leaves.size(),
                                cudaMemcpyHostToDevice, s));
      TABI_K(K_LU, s);
      lu_kernel<<<(int)big_leaves.size(), kLuThreads, 0, s>>>(
          H.pc_big.p, T.d_leaf_rng.p, T.d_blk_off.p, T.d_lu.p, T.d_piv.p, d_info.p, kPanelMaxM);
    }
  // pivot permutations and inverse diagonal blocks for the applies
  {
    T.dinv_off.resize(nl);
    int64_t doff = 0;
    std::vector<int2> dblocks;
    for (int l = 0; l < nl; ++l) {
      T.dinv_off[l] = doff;
      int m = 2 * rng[l].y;
      int nblk = (m + kDB - 1) / kDB;
      doff += (int64_t)nblk * 2 * kDB * kDB;
      for (int b = 0; b < nblk; ++b) dblocks.push_back(make_int2(l, b * kDB));
    }
    while (dblocks.size() % 4) dblocks.push_back(make_int2(-1, 0));
    T.d_dinv.alloc(std::max<int64_t>(doff, 1));
    T.d_dinv_off.alloc(nl);
    T.d_lu_perm.alloc(2 * (size_t)H.n);
    H.pc_dblocks.alloc(std::max<size_t>(dblocks.size(), 1));
    TABI_CUDA(cudaMemcpyAsync(T.d_dinv_off.p, T.dinv_off.data(), sizeof(int64_t) * nl,
                              cudaMemcpyHostToDevice, s));
    TABI_CUDA(cudaMemcpyAsync(H.pc_dblocks.p, dblocks.data(), sizeof(int2) * dblocks.size(),
                              cudaMemcpyHostToDevice, s));
    { TABI_K(K_LU_POST, s); lu_perm_kernel<<<ceil_div(nl, 64), 64, 0, s>>>(T.d_leaf_rng.p, T.d_piv.p, nl, T.d_lu_perm.p); }
    { TABI_K(K_LU_POST, s); lu_diaginv_kernel<<<(int)(dblocks.size() / 4), 128, 0, s>>>(
        H.pc_dblocks.p, T.d_leaf_rng.p, T.d_blk_off.p, T.d_dinv_off.p, T.d_lu.p, T.d_dinv.p,
        d_info.p); }
  }
  }
  {
    std::vector<int> info(nl);
    TABI_CUDA(cudaMemcpyAsync(info.data(), d_info.p, sizeof(int) * nl, cudaMemcpyDeviceToHost,
                              s));
    TABI_CUDA(cudaStreamSynchronize(s));
    for (int l = 0; l < nl; ++l) {
      if (info[l] > 0)
        throw Error(TABI_ERR_SINGULAR, "leaf block " + std::to_string(l) +
                                           " is singular (DGETRF info " +
                                           std::to_string(info[l]) + ")");
      if (info[l] < 0)
        throw Error(TABI_ERR_SINGULAR, "leaf block " + std::to_string(l) +
                                           " has a non-finite pivot at row " +
                                           std::to_string(-info[l]) +
                                           " (coincident faces or non-finite surface data)");
    }
  }
  H.pc_lu_phase.reset();
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
  TABI_PHASE(K_PHASE_APPLY, s);
  // two arrays of the block order m = 2 * leaf size, 32 doubles per warp and
  // two staged 32 x 32 inverse diagonal blocks
  size_t smem = sizeof(double) * (4 * (size_t)T.max_leaf + 512 + 2 * kDB * kDB);
  TABI_REQUIRE(smem <= 200 * 1024, TABI_ERR_LIMIT, "leaf too large for the block solve");
  if (smem > 48 * 1024) {
    raise_smem_limit((const void*)solve_kernel<256>, smem);
    raise_smem_limit((const void*)solve_kernel<512>, smem);
  }
  // a shard applies the leaves of its target range only
  const int nbig = T.ranged ? T.r_solve_big : T.n_solve_big;
  const int nsmall = T.ranged ? T.r_solve_small : T.n_solve_small;
  const int* list = T.ranged ? T.d_r_solve_list.p : T.d_solve_list.p;
  const bool fork = nbig > 0 && nsmall > 0 && H.side != nullptr;
  cudaStream_t s2 = fork ? H.side : s;
  if (fork) {
    TABI_CUDA(cudaEventRecord(H.ev_fork, s));
    TABI_CUDA(cudaStreamWaitEvent(s2, H.ev_fork, 0));
  }
  if (nbig > 0) {
    TABI_K(K_SOLVE, s);
    solve_kernel<512><<<nbig, 512, smem, s>>>(T.d_leaf_rng.p, T.d_blk_off.p, T.d_dinv_off.p,
                                              list, T.d_lu.p, T.d_dinv.p, T.d_lu_perm.p, n, r,
                                              z);
  }
  if (nsmall > 0) {
    TABI_K(K_SOLVE, s2);
    solve_kernel<256><<<nsmall, 256, smem, s2>>>(T.d_leaf_rng.p, T.d_blk_off.p, T.d_dinv_off.p,
                                                 list + nbig, T.d_lu.p, T.d_dinv.p,
                                                 T.d_lu_perm.p, n, r, z);
  }
  if (fork) {
    TABI_CUDA(cudaEventRecord(H.ev_join, s2));
    TABI_CUDA(cudaStreamWaitEvent(s, H.ev_join, 0));
  }
  TABI_CUDA(cudaGetLastError());
}

}  // namespace tabi
