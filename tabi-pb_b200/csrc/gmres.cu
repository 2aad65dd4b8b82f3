// gmres.cu -- restarted, left-preconditioned GMRES with the semantics of the
// reference's vendored SLATEC DGMRES (dgmres_dep.f) as main.f90:92-137 calls
// it: ITOL = 2 (stop when |M^-1 (b - A x)| / |M^-1 b| <= tol), JPRE = -1,
// JSCAL = 0, KMP = MAXL (full modified Gram-Schmidt), restarts from the
// recurrence residual.  The small Hessenberg / Givens work (DHEQR, DHELS) runs
// on the host exactly as SLATEC does it; every length-2N vector operation
// runs on the device:
//   DORTH (dgmres_dep.f:1376-1415)  dot -> device slot, axpy reading that slot,
//                                    so one host round trip per iteration,
//   DRLCAL (:1948-1979)             the residual recurrence collapsed into one
//                                    linear combination of the Krylov vectors,
//                                    fused with its norm (ISDGMR :2532-2650),
//   DPIGMR final update (:1836-1848) one linear combination.
#include <cooperative_groups.h>

#include <cmath>
#include <vector>

#include "reduce.cuh"
#include "tabi_impl.cuh"

namespace tabi {

double reduce_dev(Handle& H, int op, const double* a, const double* b, int n, cudaStream_t s);

namespace {

struct Coefs {
  double c[64];
};

__global__ void __launch_bounds__(kRedThreads) lincomb_kernel(const double* __restrict__ V,
                                                              int64_t ld, int n, int nv,
                                                              Coefs cf, double* __restrict__ out,
                                                              double* __restrict__ part) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int j = 0; j < nv; ++j) v = fma(cf.c[j], V[(int64_t)j * ld + i], v);
    out[i] = v;
    acc = fma(v, v, acc);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double s[kRedThreads / 32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0 && part) {
    double t = 0.0;
    for (int k = 0; k < kRedThreads / 32; ++k) t += s[k];
    part[blockIdx.x] = t;
  }
}

// y += sign * (*coef) * x
__global__ void axpy_dcoef_kernel(int n, const double* __restrict__ coef, double sign,
                                  const double* __restrict__ x, double* __restrict__ y) {
  double a = sign * (*coef);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}
__global__ void axpy_kernel(int n, double a, const double* __restrict__ x,
                            double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = fma(a, x[i], y[i]);
}
__global__ void scal_kernel(int n, double a, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = a * x[i];
}
__global__ void sub_kernel(int n, const double* __restrict__ b, double* __restrict__ r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r[i] = b[i] - r[i];
}

constexpr int kVecBlocks = 592;
constexpr int kOrthThreads = 256;

// Sum of part[0..np) in a fixed order, identical in every block.
__device__ __forceinline__ double block_sum_parts(const double* part, int np, double* sm) {
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += part[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sm[k];
  __syncthreads();
  return t;
}

__device__ __forceinline__ void block_partial(double acc, double* part, double* sm) {
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sm[k];
    part[blockIdx.x] = t;
  }
  __syncthreads();
}

// DORTH's modified Gram-Schmidt (dgmres_dep.f:1376-1395) in one cooperative
// launch: out[maxlp1] = |vn|^2 before, out[i-1] = h_i = V_i . vn followed by
// vn -= h_i V_i for i = i0..ll in order, out[maxlp1+1] = |vn|^2 after.  Each
// thread owns the same elements in every pass, so an axpy and the next dot
// need no barrier; the partial sums are double-buffered and every block adds
// them in the same order, so all blocks see the same h_i.
__global__ void __launch_bounds__(kOrthThreads) dorth_kernel(const double* __restrict__ V,
                                                            int64_t ld, int n, int i0, int ll,
                                                            int maxlp1, double* __restrict__ vn,
                                                            double* __restrict__ part,
                                                            double* __restrict__ out) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double sm[kOrthThreads / 32];
  const int np = gridDim.x;
  const int stride = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  int buf = 0;
  double acc = 0.0;
  for (int k = t0; k < n; k += stride) acc = fma(vn[k], vn[k], acc);
  block_partial(acc, part + buf * np, sm);
  grid.sync();
  {
    double s = block_sum_parts(part + buf * np, np, sm);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[maxlp1] = s;
  }
  for (int i = i0; i <= ll; ++i) {
    const double* vi = V + (int64_t)(i - 1) * ld;
    buf ^= 1;
    acc = 0.0;
    for (int k = t0; k < n; k += stride) acc = fma(vi[k], vn[k], acc);
    block_partial(acc, part + buf * np, sm);
    grid.sync();
    const double h = block_sum_parts(part + buf * np, np, sm);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[i - 1] = h;
    for (int k = t0; k < n; k += stride) vn[k] = fma(-h, vi[k], vn[k]);
  }
  buf ^= 1;
  acc = 0.0;
  for (int k = t0; k < n; k += stride) acc = fma(vn[k], vn[k], acc);
  block_partial(acc, part + buf * np, sm);
  grid.sync();
  {
    double s = block_sum_parts(part + buf * np, np, sm);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[maxlp1 + 1] = s;
  }
}

void givens(double t1, double t2, double& c, double& s) {
  if (t2 == 0.0) {
    c = 1.0;
    s = 0.0;
  } else if (std::fabs(t2) >= std::fabs(t1)) {
    double t = t1 / t2;
    s = -1.0 / std::sqrt(1.0 + t * t);
    c = -s * t;
  } else {
    double t = t2 / t1;
    c = 1.0 / std::sqrt(1.0 + t * t);
    s = -c * t;
  }
}

// A target-restricted handle computes its own shard of each operator and
// preconditioner result; the exchange completes the vector with the other
// ranks' slices (in place, ordered on s) before GMRES uses it.
void shard_exchange(Handle& H, double* v, cudaStream_t s) {
  if (!H.tree.ranged) return;
  TABI_REQUIRE(H.xchg != nullptr, TABI_ERR_STATE, "a target range is set but no exchange");
  const int rc = H.xchg(H.xchg_user, v, 2 * H.n, H.tree.rt0, H.tree.rt1, s);
  TABI_REQUIRE(rc == 0, TABI_ERR_STATE,
               "the shard exchange failed (tabi_set_exchange callback returned " +
                   std::to_string(rc) + ")");
}

void op_matvec(Handle& H, const double* x, double* y, cudaStream_t s, bool shortcut) {
  matvec_dev(H, x, y, s, shortcut);
  shard_exchange(H, y, s);
}

void op_msolve(Handle& H, const double* r, double* z, cudaStream_t s) {
  msolve_dev(H, r, z, s);
  shard_exchange(H, z, s);
}

}  // namespace

void gmres_dev(Handle& H, const double* b, double* x, int* iter_out, double* err_out,
               int* ierr_out, double* hist, int* nhist, cudaStream_t s, double tol_in,
               const double* minv_b, double minv_b_nrm) {
  const int n = 2 * H.n;
  int maxl = H.prm.maxl;
  if (maxl == 0) maxl = 10;
  if (maxl > n) maxl = n;
  TABI_REQUIRE(maxl <= 60, TABI_ERR_ARG, "maxl must be <= 60");
  const int kmp = maxl;
  int nrmax = H.prm.nrmax;
  if (nrmax == 0) nrmax = 10;
  if (nrmax == -1) nrmax = 0;
  double tol = tol_in >= 0.0 ? tol_in : H.prm.tol;
  if (tol == 0.0) tol = 500 * 1e-20;
  const int maxlp1 = maxl + 1, ldh = maxlp1;
  H.d_v.alloc((size_t)n * maxlp1);
  H.d_wk.alloc(n);
  H.d_dl.alloc(n);
  H.d_gz.alloc(n);
  H.d_r.alloc(n);
  H.d_coef.alloc(4 * (size_t)maxlp1 + kRedBlocks + 8);
  H.d_red.alloc(kRedBlocks + 8);
  // cooperative DORTH: every block must be resident
  int orth_blocks = 0;
  {
    int per_sm = 0, nsm = 0, dev = 0;
    TABI_CUDA(cudaGetDevice(&dev));
    TABI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    TABI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dorth_kernel, kOrthThreads, 0));
    orth_blocks = std::max(1, std::min(2, per_sm)) * nsm;
    orth_blocks = std::min(orth_blocks, std::max(1, ceil_div(n, kOrthThreads)));
  }
  H.d_orth.alloc(2 * (size_t)orth_blocks + 8);
  double* d_orth_part = H.d_orth.p;
  double* V = H.d_v.p;
  double* wk = H.d_wk.p;
  double* dl = H.d_dl.p;
  double* z = H.d_gz.p;
  double* r = H.d_r.p;
  double* d_h = H.d_coef.p;                       // HES column slots
  double* d_part = H.d_coef.p + 4 * maxlp1;       // partial sums
  std::vector<double> hes((size_t)maxlp1 * maxl), q(2 * maxl), r0ls(maxlp1 + 1);
  auto HES = [&](int i, int j) -> double& { return hes[(size_t)(j - 1) * ldh + (i - 1)]; };
  auto Vc = [&](int j) { return V + (size_t)(j - 1) * n; };
  const int vb = kVecBlocks, vt = 256;
  auto lincomb_norm = [&](int nv, const Coefs& cf, double* out, bool want_norm) -> double {
    int nb = std::min(kRedBlocks, ceil_div(n, kRedThreads));
    { TABI_K(K_VEC, s); lincomb_kernel<<<nb, kRedThreads, 0, s>>>(V, n, n, nv, cf, out, want_norm ? d_part : nullptr); }
    if (!want_norm) return 0.0;
    { TABI_K(K_VEC, s); reduce_final_kernel<<<1, 256, 0, s>>>(d_part, nb, d_part + kRedBlocks); }
    TABI_CUDA(cudaMemcpyAsync(H.h_pinned, d_part + kRedBlocks, sizeof(double),
                              cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(H.h_pinned[0]);
  };

  int iter = 0, ierr = 0, nh = 0;
  double err = 0.0;
  int nrsts = 0;
  // DGMRES :754-781: BNRM = |M^-1 b|, r = b - A x
  double bnrm;
  if (minv_b) {
    TABI_CUDA(cudaMemcpyAsync(r, minv_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    bnrm = minv_b_nrm;
  } else {
    op_msolve(H, b, r, s);
    bnrm = nrm2_dev(H, r, n, s);
  }
  // the reference would iterate on NaNs to the iteration limit; a non-finite
  // right-hand side is refused instead
  TABI_REQUIRE(std::isfinite(bnrm), TABI_ERR_ARG,
               "the right-hand side is not finite (|M^-1 b| is NaN or Inf)");
  // r0 = b - A x; MATVECmain (main.f90:478-479) returns y = x for sum|x| <
  // 1e-10, so an x of exact zeros gives r0 = b bit for bit and M^-1 r0 is the
  // M^-1 b already in r: DPIGMR's first preconditioner apply is skipped
  const double ax = asum_dev(H, x, n, s);
  const bool x_zero = ax == 0.0;
  if (!x_zero) {
    if (ax < 1e-10)
      TABI_CUDA(cudaMemcpyAsync(r, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    else
      op_matvec(H, x, r, s, false);
    { TABI_K(K_VEC, s); sub_kernel<<<vb, vt, 0, s>>>(n, b, r); }
  }
  for (;;) {
    if (nrsts > nrmax) {
      ierr = 1;
      break;
    }
    if (nrsts > 0) TABI_CUDA(cudaMemcpyAsync(r, dl, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    // ---- DPIGMR
    int iflag = 0, lgmr = 0;
    double snormw = 0.0, prod = 1.0, rho = 0.0;
    if (nrsts == 0 && !x_zero) {
      TABI_CUDA(cudaMemcpyAsync(wk, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      op_msolve(H, wk, r, s);
    }
    TABI_CUDA(cudaMemcpyAsync(Vc(1), r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    double r0nrm = nrm2_dev(H, Vc(1), n, s);
    TABI_REQUIRE(nrsts > 0 || std::isfinite(r0nrm), TABI_ERR_ARG,
                 "the initial residual is not finite (x0 holds NaN or Inf)");
    err = r0nrm / bnrm;  // ISDGMR with LGMR = 0
    bool zero_z = true;
    if (!(err <= tol)) {
      { TABI_K(K_VEC, s); scal_kernel<<<vb, vt, 0, s>>>(n, 1.0 / r0nrm, Vc(1)); }
      std::fill(hes.begin(), hes.end(), 0.0);
      prod = 1.0;
      bool go200 = false, go120 = false;
      for (int ll = 1; ll <= maxl; ++ll) {
        lgmr = ll;
        double* vn = Vc(ll + 1);
        op_matvec(H, Vc(ll), wk, s, false);  // |V(:,ll)| = 1: never the zero shortcut
        op_msolve(H, wk, vn, s);
        // ---- DORTH: one cooperative launch for the whole sweep
        int i0 = std::max(1, ll - kmp + 1);
        {
          TABI_K(K_VEC, s);
          const double* Vp = V;
          int64_t ldv = n;
          int nn = n, ii0 = i0, lll = ll, mlp1 = maxlp1;
          double* vnp = vn;
          double* pp = d_orth_part;
          double* op = d_h;
          void* args[] = {(void*)&Vp, (void*)&ldv, (void*)&nn, (void*)&ii0, (void*)&lll,
                          (void*)&mlp1, (void*)&vnp, (void*)&pp, (void*)&op};
          TABI_CUDA(cudaLaunchCooperativeKernel((const void*)dorth_kernel, dim3(orth_blocks),
                                                dim3(kOrthThreads), args, 0, s));
        }
        TABI_CUDA(cudaMemcpyAsync(H.h_pinned, d_h, sizeof(double) * (maxlp1 + 2),
                                  cudaMemcpyDeviceToHost, s));
        TABI_CUDA(cudaStreamSynchronize(s));
        for (int i = i0; i <= ll; ++i) HES(i, ll) = H.h_pinned[i - 1];
        double vnrm = std::sqrt(H.h_pinned[maxlp1]);
        snormw = std::sqrt(H.h_pinned[maxlp1 + 1]);
        if (!(vnrm + 0.001 * snormw != vnrm)) {
          // conditional re-orthogonalisation (dgmres_dep.f:1397-1414)
          double sumdsq = 0.0;
          for (int i = i0; i <= ll; ++i) {
            double tem = -dot_dev(H, Vc(i), vn, n, s);
            if (HES(i, ll) + 0.001 * tem == HES(i, ll)) continue;
            HES(i, ll) = HES(i, ll) - tem;
            { TABI_K(K_VEC, s); axpy_kernel<<<vb, vt, 0, s>>>(n, tem, Vc(i), vn); }
            sumdsq += tem * tem;
          }
          if (sumdsq != 0.0) snormw = std::sqrt(std::max(0.0, snormw * snormw - sumdsq));
        }
        HES(ll + 1, ll) = snormw;
        // ---- DHEQR (IJOB = 1 for ll = 1, else 2)
        int info = 0;
        for (int k = 1; k <= ll - 1; ++k) {
          double t1 = HES(k, ll), t2 = HES(k + 1, ll);
          double c = q[2 * (k - 1)], sn = q[2 * (k - 1) + 1];
          HES(k, ll) = c * t1 - sn * t2;
          HES(k + 1, ll) = sn * t1 + c * t2;
        }
        {
          double c, sn, t1 = HES(ll, ll), t2 = HES(ll + 1, ll);
          givens(t1, t2, c, sn);
          q[2 * ll - 2] = c;
          q[2 * ll - 1] = sn;
          HES(ll, ll) = c * t1 - sn * t2;
          if (HES(ll, ll) == 0.0) info = ll;
        }
        if (info == ll) {
          go120 = true;
          break;
        }
        prod = prod * q[2 * ll - 1];
        rho = std::fabs(prod * r0nrm);
        // ---- ISDGMR with DRLCAL: dl = r0nrm*prod * (recurrence of V columns)
        Coefs cf{};
        cf.c[0] = 1.0;
        for (int i = 1; i <= ll - 1; ++i) {
          double sn = q[2 * i - 1], c = q[2 * i - 2];
          for (int j = 0; j < i; ++j) cf.c[j] *= sn;
          cf.c[i] += c;
        }
        {
          double sn = q[2 * ll - 1], c = q[2 * ll - 2] / snormw;
          for (int j = 0; j < ll; ++j) cf.c[j] *= sn;
          cf.c[ll] += c;
        }
        for (int j = 0; j <= ll; ++j) cf.c[j] *= r0nrm * prod;
        double rl = lincomb_norm(ll + 1, cf, dl, true);
        err = rl / bnrm;
        if (hist) hist[nh] = err;
        nh++;
        if (err <= tol) {
          go200 = true;
          break;
        }
        if (ll == maxl) break;
        { TABI_K(K_VEC, s); scal_kernel<<<vb, vt, 0, s>>>(n, 1.0 / snormw, vn); }
      }
      if (!go200 && !go120) {
        if (rho < r0nrm) {
          iflag = 1;
          // DRLCAL(MAXL) at label 150: already in dl from the last iteration
          go200 = true;
        } else {
          go120 = true;
        }
      }
      if (go120) {
        iflag = 2;
      } else {
        // DHELS (dgmres_dep.f:925-950) and z = V(:,1:lgmr) * y
        int l = lgmr;
        std::fill(r0ls.begin(), r0ls.end(), 0.0);
        r0ls[0] = r0nrm;
        for (int k = 1; k <= l; ++k) {
          double c = q[2 * (k - 1)], sn = q[2 * (k - 1) + 1];
          double t1 = r0ls[k - 1], t2 = r0ls[k];
          r0ls[k - 1] = c * t1 - sn * t2;
          r0ls[k] = sn * t1 + c * t2;
        }
        for (int kb = 1; kb <= l; ++kb) {
          int k = l + 1 - kb;
          r0ls[k - 1] = r0ls[k - 1] / HES(k, k);
          double t = -r0ls[k - 1];
          for (int i = 1; i <= k - 1; ++i) r0ls[i - 1] += t * HES(i, k);
        }
        Coefs cf{};
        for (int i = 0; i < l; ++i) cf.c[i] = r0ls[i];
        lincomb_norm(l, cf, z, false);
        zero_z = false;
      }
    }
    // ---- DGMRES :796-814
    iter += lgmr;
    if (!zero_z) { TABI_K(K_VEC, s); axpy_kernel<<<vb, vt, 0, s>>>(n, 1.0, z, x); }
    if (iflag == 0) {
      ierr = 0;
      break;
    }
    if (iflag == 1) {
      nrsts++;
      continue;
    }
    ierr = 2;
    break;
  }
  TABI_CUDA(cudaStreamSynchronize(s));
  TABI_CUDA(cudaGetLastError());
  *iter_out = iter;
  *err_out = err;
  *ierr_out = ierr;
  if (nhist) *nhist = nh;
}

// Mixed precision: FP64 iterative refinement around GMRES on the FP32
// treecode operator.  Each outer step forms the true residual r = b - A x with
// the FP64 operator and measures it the way DGMRES does for ITOL = 2,
// |M^-1 r| / |M^-1 b|; while that is above tol, GMRES (FP64 vectors, Arnoldi
// and Givens, FP32 operator) solves A d = r to the relative tolerance
// tol * |M^-1 b| / |M^-1 r| and x += d.  The FP64 residual decides: the
// solve stops only when it is below tol.  iter counts the inner iterations,
// err is the final FP64 measure, err_hist the inner estimates rescaled to
// |M^-1 b| (at most (nrmax+1)*maxl of them, the same cap as the FP64 path,
// which also bounds the inner iterations in total).
void solve_dev(Handle& H, const double* b, double* x, int* iter_out, double* err_out,
               int* ierr_out, double* hist, int* nhist, cudaStream_t s) {
  TABI_REQUIRE(!H.tree.ranged || H.xchg, TABI_ERR_STATE,
               "a target range is set: the handle computes one shard of the operator, and "
               "the solve across the shards needs an exchange (tabi_set_exchange)");
  if (H.prm.precision != TABI_PREC_MIXED) {
    H.mv_prec = TABI_PREC_FP64;
    gmres_dev(H, b, x, iter_out, err_out, ierr_out, hist, nhist, s);
    return;
  }
  const int n = 2 * H.n;
  int maxl = H.prm.maxl == 0 ? 10 : H.prm.maxl;
  int nrmax = H.prm.nrmax == 0 ? 10 : (H.prm.nrmax == -1 ? 0 : H.prm.nrmax);
  const int cap = (nrmax + 1) * maxl;
  double tol = H.prm.tol;
  if (tol == 0.0) tol = 500 * 1e-20;
  H.d_ir_r.alloc(n);
  H.d_ir_d.alloc(n);
  H.d_ir_t.alloc(n);
  double* r = H.d_ir_r.p;
  double* d = H.d_ir_d.p;
  double* t = H.d_ir_t.p;
  const int vb = kVecBlocks, vt = 256;
  op_msolve(H, b, t, s);
  const double bnrm = nrm2_dev(H, t, n, s);
  TABI_REQUIRE(std::isfinite(bnrm), TABI_ERR_ARG,
               "the right-hand side is not finite (|M^-1 b| is NaN or Inf)");
  std::vector<double> inner_hist((size_t)cap + 1);
  int iter = 0, ierr = 0, nh = 0;
  double err = 0.0;
  constexpr int kMaxOuter = 20;
  double tnrm = bnrm;  // |M^-1 r| of the current residual
  for (int outer = 0;; ++outer) {
    // FP64 residual and its ITOL = 2 measure; from an x of exact zeros the
    // residual is b and M^-1 b is already in t
    H.mv_prec = TABI_PREC_FP64;
    if (outer == 0 && asum_dev(H, x, n, s) == 0.0) {
      TABI_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
      op_matvec(H, x, r, s, true);
      { TABI_K(K_VEC, s); sub_kernel<<<vb, vt, 0, s>>>(n, b, r); }
      op_msolve(H, r, t, s);
      tnrm = nrm2_dev(H, t, n, s);
    }
    err = tnrm / bnrm;
    TABI_REQUIRE(outer > 0 || std::isfinite(err), TABI_ERR_ARG,
                 "the initial residual is not finite (x0 holds NaN or Inf)");
    if (err <= tol) {
      ierr = 0;
      break;
    }
    if (outer == kMaxOuter || iter >= cap) {
      ierr = 1;
      break;
    }
    // inner GMRES on the FP32 operator: A d = r from d = 0
    H.mv_prec = TABI_PREC_MIXED;
    TABI_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, s));
    int it = 0, ie = 0, nhi = 0;
    double ei = 0.0;
    gmres_dev(H, r, d, &it, &ei, &ie, inner_hist.data(), &nhi, s, tol / err, t, tnrm);
    for (int k = 0; k < nhi && nh < cap; ++k) {
      if (hist) hist[nh] = inner_hist[k] * err;
      ++nh;
    }
    iter += it;
    { TABI_K(K_VEC, s); axpy_kernel<<<vb, vt, 0, s>>>(n, 1.0, d, x); }
    if (ie == 2 || ie < 0) {  // stagnation (or an input error) of the inner solve
      H.mv_prec = TABI_PREC_FP64;
      op_matvec(H, x, r, s, true);
      { TABI_K(K_VEC, s); sub_kernel<<<vb, vt, 0, s>>>(n, b, r); }
      op_msolve(H, r, t, s);
      err = nrm2_dev(H, t, n, s) / bnrm;
      ierr = err <= tol ? 0 : ie;
      break;
    }
  }
  H.mv_prec = TABI_PREC_MIXED;
  TABI_CUDA(cudaStreamSynchronize(s));
  TABI_CUDA(cudaGetLastError());
  *iter_out = iter;
  *err_out = err;
  *ierr_out = ierr;
  if (nhist) *nhist = nh;
}

}  // namespace tabi
