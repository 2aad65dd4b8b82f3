// tree.cu -- device tree build and interaction lists.
//
// Tree (treecode3d_pb.f:142-356 CREATE_TREE / PARTITION_8 / PARTITION):
// a node holding more than maxparnode faces is split at the midpoint of its
// box along every dimension whose length is >= lmax/sqrt(2) (x, then y, then
// z; faces with coordinate <= mid go to the low side), giving 2, 4 or 8
// children in the reference's order (x bit lowest) and its array layout
// (first split dimension most significant in position); empty children are
// dropped and a child with >= 2 faces gets the bounding box of its faces.
// The build here is level-synchronous: per level one pass computes each
// face's child code and per-chunk histograms, the host turns the histograms
// into child ranges, and a stable scatter moves the faces.  Node sets, boxes,
// midpoints and radii are bit-identical to the reference's (IEEE min/max,
// midpoint and radius without contraction); only the order of faces inside a
// node differs (the reference's PARTITION is not stable).
//
// Interaction lists (treecode3d_pb.f:359-436 COMPP_TREE): a warp walks the
// tree for 32 consecutive targets with a shared stack of (node, lane mask).
// Each lane applies the reference's per-target MAC
//     radius < theta * |mid - target|  and  numpar > 40
// so every target gets exactly the reference's far clusters and near leaves.
// Lists depend only on geometry and are built once per tree.
#include <algorithm>
#include <cstdio>
#include <numeric>

#include "tabi_impl.cuh"

namespace tabi {

namespace {

constexpr int kChunk = 4096;  // faces per tree-build chunk
constexpr int kBT = 256;      // tree-build block size

__device__ __forceinline__ unsigned long long ord_enc(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double ord_dec(unsigned long long e) {
  unsigned long long b = (e >> 63) ? (e & 0x7FFFFFFFFFFFFFFFULL) : ~e;
  return __longlong_as_double((long long)b);
}

__global__ void bbox_init_kernel(unsigned long long* bb, int n0, int n1) {
  int c = n0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n1) return;
  unsigned long long lo = ord_enc(__longlong_as_double(0x7FF0000000000000LL));   // +inf
  unsigned long long hi = ord_enc(__longlong_as_double((long long)0xFFF0000000000000ULL));  // -inf
  bb[6 * c + 0] = lo;
  bb[6 * c + 1] = hi;
  bb[6 * c + 2] = lo;
  bb[6 * c + 3] = hi;
  bb[6 * c + 4] = lo;
  bb[6 * c + 5] = hi;
}

// chunks: (node, start, count, -)
__global__ void __launch_bounds__(kBT) bbox_kernel(const int4* chunks, const double* x,
                                                   const double* y, const double* z,
                                                   unsigned long long* bb) {
  int4 ch = chunks[blockIdx.x];
  const double inf = __longlong_as_double(0x7FF0000000000000LL);
  double mn[3] = {inf, inf, inf};
  double mx[3] = {-inf, -inf, -inf};
  for (int i = threadIdx.x; i < ch.z; i += blockDim.x) {
    int k = ch.y + i;
    double v[3] = {x[k], y[k], z[k]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mn[d] = fmin(mn[d], v[d]);
      mx[d] = fmax(mx[d], v[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = fmin(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  }
  __shared__ double smn[3][kBT / 32], smx[3][kBT / 32];
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int d = 0; d < 3; ++d) {
      smn[d][w] = mn[d];
      smx[d][w] = mx[d];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int d = 0; d < 3; ++d) {
      double a = smn[d][0], b = smx[d][0];
      for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
        a = fmin(a, smn[d][k]);
        b = fmax(b, smx[d][k]);
      }
      atomicMin(&bb[6 * ch.x + 2 * d], ord_enc(a));
      atomicMax(&bb[6 * ch.x + 2 * d + 1], ord_enc(b));
    }
  }
}

// Node geometry (treecode3d_pb.f:186-209) and split dimensions
// (PARTITION_8 :312-353) for nodes [n0, n1).
__global__ void finalize_kernel(const unsigned long long* bb, const int* num, int n0, int n1,
                                int maxparnode, double* mid, double* rad, int* split) {
  int c = n0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n1) return;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = ord_dec(bb[6 * c + 2 * d]);
    hi[d] = ord_dec(bb[6 * c + 2 * d + 1]);
  }
  double m[3], t[3], len[3];
  for (int d = 0; d < 3; ++d) {
    m[d] = __dmul_rn(__dadd_rn(hi[d], lo[d]), 0.5);  // (max+min)/2, exact halving
    t[d] = __dsub_rn(hi[d], m[d]);
    len[d] = __dsub_rn(hi[d], lo[d]);
    mid[3 * c + d] = m[d];
  }
  double r2 = __dadd_rn(__dadd_rn(__dmul_rn(t[0], t[0]), __dmul_rn(t[1], t[1])),
                        __dmul_rn(t[2], t[2]));
  rad[c] = __dsqrt_rn(r2);
  int s = 0;
  if (num[c] > maxparnode) {
    double lmax = fmax(fmax(len[0], len[1]), len[2]);
    double crit = __ddiv_rn(lmax, __dsqrt_rn(2.0));
    if (len[0] >= crit) s |= 1;
    if (len[1] >= crit) s |= 2;
    if (len[2] >= crit) s |= 4;
    if (lmax == 0.0) s |= 8;  // coincident centroids: cannot be split
  }
  split[c] = s;
}

__device__ __forceinline__ int child_code(double x, double y, double z, const double* m,
                                          int s) {
  int code = 0, bit = 0;
  if (s & 1) code |= (x > m[0]) << bit++;
  if (s & 2) code |= (y > m[1]) << bit++;
  if (s & 4) code |= (z > m[2]) << bit++;
  return code;
}

__global__ void __launch_bounds__(kBT) code_kernel(const int4* chunks, const double* x,
                                                   const double* y, const double* z,
                                                   const double* mid, const int* split,
                                                   unsigned char* code, int* hist) {
  int4 ch = chunks[blockIdx.x];
  __shared__ int h[8];
  if (threadIdx.x < 8) h[threadIdx.x] = 0;
  __syncthreads();
  double m[3] = {mid[3 * ch.x], mid[3 * ch.x + 1], mid[3 * ch.x + 2]};
  int s = split[ch.x];
  for (int i = threadIdx.x; i < ch.z; i += blockDim.x) {
    int k = ch.y + i;
    int c = child_code(x[k], y[k], z[k], m, s);
    code[k] = (unsigned char)c;
    atomicAdd(&h[c], 1);
  }
  __syncthreads();
  if (threadIdx.x < 8) hist[8 * blockIdx.x + threadIdx.x] = h[threadIdx.x];
}

// Stable scatter of a chunk's faces to base[chunk][code] + rank.
__global__ void __launch_bounds__(kBT) scatter_kernel(const int4* chunks, const int* base,
                                                      const unsigned char* code,
                                                      const double* x, const double* y,
                                                      const double* z, const int* perm,
                                                      double* tx, double* ty, double* tz,
                                                      int* tperm) {
  int4 ch = chunks[blockIdx.x];
  __shared__ int wcnt[kBT / 32][8];
  __shared__ int carry[8];
  if (threadIdx.x < 8) carry[threadIdx.x] = base[8 * blockIdx.x + threadIdx.x];
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  unsigned lt = (1u << l) - 1u;
  for (int t0 = 0; t0 < ch.z; t0 += blockDim.x) {
    __syncthreads();
    int i = t0 + threadIdx.x;
    bool ok = i < ch.z;
    int c = ok ? code[ch.y + i] : 8;
    int rank = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      unsigned m = __ballot_sync(0xffffffffu, c == k);
      if (c == k) rank = __popc(m & lt);
      if (l == 0) wcnt[w][k] = __popc(m);
    }
    __syncthreads();
    if (ok) {
      int off = carry[c];
      for (int ww = 0; ww < w; ++ww) off += wcnt[ww][c];
      int dst = off + rank;
      int src = ch.y + i;
      tx[dst] = x[src];
      ty[dst] = y[src];
      tz[dst] = z[src];
      tperm[dst] = perm[src];
    }
    __syncthreads();
    if (threadIdx.x < 8) {
      int tot = 0;
      for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) tot += wcnt[ww][threadIdx.x];
      carry[threadIdx.x] += tot;
    }
  }
}

__global__ void copy_back_kernel(const int4* chunks, const double* tx, const double* ty,
                                 const double* tz, const int* tperm, double* x, double* y,
                                 double* z, int* perm) {
  int4 ch = chunks[blockIdx.x];
  for (int i = threadIdx.x; i < ch.z; i += blockDim.x) {
    int k = ch.y + i;
    x[k] = tx[k];
    y[k] = ty[k];
    z[k] = tz[k];
    perm[k] = tperm[k];
  }
}

__global__ void iota_kernel(int* p, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

__global__ void gather4_kernel(const int* perm, int n, const double* a, const double* b,
                               const double* c, const double* d, double* ta, double* tb,
                               double* tc, double* td) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int o = perm[i];
  ta[i] = a[o];
  tb[i] = b[o];
  tc[i] = c[o];
  td[i] = d[o];
}

// ---------------------------------------------------------------- lists

constexpr int kTW = 4;  // warps per traversal block

template <bool FILL>
__global__ void __launch_bounds__(32 * kTW) traverse_kernel(
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
    int n, const int* __restrict__ nd_num, const int* __restrict__ nd_child0,
    const int* __restrict__ nd_nchild, const double* __restrict__ nd_mid,
    const double* __restrict__ nd_rad, double theta, int* tgt_cnt, int* node_far_cnt,
    int* node_near_cnt, const int64_t* __restrict__ slot_off,
    const int64_t* __restrict__ far_off, const int64_t* __restrict__ near_off, int* far_fill,
    int* near_fill, int2* far_ent, int2* near_ent, int* err) {
  __shared__ int2 stack[kTW][kStack];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int t = (blockIdx.x * kTW + w) * 32 + lane;
  bool active = t < n;
  unsigned m0 = __ballot_sync(0xffffffffu, active);
  if (m0 == 0) return;
  double tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = px[t];
    ty = py[t];
    tz = pz[t];
  }
  unsigned lt = (1u << lane) - 1u;
  int sp = 0;
  if (lane == 0) stack[w][0] = make_int2(0, (int)m0);
  sp = 1;
  int cnt = 0;
  long long slot = (FILL && active) ? slot_off[t] : 0;
  __syncwarp();
  while (sp > 0) {
    --sp;
    int2 e = stack[w][sp];
    __syncwarp();
    int c = e.x;
    unsigned m = (unsigned)e.y;
    bool in = (m >> lane) & 1u;
    int num = nd_num[c];
    bool acc = false;
    if (in && num > kMacMinPar) {
      double dx = __dsub_rn(nd_mid[3 * c], tx);
      double dy = __dsub_rn(nd_mid[3 * c + 1], ty);
      double dz = __dsub_rn(nd_mid[3 * c + 2], tz);
      double dist = __dsqrt_rn(
          __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
      acc = nd_rad[c] < __dmul_rn(dist, theta);
    }
    unsigned am = __ballot_sync(0xffffffffu, acc);
    unsigned rm = m & ~am;
    if (am) {
      if (!FILL) {
        if (acc) cnt++;
        if (lane == __ffs(am) - 1) atomicAdd(&node_far_cnt[c], __popc(am));
      } else {
        int base = 0;
        if (lane == __ffs(am) - 1) base = atomicAdd(&far_fill[c], __popc(am));
        base = __shfl_sync(0xffffffffu, base, __ffs(am) - 1);
        if (acc) {
          long long pos = far_off[c] + base + __popc(am & lt);
          far_ent[pos] = make_int2(t, (int)slot);
          slot++;
        }
      }
    }
    if (rm) {
      int nc = nd_nchild[c];
      if (nc == 0) {
        bool rej = (rm >> lane) & 1u;
        if (!FILL) {
          if (rej) cnt++;
          if (lane == __ffs(rm) - 1) atomicAdd(&node_near_cnt[c], __popc(rm));
        } else {
          int base = 0;
          if (lane == __ffs(rm) - 1) base = atomicAdd(&near_fill[c], __popc(rm));
          base = __shfl_sync(0xffffffffu, base, __ffs(rm) - 1);
          if (rej) {
            long long pos = near_off[c] + base + __popc(rm & lt);
            near_ent[pos] = make_int2(t, (int)slot);
            slot++;
          }
        }
      } else {
        if (sp + nc > kStack) {
          if (lane == 0) atomicExch(err, 1);
          return;
        }
        int c0 = nd_child0[c];
        // push in reverse so children pop in reference order
        if (lane < nc) stack[w][sp + nc - 1 - lane] = make_int2(c0 + lane, (int)rm);
        sp += nc;
        __syncwarp();
      }
    }
  }
  if (!FILL && active) tgt_cnt[t] = cnt;
}

// exclusive scan of int counts into int64 offsets (n+1 entries)
constexpr int kScanB = 1024;
__global__ void scan_block_kernel(const int* in, int n, int64_t* out, int64_t* bsum) {
  __shared__ int64_t s[kScanB];
  int i = blockIdx.x * kScanB + threadIdx.x;
  int64_t v = (i < n) ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < kScanB; o <<= 1) {
    int64_t a = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += a;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == kScanB - 1) bsum[blockIdx.x] = s[threadIdx.x];
}
__global__ void scan_top_kernel(int64_t* bsum, int nb) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int64_t acc = 0;
  for (int b = 0; b < nb; ++b) {
    int64_t v = bsum[b];
    bsum[b] = acc;
    acc += v;
  }
  bsum[nb] = acc;
}
__global__ void scan_add_kernel(int64_t* out, int n, const int64_t* bsum) {
  int i = blockIdx.x * kScanB + threadIdx.x;
  if (i < n) out[i] += bsum[blockIdx.x];
  if (i == 0) out[n] = bsum[gridDim.x];
}

}  // namespace

// ------------------------------------------------------------------ host

void build_tree(Handle& H, cudaStream_t s) {
  Tree& T = H.tree;
  const int n = H.n;
  const int L = H.prm.maxparnode;
  T.clear();
  T.n = n;
  H.d_tx.alloc(n);
  H.d_ty.alloc(n);
  H.d_tz.alloc(n);
  H.d_tperm.alloc(n);
  H.d_code.alloc(n);
  H.d_perm.alloc(n);
  H.d_err.alloc(1);
  { TABI_K(K_TREE, s); iota_kernel<<<ceil_div(n, 256), 256, 0, s>>>(H.d_perm.p, n); }
  // node table, grown per level
  DBuf<unsigned long long>& bb = H.tb_bb;
  DBuf<double>& mid = H.tb_mid;
  DBuf<double>& rad = H.tb_rad;
  DBuf<int>& split = H.tb_split;
  DBuf<int>& numd = H.tb_num;
  int cap = (int)std::min({bb.n / 6, mid.n / 3, rad.n, split.n, numd.n});
  auto ensure = [&](int need) {
    if (need <= cap && bb.p) return;
    int nc = std::max(need, 2 * cap);
    DBuf<unsigned long long> bb2;
    DBuf<double> mid2, rad2;
    DBuf<int> sp2, nu2;
    bb2.alloc(6 * (size_t)nc);
    mid2.alloc(3 * (size_t)nc);
    rad2.alloc(nc);
    sp2.alloc(nc);
    nu2.alloc(nc);
    if (bb.p) {
      TABI_CUDA(cudaMemcpyAsync(bb2.p, bb.p, 6 * sizeof(unsigned long long) * cap,
                                cudaMemcpyDeviceToDevice, s));
      TABI_CUDA(cudaMemcpyAsync(mid2.p, mid.p, 3 * sizeof(double) * cap,
                                cudaMemcpyDeviceToDevice, s));
      TABI_CUDA(cudaMemcpyAsync(rad2.p, rad.p, sizeof(double) * cap, cudaMemcpyDeviceToDevice, s));
      TABI_CUDA(cudaMemcpyAsync(sp2.p, split.p, sizeof(int) * cap, cudaMemcpyDeviceToDevice, s));
      TABI_CUDA(cudaMemcpyAsync(nu2.p, numd.p, sizeof(int) * cap, cudaMemcpyDeviceToDevice, s));
      TABI_CUDA(cudaStreamSynchronize(s));
    }
    std::swap(bb.p, bb2.p);
    std::swap(bb.n, bb2.n);
    std::swap(mid.p, mid2.p);
    std::swap(mid.n, mid2.n);
    std::swap(rad.p, rad2.p);
    std::swap(rad.n, rad2.n);
    std::swap(split.p, sp2.p);
    std::swap(split.n, sp2.n);
    std::swap(numd.p, nu2.p);
    std::swap(numd.n, nu2.n);
    cap = nc;
  };
  ensure(1);
  T.ibeg = {0};
  T.num = {n};
  T.level = {0};
  T.child0 = {0};
  T.nchild = {0};
  int lv0 = 0, lv1 = 1;  // node range of the current level
  std::vector<int4> chunks;
  auto make_chunks = [&](const std::vector<int>& nodes) {
    chunks.clear();
    for (int c : nodes)
      for (int st = 0; st < T.num[c]; st += kChunk)
        chunks.push_back(make_int4(c, T.ibeg[c] + st, std::min(kChunk, T.num[c] - st), 0));
  };
  auto upload_chunks = [&]() {
    H.d_chunks.alloc(std::max<size_t>(chunks.size(), 1));
    TABI_CUDA(cudaMemcpyAsync(H.d_chunks.p, chunks.data(), sizeof(int4) * chunks.size(),
                              cudaMemcpyHostToDevice, s));
  };
  // root bounding box (SETUP :120-125)
  {
    std::vector<int> lvl = {0};
    make_chunks(lvl);
    upload_chunks();
    { TABI_K(K_TREE, s); bbox_init_kernel<<<1, 32, 0, s>>>(bb.p, 0, 1); }
    { TABI_K(K_TREE, s); bbox_kernel<<<(int)chunks.size(), kBT, 0, s>>>(H.d_chunks.p, H.d_x.p, H.d_y.p, H.d_z.p,
                                                   bb.p); }
  }
  std::vector<int> hsplit;
  for (int level = 0;; ++level) {
    TABI_REQUIRE(level < 200, TABI_ERR_LIMIT, "tree deeper than 200 levels");
    TABI_CUDA(cudaMemcpyAsync(numd.p + lv0, T.num.data() + lv0, sizeof(int) * (lv1 - lv0),
                              cudaMemcpyHostToDevice, s));
    { TABI_K(K_TREE, s); finalize_kernel<<<ceil_div(lv1 - lv0, 128), 128, 0, s>>>(bb.p, numd.p, lv0, lv1, L, mid.p,
                                                            rad.p, split.p); }
    hsplit.resize(lv1);
    TABI_CUDA(cudaMemcpyAsync(hsplit.data() + lv0, split.p + lv0, sizeof(int) * (lv1 - lv0),
                              cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
    std::vector<int> splitting;
    for (int c = lv0; c < lv1; ++c) {
      if (hsplit[c] & 8)
        throw Error(TABI_ERR_ARG, "more than maxparnode coincident face centroids");
      if (T.num[c] > L) splitting.push_back(c);
    }
    if (splitting.empty()) break;
    make_chunks(splitting);
    upload_chunks();
    int nch = (int)chunks.size();
    H.d_hist.alloc(8 * (size_t)nch);
    H.d_base.alloc(8 * (size_t)nch);
    { TABI_K(K_TREE, s); code_kernel<<<nch, kBT, 0, s>>>(H.d_chunks.p, H.d_x.p, H.d_y.p, H.d_z.p, mid.p, split.p,
                                    H.d_code.p, H.d_hist.p); }
    std::vector<int> hist(8 * (size_t)nch), base(8 * (size_t)nch);
    TABI_CUDA(cudaMemcpyAsync(hist.data(), H.d_hist.p, sizeof(int) * hist.size(),
                              cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
    // child ranges: per node, code-major then chunk order
    int nxt0 = (int)T.ibeg.size();
    size_t ci = 0;
    for (int c : splitting) {
      size_t c0 = ci;
      while (ci < chunks.size() && chunks[ci].x == c) ++ci;
      int cnt[8] = {0};
      for (size_t k = c0; k < ci; ++k)
        for (int b = 0; b < 8; ++b) cnt[b] += hist[8 * k + b];
      // Array layout of the reference's PARTITION_8: each split halves the
      // ranges made by the previous one, so the FIRST split dimension is the
      // most significant in position, while children are numbered (and
      // visited) with it as the least significant bit.
      int nbits = ((hsplit[c] >> 0) & 1) + ((hsplit[c] >> 1) & 1) + ((hsplit[c] >> 2) & 1);
      int start[8] = {0};
      int off = T.ibeg[c];
      for (int k = 0; k < (1 << nbits); ++k) {
        int b = 0;
        for (int q = 0; q < nbits; ++q) b |= ((k >> q) & 1) << (nbits - 1 - q);
        start[b] = off;
        off += cnt[b];
      }
      int first_child = (int)T.ibeg.size();
      int nkids = 0;
      for (int b = 0; b < 8; ++b) {
        int run = start[b];
        for (size_t k = c0; k < ci; ++k) {
          base[8 * k + b] = run;
          run += hist[8 * k + b];
        }
        if (cnt[b] > 0) {
          T.ibeg.push_back(start[b]);
          T.num.push_back(cnt[b]);
          T.level.push_back(level + 1);
          T.child0.push_back(0);
          T.nchild.push_back(0);
          ++nkids;
        }
      }
      T.child0[c] = first_child;
      T.nchild[c] = nkids;
    }
    int nxt1 = (int)T.ibeg.size();
    TABI_CUDA(cudaMemcpyAsync(H.d_base.p, base.data(), sizeof(int) * base.size(),
                              cudaMemcpyHostToDevice, s));
    { TABI_K(K_TREE, s); scatter_kernel<<<nch, kBT, 0, s>>>(H.d_chunks.p, H.d_base.p, H.d_code.p, H.d_x.p, H.d_y.p,
                                       H.d_z.p, H.d_perm.p, H.d_tx.p, H.d_ty.p, H.d_tz.p,
                                       H.d_tperm.p); }
    { TABI_K(K_TREE, s); copy_back_kernel<<<nch, kBT, 0, s>>>(H.d_chunks.p, H.d_tx.p, H.d_ty.p, H.d_tz.p,
                                         H.d_tperm.p, H.d_x.p, H.d_y.p, H.d_z.p, H.d_perm.p); }
    // bounding boxes of the new level
    ensure(nxt1);
    std::vector<int> kids(nxt1 - nxt0);
    std::iota(kids.begin(), kids.end(), nxt0);
    make_chunks(kids);
    upload_chunks();
    { TABI_K(K_TREE, s); bbox_init_kernel<<<ceil_div(nxt1 - nxt0, 128), 128, 0, s>>>(bb.p, nxt0, nxt1); }
    { TABI_K(K_TREE, s); bbox_kernel<<<(int)chunks.size(), kBT, 0, s>>>(H.d_chunks.p, H.d_x.p, H.d_y.p, H.d_z.p,
                                                   bb.p); }
    lv0 = nxt0;
    lv1 = nxt1;
    T.depth = level + 1;
  }
  T.nnodes = (int)T.ibeg.size();
  T.mid.resize(3 * (size_t)T.nnodes);
  T.rad.resize(T.nnodes);
  TABI_CUDA(cudaMemcpyAsync(T.mid.data(), mid.p, sizeof(double) * 3 * T.nnodes,
                            cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(T.rad.data(), rad.p, sizeof(double) * T.nnodes,
                            cudaMemcpyDeviceToHost, s));
  // device node table
  T.d_ibeg.alloc(T.nnodes);
  T.d_num.alloc(T.nnodes);
  T.d_child0.alloc(T.nnodes);
  T.d_nchild.alloc(T.nnodes);
  T.d_mid.alloc(3 * (size_t)T.nnodes);
  T.d_rad.alloc(T.nnodes);
  TABI_CUDA(cudaMemcpyAsync(T.d_ibeg.p, T.ibeg.data(), sizeof(int) * T.nnodes,
                            cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(T.d_num.p, T.num.data(), sizeof(int) * T.nnodes,
                            cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(T.d_child0.p, T.child0.data(), sizeof(int) * T.nnodes,
                            cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(T.d_nchild.p, T.nchild.data(), sizeof(int) * T.nnodes,
                            cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(T.d_mid.p, mid.p, sizeof(double) * 3 * T.nnodes,
                            cudaMemcpyDeviceToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(T.d_rad.p, rad.p, sizeof(double) * T.nnodes,
                            cudaMemcpyDeviceToDevice, s));
  // leaves in tree order
  for (int c = 0; c < T.nnodes; ++c)
    if (T.nchild[c] == 0) T.leaves.push_back(c);
  std::sort(T.leaves.begin(), T.leaves.end(),
            [&](int a, int b) { return T.ibeg[a] < T.ibeg[b]; });
  T.nleaf = (int)T.leaves.size();
  for (int c : T.leaves) T.max_leaf = std::max(T.max_leaf, T.num[c]);
  // permute normals and areas into tree order
  H.d_tx.alloc(n);
  H.d_ty.alloc(n);
  H.d_tz.alloc(n);
  DBuf<double>& tarea = H.tb_tmp;
  tarea.alloc(n);
  { TABI_K(K_TREE, s); gather4_kernel<<<ceil_div(n, 256), 256, 0, s>>>(H.d_perm.p, n, H.d_nx.p, H.d_ny.p, H.d_nz.p,
                                                  H.d_area.p, H.d_tx.p, H.d_ty.p, H.d_tz.p,
                                                  tarea.p); }
  TABI_CUDA(cudaMemcpyAsync(H.d_nx.p, H.d_tx.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(H.d_ny.p, H.d_ty.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(H.d_nz.p, H.d_tz.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(H.d_area.p, tarea.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  H.h_perm.resize(n);
  TABI_CUDA(cudaMemcpyAsync(H.h_perm.data(), H.d_perm.p, sizeof(int) * n,
                            cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
}

void build_lists(Handle& H, cudaStream_t s) {
  Tree& T = H.tree;
  const int n = H.n;
  const int nn = T.nnodes;
  DBuf<int>& tgt_cnt = H.ls_tgt;
  DBuf<int>& far_cnt = H.ls_far;
  DBuf<int>& near_cnt = H.ls_near;
  tgt_cnt.alloc(n);
  far_cnt.alloc(nn);
  near_cnt.alloc(nn);
  TABI_CUDA(cudaMemsetAsync(far_cnt.p, 0, sizeof(int) * nn, s));
  TABI_CUDA(cudaMemsetAsync(near_cnt.p, 0, sizeof(int) * nn, s));
  TABI_CUDA(cudaMemsetAsync(H.d_err.p, 0, sizeof(int), s));
  int nwarps = ceil_div(n, 32);
  int grid = ceil_div(nwarps, kTW);
  { TABI_K(K_LISTS, s); traverse_kernel<false><<<grid, 32 * kTW, 0, s>>>(
      H.d_x.p, H.d_y.p, H.d_z.p, n, T.d_num.p, T.d_child0.p, T.d_nchild.p, T.d_mid.p,
      T.d_rad.p, H.prm.theta, tgt_cnt.p, far_cnt.p, near_cnt.p, nullptr, nullptr, nullptr,
      nullptr, nullptr, nullptr, nullptr, H.d_err.p); }
  // per-target slot offsets (device scan)
  T.d_slot_off.alloc((size_t)n + 1);
  int nb = ceil_div(n, kScanB);
  DBuf<int64_t>& bsum = H.ls_bsum;
  bsum.alloc((size_t)nb + 1);
  { TABI_K(K_LISTS, s); scan_block_kernel<<<nb, kScanB, 0, s>>>(tgt_cnt.p, n, T.d_slot_off.p, bsum.p); }
  { TABI_K(K_LISTS, s); scan_top_kernel<<<1, 32, 0, s>>>(bsum.p, nb); }
  { TABI_K(K_LISTS, s); scan_add_kernel<<<nb, kScanB, 0, s>>>(T.d_slot_off.p, n, bsum.p); }
  std::vector<int> hf(nn), hn(nn);
  int herr = 0;
  TABI_CUDA(cudaMemcpyAsync(hf.data(), far_cnt.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(hn.data(), near_cnt.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(&herr, H.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaMemcpyAsync(&T.n_slots, T.d_slot_off.p + n, sizeof(int64_t),
                            cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  TABI_REQUIRE(herr == 0, TABI_ERR_LIMIT, "tree traversal stack overflow");
  std::vector<int64_t> foff(nn), noff(nn);
  int64_t tf = 0, tn = 0, pairs = 0;
  for (int c = 0; c < nn; ++c) {
    foff[c] = tf;
    noff[c] = tn;
    tf += hf[c];
    tn += hn[c];
    pairs += (int64_t)hn[c] * T.num[c];
  }
  T.n_far = tf;
  T.n_near_pairs = pairs - n;  // every target meets its own leaf once
  TABI_REQUIRE(T.n_slots == tf + tn, TABI_ERR_CUDA, "interaction count mismatch");
  TABI_REQUIRE(T.n_slots < (1LL << 31), TABI_ERR_LIMIT, "more than 2^31 interactions");
  DBuf<int64_t>& d_foff = H.ls_foff;
  DBuf<int64_t>& d_noff = H.ls_noff;
  d_foff.alloc(nn);
  d_noff.alloc(nn);
  TABI_CUDA(cudaMemcpyAsync(d_foff.p, foff.data(), sizeof(int64_t) * nn,
                            cudaMemcpyHostToDevice, s));
  TABI_CUDA(cudaMemcpyAsync(d_noff.p, noff.data(), sizeof(int64_t) * nn,
                            cudaMemcpyHostToDevice, s));
  T.d_far_ent.alloc(std::max<int64_t>(tf, 1));
  T.d_near_ent.alloc(std::max<int64_t>(tn, 1));
  TABI_CUDA(cudaMemsetAsync(far_cnt.p, 0, sizeof(int) * nn, s));
  TABI_CUDA(cudaMemsetAsync(near_cnt.p, 0, sizeof(int) * nn, s));
  { TABI_K(K_LISTS, s); traverse_kernel<true><<<grid, 32 * kTW, 0, s>>>(
      H.d_x.p, H.d_y.p, H.d_z.p, n, T.d_num.p, T.d_child0.p, T.d_nchild.p, T.d_mid.p,
      T.d_rad.p, H.prm.theta, nullptr, nullptr, nullptr, T.d_slot_off.p, d_foff.p, d_noff.p,
      far_cnt.p, near_cnt.p, T.d_far_ent.p, T.d_near_ent.p, H.d_err.p); }
  // work items and moment slots
  const int kFarChunk = 64, kNearChunk = 128, kMomChunk = 256;
  T.far_work.clear();
  T.near_work.clear();
  T.mslot_node.clear();
  T.mchunk_node.clear();
  T.mslot_chunk0.clear();
  T.mslot_nchunk.clear();
  std::vector<int4> mch;
  for (int c = 0; c < nn; ++c) {
    if (hf[c] > 0) {
      int slot = (int)T.mslot_node.size();
      T.mslot_node.push_back(c);
      T.mslot_chunk0.push_back((int)mch.size());
      for (int st = 0; st < T.num[c]; st += kMomChunk)
        mch.push_back(make_int4(slot, T.ibeg[c] + st, std::min(kMomChunk, T.num[c] - st),
                                (int)mch.size()));
      T.mslot_nchunk.push_back((int)mch.size() - T.mslot_chunk0.back());
      for (int st = 0; st < hf[c]; st += kFarChunk)
        T.far_work.push_back({c, (int)(foff[c] + st), std::min(kFarChunk, hf[c] - st), slot});
    }
    if (hn[c] > 0)
      for (int st = 0; st < hn[c]; st += kNearChunk)
        T.near_work.push_back({c, (int)(noff[c] + st), std::min(kNearChunk, hn[c] - st),
                               T.ibeg[c]});
  }
  T.nmslot = (int)T.mslot_node.size();
  T.d_far_work.alloc(std::max<size_t>(T.far_work.size(), 1));
  T.d_near_work.alloc(std::max<size_t>(T.near_work.size(), 1));
  T.d_mchunks.alloc(std::max<size_t>(mch.size(), 1));
  std::vector<int2> msc(T.nmslot);
  for (int k = 0; k < T.nmslot; ++k) msc[k] = make_int2(T.mslot_chunk0[k], T.mslot_nchunk[k]);
  T.d_mslot_chunks.alloc(std::max(T.nmslot, 1));
  T.d_mslot_node.alloc(std::max(T.nmslot, 1));
  T.far_work.upload(T.d_far_work, s);
  T.near_work.upload(T.d_near_work, s);
  if (!mch.empty())
    TABI_CUDA(cudaMemcpyAsync(T.d_mchunks.p, mch.data(), sizeof(int4) * mch.size(),
                              cudaMemcpyHostToDevice, s));
  if (T.nmslot) {
    TABI_CUDA(cudaMemcpyAsync(T.d_mslot_chunks.p, msc.data(), sizeof(int2) * T.nmslot,
                              cudaMemcpyHostToDevice, s));
    TABI_CUDA(cudaMemcpyAsync(T.d_mslot_node.p, T.mslot_node.data(), sizeof(int) * T.nmslot,
                              cudaMemcpyHostToDevice, s));
  }
  TABI_CUDA(cudaMemcpyAsync(&herr, H.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TABI_CUDA(cudaStreamSynchronize(s));
  TABI_REQUIRE(herr == 0, TABI_ERR_LIMIT, "tree traversal stack overflow");
  // scratch sized for the lists
  H.d_res.alloc(std::max<int64_t>(T.n_slots, 1));
  H.d_mraw.alloc(std::max<size_t>(mch.size(), 1) * 4 * 165);
  H.d_mw.alloc(std::max(T.nmslot, 1) * (size_t)16 * 165);
}

}  // namespace tabi
