// tabi_impl.cuh -- internal state and kernel declarations of libtabi_gpu.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/tabi_gpu.h"

namespace tabi {

constexpr double kPi = 3.141592653589793238462643383279;
constexpr double kOneOver4Pi = 0.25 / 3.141592653589793238462643383279;
constexpr int kMaxOrder = 8;
constexpr int kMacMinPar = 40;   // treecode3d_pb.f:393 (numpar > 40)
constexpr int kStack = 512;      // per-warp traversal stack entries

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define TABI_CUDA(call)                                                     \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      throw ::tabi::Error(e_ == cudaErrorMemoryAllocation ? TABI_ERR_NOMEM  \
                                                          : TABI_ERR_CUDA,  \
                          std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TABI_REQUIRE(cond, code, msg)                   \
  do {                                                  \
    if (!(cond)) throw ::tabi::Error((code), (msg));    \
  } while (0)

// Device buffer owned by the handle (freed on reset / destroy).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  // Grows only.  A buffer that has to grow again gets 1.5x the request: every
  // cudaFree synchronises the whole device, which stalls the other handles'
  // work (batch workers share the GPU), so regrowth should be rare.
  void alloc(size_t count) {
    if (count <= n && p) return;
    const bool regrow = p != nullptr;
    release();
    if (count == 0) return;
    if (regrow) count += count / 2;
    TABI_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
};

// Page-locked host staging vector owned by the handle: host tables built per
// solve (launch plans, offsets) are written here and copied to the device
// asynchronously.  A copy from pageable memory may wait for the stream's
// earlier work before it returns, which kept the host from planning while the
// GPU ran; from page-locked memory the copy returns at once.  `upload`
// records an event after the copy and `restart` waits for it, so the contents
// are never rewritten under a pending copy.  Grows only (by doubling, keeping
// the contents); freeing page-locked memory synchronises the device, so
// growth should be rare.
template <typename T>
struct PinVec {
  T* p = nullptr;
  size_t len = 0, cap = 0;
  cudaEvent_t done = nullptr;
  // starts a new fill (after the last copy out of the buffer has finished)
  void restart() {
    if (done) cudaEventSynchronize(done);
    len = 0;
  }
  // a few std::vector names, for host lists kept on the host as well
  void clear() { restart(); }
  void push_back(const T& v) { push(v); }
  size_t size() const { return len; }
  bool empty() const { return len == 0; }
  T* data() { return p; }
  const T* data() const { return p; }
  const T* begin() const { return p; }
  const T* end() const { return p + len; }
  void grow(size_t need) {
    const size_t nc = std::max<size_t>(std::max<size_t>(need, 2 * cap), 256);
    T* q = nullptr;
    TABI_CUDA(cudaMallocHost(&q, nc * sizeof(T)));
    if (len) std::memcpy(q, p, len * sizeof(T));
    if (p) cudaFreeHost(p);
    p = q;
    cap = nc;
  }
  void push(const T& v) {
    if (__builtin_expect(len == cap, 0)) grow(len + 1);
    p[len++] = v;
  }
  void assign(const T* src, size_t n) {
    restart();
    if (n > cap) grow(n);
    if (n) std::memcpy(p, src, n * sizeof(T));
    len = n;
  }
  // the contents to dst (grown to at least one element) on stream s
  void upload(DBuf<T>& dst, cudaStream_t s) {
    dst.alloc(std::max<size_t>(len, 1));
    if (len)
      TABI_CUDA(cudaMemcpyAsync(dst.p, p, sizeof(T) * len, cudaMemcpyHostToDevice, s));
    if (!done) TABI_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    TABI_CUDA(cudaEventRecord(done, s));
  }
  ~PinVec() {
    if (done) {
      cudaEventSynchronize(done);
      cudaEventDestroy(done);
    }
    if (p) cudaFreeHost(p);
  }
  PinVec() = default;
  PinVec(const PinVec&) = delete;
  PinVec& operator=(const PinVec&) = delete;
};

// Work item of the interaction kernels: node and a chunk of its entry list.
struct WorkItem {
  int node;
  int start;  // offset into the node's entry list
  int count;
  int mslot;  // moment slot (far) or leaf ibeg (near)
};

struct Tree {
  // Clears the host-side description; device buffers are kept and reused
  // (they only ever grow), so rebuilding a tree allocates nothing once the
  // sizes have been seen.
  void clear() {
    n = nnodes = nleaf = depth = 0;
    ibeg.clear(); num.clear(); child0.clear(); nchild.clear(); level.clear();
    mid.clear(); rad.clear(); leaves.clear();
    n_near_pairs = n_far = n_slots = 0;
    far_work.clear(); near_work.clear();
    nmslot = 0;
    mslot_node.clear(); mslot_chunk0.clear(); mslot_nchunk.clear();
    blk_off.clear();
    dinv_off.clear();
    n_solve_big = n_solve_small = 0;
    max_leaf = 0;
    lrel_ready = false;
    ranged = false;
    r_far_work.clear();
    r_near_work.clear();
  }
  int n = 0;          // faces
  int nnodes = 0;
  int nleaf = 0;
  int depth = 0;
  // host mirror of the node table (BFS order: children of a node contiguous)
  std::vector<int> ibeg, num, child0, nchild, level;
  std::vector<double> mid, rad;  // mid 3 per node
  std::vector<int> leaves;       // leaf node ids in tree order
  // device node table
  DBuf<int> d_ibeg, d_num, d_child0, d_nchild;
  DBuf<double> d_mid, d_rad;
  // interaction lists
  int64_t n_near_pairs = 0, n_far = 0, n_slots = 0;
  DBuf<int64_t> d_slot_off;    // n+1
  DBuf<int2> d_far_ent;        // (target, slot) grouped by cluster
  DBuf<int2> d_near_ent;       // (target, slot) grouped by leaf
  PinVec<WorkItem> far_work, near_work;  // page-locked: uploaded per tree
  DBuf<WorkItem> d_far_work, d_near_work;
  int nmslot = 0;
  std::vector<int> mslot_node;  // node id per moment slot
  DBuf<int> d_mslot_node;
  std::vector<int> mchunk_node, mchunk_start, mchunk_count;  // moment chunks
  DBuf<int4> d_mchunks;  // (slot, node ibeg+start, count, chunk id)
  std::vector<int> mslot_chunk0, mslot_nchunk;
  DBuf<int2> d_mslot_chunks;
  // preconditioner
  std::vector<int64_t> blk_off;  // per leaf offset into the factor buffer
  DBuf<double> d_lu;
  DBuf<int> d_piv;               // 2n per leaf, offsets 2*ibeg
  DBuf<int64_t> d_blk_off;
  DBuf<int2> d_leaf_rng;         // (ibeg, n) per leaf
  DBuf<int> d_solve_list;        // leaves of the apply launches (big ones first)
  std::vector<int64_t> dinv_off;  // per leaf offset of its inverse diagonal blocks
  DBuf<int64_t> d_dinv_off;
  DBuf<double> d_dinv;           // per 32-row block: L^{-1}, U^{-1} (32 x 32 each)
  DBuf<int> d_lu_perm;           // per leaf row permutation of all pivots
  int n_solve_big = 0, n_solve_small = 0;
  int max_leaf = 0;
  // mixed precision: leaf ids on the device; each face relative to its leaf
  // centre as FP32 hi + lo (with its area in lpos.w) and its normal in FP32
  // (built on first use)
  DBuf<int> d_leaves;
  DBuf<float4> d_lpos, d_llo, d_lnrm;
  bool lrel_ready = false;
  // a shard's target range (tabi_set_target_range): the interaction lists
  // restricted to targets [rt0, rt1) and the leaves inside it
  bool ranged = false;
  int rt0 = 0, rt1 = 0;
  std::vector<WorkItem> r_far_work, r_near_work;
  DBuf<WorkItem> d_r_far_work, d_r_near_work;
  DBuf<int2> d_r_far_ent, d_r_near_ent;
  DBuf<int> d_r_solve_list;
  int r_solve_big = 0, r_solve_small = 0;
};

// Kernel classes for the launch counters / event timers (tabi_profile_*).
enum KClass {
  K_FORM = 0, K_TREE, K_LISTS, K_MOMENTS, K_FAR, K_NEAR, K_REDUCE, K_ASSEMBLE, K_LU,
  K_SOLVE, K_VEC, K_ENERGY, K_LU_UPDATE, K_LU_POST, K_LU_STRIP, K_LU_SWAP,
  K_PHASE_MATVEC,  // whole treecode matvec (a phase: timed, not a launch)
  K_PHASE_LU,      // the leaf-block factorisation, first LU launch to the join of both streams
  K_PHASE_APPLY,   // one preconditioner apply, fork to join
  K_NCLASS
};

struct Handle;

struct Prof {
  bool on = false;
  int64_t launches[K_NCLASS] = {};
  double ms[K_NCLASS] = {};
  struct Rec {
    cudaEvent_t a, b;
    int kind;
  };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  void resolve() {
    for (auto& r : pending) {
      float f = 0.f;
      cudaEventSynchronize(r.b);
      cudaEventElapsedTime(&f, r.a, r.b);
      ms[r.kind] += f;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
  void reset() {
    resolve();
    for (int k = 0; k < K_NCLASS; ++k) {
      launches[k] = 0;
      ms[k] = 0.0;
    }
  }
  ~Prof() {
    for (auto& r : pending) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

// Counts one kernel launch of class `kind` and, when profiling is on, times
// it with events recorded on the launching stream around the launch.
struct KScope {
  Prof& P;
  int kind;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  KScope(Prof& p, int k, cudaStream_t st) : P(p), kind(k), s(st) {
    P.launches[kind]++;  // for a phase class: the number of times it ran
    if (P.on) {
      a = P.get();
      cudaEventRecord(a, s);
    }
  }
  ~KScope() {
    if (P.on) {
      cudaEvent_t b = P.get();
      cudaEventRecord(b, s);
      P.pending.push_back({a, b, kind});
    }
  }
};
#define TABI_K(kind, s) ::tabi::KScope _kscope_(H.prof, (kind), (s))
#define TABI_PHASE(kind, s) ::tabi::KScope _pscope_(H.prof, (kind), (s))

struct Handle {
  tabi_params prm{};
  Prof prof;
  std::string err;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;           // second stream of the matvec (near field)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Streams of the leaf LU, forked from the caller's stream and joined back:
  // the large-block group's chain at the highest priority; the trailing
  // updates' columns beyond the next outer block (throughput work beside the
  // chain) and the small-block group below it, so that the block scheduler
  // gives freed SMs to the chain first.
  cudaStream_t lu_hi = nullptr, lu_small = nullptr, aux = nullptr;
  // the leaf factorisation's phase timer, from its first launch
  // (build_precond) to the join of its streams (finish_precond)
  std::optional<KScope> pc_lu_phase;
  // the exchange of a target-sharded solve (tabi_set_exchange)
  tabi_exchange_fn xchg = nullptr;
  void* xchg_user = nullptr;
  cudaEvent_t ev_la = nullptr, ev_rest = nullptr, ev_lu_join = nullptr;
  int device = 0;
  int n = 0;  // faces
  bool has_surface = false, has_tree = false, has_precond = false;
  // surface in the handle's current order (original before the tree, tree
  // order after)
  DBuf<double> d_x, d_y, d_z, d_nx, d_ny, d_nz, d_area;
  DBuf<int> d_perm;  // tree slot -> original index
  std::vector<int> h_perm;
  Tree tree;
  // matvec scratch
  DBuf<double> d_mraw;    // moment partials
  DBuf<double> d_mw;      // weighted moments, 16 x NT per slot
  DBuf<float> d_mwf;      // the same in FP32 (mixed-precision far field)
  int mv_prec = TABI_PREC_FP64;  // arithmetic of the treecode operator
  DBuf<double2> d_res;    // per-slot interaction results
  DBuf<double2> d_dirpart;  // direct-sum partials (accuracy reference)
  DBuf<double> d_red;     // reduction scratch
  DBuf<double> h_red_pinned_dummy;
  double* h_pinned = nullptr;  // small pinned host scratch (64 doubles)
  // GMRES workspace
  DBuf<double> d_v, d_wk, d_dl, d_gz, d_r, d_b, d_xio, d_tmp;
  DBuf<double> d_coef, d_orth;
  DBuf<double> d_ir_r, d_ir_d, d_ir_t;  // mixed-precision refinement
  // energy scratch
  DBuf<double> d_ptl;
  DBuf<double> d_atoms;
  // tree-build scratch
  DBuf<double> d_tx, d_ty, d_tz;
  DBuf<int> d_tperm;
  DBuf<unsigned char> d_code;
  DBuf<unsigned long long> d_bbox;
  DBuf<int> d_hist, d_base;
  DBuf<int4> d_chunks;
  DBuf<int> d_cnt;
  DBuf<int> d_err;
  // persistent workspaces of the build steps (grow-only)
  DBuf<unsigned long long> tb_bb;
  DBuf<double> tb_mid, tb_rad, tb_tmp;
  DBuf<int> tb_split, tb_num;
  DBuf<int> ls_tgt, ls_far, ls_near;
  DBuf<int64_t> ls_bsum, ls_foff, ls_noff;
  DBuf<int2> pc_tiles;
  DBuf<int> pc_info;
  // one LU plan per leaf group (large blocks on the handle's stream, small
  // ones on its side stream): panel leaves, strip / gemm / row-swap items,
  // swap-map leaves and maps
  struct LuPlan {
    DBuf<int> list, mleaves, map;
    DBuf<int4> items, gitems, ritems;
  } pc_plan[2];
  // the unpivoted factorisation: per group, the diagonal kernels' leaves per
  // step, panel and update items, and the inverses of the step's diagonal
  // blocks; per leaf a failed-certificate flag
  struct NpPlan {
    DBuf<int> dleaves;
    DBuf<int4> pitems, gitems;
    DBuf<double> scr;
    PinVec<int> h_dleaves;  // page-locked staging of the three item lists
    PinVec<int4> h_pitems, h_gitems;
  } pc_np[2];
  // page-locked staging of the per-tree preconditioner tables
  PinVec<int2> pc_h_tiles, pc_h_rng;
  PinVec<int64_t> pc_h_blk_off, pc_h_dinv_off;
  PinVec<int> pc_h_solve_list;
  DBuf<int> pc_fail, pc_big;
  DBuf<int2> pc_tiles2;
  int pc_pv_leaves = 0;  // leaves of the last tree factored with pivoting
  DBuf<int2> pc_dblocks;
  // staging of the host-array entry points and of tabi_run_dev
  DBuf<double> st_pos, st_nrm, st_cp, st_q, st_b, st_axyz, st_aq, st_x;
  DBuf<int> st_fv;
  DBuf<double> rn_b0, rn_b, rn_x, rn_z;
  // device face filter
  DBuf<unsigned char> ff_keep;
  DBuf<int> ff_cnt;
  DBuf<double> ff_area;
  // output_potential
  DBuf<double> vp_cen, vp_xo, vp_vert, vp_pos;
  DBuf<int> vp_cnt, vp_off, vp_list, vp_err, vp_scan, vp_nv;
};

// ---- kernels / launchers (defined in the .cu files) ----
// form_matrix / rhs / energy (rhs_energy.cu)
void launch_form_matrix(Handle& H, int nspt, const double* sptpos, const double* sptnrm,
                        int nface, const int* nvert, int nchr, const double* atoms4,
                        double* d_b, cudaStream_t s);
void launch_rhs(Handle& H, int nchr, const double* atoms4, double* d_b, cudaStream_t s);
// readin.f90:264-333 surface_area on device arrays: nvert_out (3 x nface
// capacity) receives the kept faces in order; *nkept and *s_area on the host
void face_filter_dev(Handle& H, int nspt, const double* sptpos, int nface, const int* nvert,
                     int* nvert_out, int* nkept, double* s_area, cudaStream_t s);
void energy_dev(Handle& H, int nchr, const double* chrpos, const double* atmchr, const double* x,
                double* soleng, double* couleng, cudaStream_t s);
// tree + lists (tree.cu)
void build_tree(Handle& H, cudaStream_t s);
void build_lists(Handle& H, cudaStream_t s);
// matvec (matvec.cu)
void matvec_dev(Handle& H, const double* x, double* y, cudaStream_t s, bool check_zero);
// restricts matvec_dev / msolve_dev to the leaf-aligned target range [t0, t1)
// of the tree order (the whole range lifts the restriction)
void set_target_range(Handle& H, int t0, int t1, cudaStream_t s);
// FP64 direct sum of the operator at nt targets (current face order): y is
// [y1 of the targets; y2 of the targets] (2 nt)
void direct_targets_dev(Handle& H, int nt, const int* targets, const double* x, double* y,
                        cudaStream_t s);
double asum_dev(Handle& H, const double* x, int n, cudaStream_t s);
// preconditioner (precond.cu)
// The leaf-block preconditioner in two halves: build_precond assembles the
// blocks and launches the factorisation on the handle's LU streams (which
// only need the tree); finish_precond joins them into s, reads the
// certificates and factors the failed leaves with partial pivoting.  The
// interaction lists are built in between, on s, beside the factorisation.
void build_precond(Handle& H, cudaStream_t s);
void finish_precond(Handle& H, cudaStream_t s);
void msolve_dev(Handle& H, const double* r, double* z, cudaStream_t s);
// output_potential (potential.cu): x in tree order -> x_orig (2 n, original
// face order) and vert_ptl (2 per vertex), both scaled by 332.0716 * 4 pi
void output_potential_dev(Handle& H, int nspt, const double* sptpos, int nface, const int* nvert,
                          const double* x, double* x_orig, double* vert_ptl, cudaStream_t s);
// gmres (gmres.cu)
// minv_b (may be null): M^-1 b already formed (device, 2n) and its norm
void gmres_dev(Handle& H, const double* b, double* x, int* iter, double* err, int* ierr,
               double* hist, int* nhist, cudaStream_t s, double tol = -1.0,
               const double* minv_b = nullptr, double minv_b_nrm = 0.0);
// the solve the handle's precision asks for: gmres_dev (FP64) or FP64 GMRES-IR
// around FP32-operator GMRES (mixed)
void solve_dev(Handle& H, const double* b, double* x, int* iter, double* err, int* ierr,
               double* hist, int* nhist, cudaStream_t s);
double dot_dev(Handle& H, const double* a, const double* b, int n, cudaStream_t s);
double nrm2_dev(Handle& H, const double* a, int n, cudaStream_t s);

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// Raises a kernel's dynamic shared memory limit on the current device to at
// least `bytes` (never lowers it).  The limit is process-wide state of the
// kernel, so handles solving on several host threads must not set it to their
// own molecule's need: one thread could lower it under another's launch.
inline void raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> high;
  int dev = 0;
  TABI_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t& h = high[{func, dev}];
  if (bytes <= h) return;
  TABI_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  h = bytes;
}

// Programmatic dependent launch for chains of dependent kernels on one stream
// (the leaf LU's diagonal, panel and update launches).  A kernel launched by
// launch_chained may be scheduled while the kernel before it in the stream is
// still running, once every CTA of that kernel has started and signalled
// (chain_signal); it must call chain_wait before it reads anything the
// earlier kernel writes.  chain_wait blocks until the earlier grid has
// completed and its memory operations are visible, so the launch latency
// between the two kernels overlaps the earlier one's tail.  In a kernel
// launched the ordinary way, or after a non-kernel operation in the stream,
// both are no-ops.
__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void chain_signal() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// `chain` false launches the ordinary way: used for the first kernel after a
// copy, an event record or a wait on another stream, so that such an
// operation is never overtaken.
template <typename... KArgs, typename... Args>
void launch_chained(bool chain, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                    cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = chain ? 1 : 0;
  TABI_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

}  // namespace tabi
