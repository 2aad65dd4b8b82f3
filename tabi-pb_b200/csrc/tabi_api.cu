// tabi_api.cu -- the C ABI (include/tabi_gpu.h): argument checks, host <-> device
// staging, and the order of the steps main.f90 performs.
#include <algorithm>
#include <chrono>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <memory>
#include <thread>
#include <vector>

#include "tabi_impl.cuh"
#include "warmstart.cuh"

namespace tabi {
void pack_atoms_dev(Handle& H, int nchr, const double* chrpos_dev, const double* atmchr_dev,
                    cudaStream_t s);
void energy_noalloc(int nface, const double* tr_xyz, const double* tr_q, const double* tr_area,
                    const double* x, int nchr, const double* chrpos, const double* atmchr,
                    double kappa, double eps0, double eps1, double* out, cudaStream_t s);
}

using namespace tabi;

struct tabi_handle_s {
  Handle H;
  WsNet* ws = nullptr;  // attached warm-start network (not owned)
};

struct tabi_ws_s {
  WsNet* net = nullptr;
};

namespace {

thread_local std::string g_err;

template <typename F>
int guarded(tabi_h h, F&& f) {
  try {
    f();
    if (h) h->H.err.clear();
    return TABI_OK;
  } catch (const Error& e) {
    if (h) h->H.err = e.what();
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    if (h) h->H.err = "host allocation failed";
    g_err = "host allocation failed";
    return TABI_ERR_NOMEM;
  } catch (const std::exception& e) {
    if (h) h->H.err = e.what();
    g_err = e.what();
    return TABI_ERR_CUDA;
  }
}

cudaStream_t pick(Handle& H, void* stream) {
  return stream ? (cudaStream_t)stream : H.stream;
}

void set_device(Handle& H) { TABI_CUDA(cudaSetDevice(H.device)); }

void alloc_surface(Handle& H, int n) {
  H.n = n;
  H.d_x.alloc(n);
  H.d_y.alloc(n);
  H.d_z.alloc(n);
  H.d_nx.alloc(n);
  H.d_ny.alloc(n);
  H.d_nz.alloc(n);
  H.d_area.alloc(n);
  H.has_surface = H.has_tree = H.has_precond = false;
}

__global__ void soa_from_aos_kernel(const double* xyz, const double* q, const double* area, int n,
                                    double* x, double* y, double* z, double* nx, double* ny,
                                    double* nz, double* a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = xyz[3 * (size_t)i];
  y[i] = xyz[3 * (size_t)i + 1];
  z[i] = xyz[3 * (size_t)i + 2];
  nx[i] = q[3 * (size_t)i];
  ny[i] = q[3 * (size_t)i + 1];
  nz[i] = q[3 * (size_t)i + 2];
  a[i] = area[i];
}

__global__ void aos_from_soa_kernel(const double* x, const double* y, const double* z,
                                    const double* nx, const double* ny, const double* nz, int n,
                                    double* xyz, double* q) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xyz[3 * (size_t)i] = x[i];
  xyz[3 * (size_t)i + 1] = y[i];
  xyz[3 * (size_t)i + 2] = z[i];
  q[3 * (size_t)i] = nx[i];
  q[3 * (size_t)i + 1] = ny[i];
  q[3 * (size_t)i + 2] = nz[i];
}

__global__ void permute_b_kernel(const int* perm, int n, const double* b, double* tb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int o = perm[i];
  tb[i] = b[o];
  tb[n + i] = b[n + o];
}

// FMA peak probe: eight independent chains per thread (T = double or float)
template <typename T>
__global__ void fma_peak_kernel(T* out, long iters) {
  T a0 = threadIdx.x * T(1e-9), a1 = a0 + T(1e-9), a2 = a0 + T(2e-9), a3 = a0 + T(3e-9);
  T a4 = a0 + T(4e-9), a5 = a0 + T(5e-9), a6 = a0 + T(6e-9), a7 = a0 + T(7e-9);
  const T m = T(0.999999), c = T(1e-7);
  for (long i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fma(a0, m, c);
      a1 = fma(a1, m, c);
      a2 = fma(a2, m, c);
      a3 = fma(a3, m, c);
      a4 = fma(a4, m, c);
      a5 = fma(a5, m, c);
      a6 = fma(a6, m, c);
      a7 = fma(a7, m, c);
    }
  }
  T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == T(123.456)) out[0] = s;  // keeps the loop alive
}

template <typename T>
int probe_fma_peak(double ms, double* flops) {
  if (!flops) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    int dev = 0, nsm = 0;
    TABI_CUDA(cudaGetDevice(&dev));
    TABI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DBuf<T> out;
    out.alloc(1);
    cudaEvent_t e0, e1;
    TABI_CUDA(cudaEventCreate(&e0));
    TABI_CUDA(cudaEventCreate(&e1));
    int blocks = nsm * 8, threads = 256;
    long iters = 64;
    double t = 0.0;
    for (int rep = 0; rep < 12; ++rep) {
      TABI_CUDA(cudaEventRecord(e0));
      fma_peak_kernel<T><<<blocks, threads>>>(out.p, iters);
      TABI_CUDA(cudaEventRecord(e1));
      TABI_CUDA(cudaEventSynchronize(e1));
      float f = 0;
      TABI_CUDA(cudaEventElapsedTime(&f, e0, e1));
      t = f;
      if (t >= ms) break;
      iters = (long)(iters * std::min(8.0, std::max(1.5, ms / std::max(t, 1e-3))));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double fl = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *flops = fl / (t * 1e-3);
  });
}

void check_params(const tabi_params& p) {
  TABI_REQUIRE(p.order >= 1 && p.order <= kMaxOrder, TABI_ERR_ARG, "order must be in 1..8");
  TABI_REQUIRE(p.maxparnode >= 1, TABI_ERR_ARG, "maxparnode must be >= 1");
  TABI_REQUIRE(p.theta > 0.0 && p.theta < 1.0, TABI_ERR_ARG,
               "theta must be in (0, 1): the self-interaction removal of the reference needs "
               "the MAC to fail on every cluster holding the target");
  TABI_REQUIRE(p.kappa >= 0.0 && std::isfinite(p.kappa), TABI_ERR_ARG, "kappa must be >= 0");
  TABI_REQUIRE(p.eps0 > 0.0 && p.eps1 > 0.0, TABI_ERR_ARG, "dielectrics must be > 0");
  TABI_REQUIRE(p.maxl >= 0 && p.maxl <= 60, TABI_ERR_ARG, "maxl must be in 0..60");
  TABI_REQUIRE(p.nrmax >= -1, TABI_ERR_ARG, "nrmax must be >= -1");
  TABI_REQUIRE(p.tol >= 0.0, TABI_ERR_ARG, "tol must be >= 0");
  TABI_REQUIRE(p.precision == TABI_PREC_FP64 || p.precision == TABI_PREC_MIXED, TABI_ERR_ARG,
               "precision must be TABI_PREC_FP64 or TABI_PREC_MIXED");
  TABI_REQUIRE(p.maxparnode <= 12000, TABI_ERR_LIMIT, "maxparnode above 12000");
  TABI_REQUIRE((p.flags & ~TABI_FLAG_PIVOTED_LU) == 0, TABI_ERR_ARG, "unknown flags");
}

void require_tree(Handle& H, int n2) {
  TABI_REQUIRE(H.has_tree, TABI_ERR_STATE, "tabi_build_tree has not been called");
  TABI_REQUIRE(n2 == 2 * H.n, TABI_ERR_ARG, "vector length must be 2*nface");
}

// After the tree: the leaf factorisation is launched on the handle's LU
// streams first, then the interaction lists are built on s beside it (their
// host round trips and kernels overlap the factorisation), then the
// factorisation is joined and checked.  A tree whose leaf blocks cannot be
// factored (TABI_ERR_SINGULAR), or any failure on the way, leaves the handle
// without a tree, after the LU streams have finished what was launched.
void lists_and_precond(Handle& H, cudaStream_t s, const std::function<void(const char*)>& mark) {
  try {
    build_precond(H, s);
    build_lists(H, s);
    H.has_tree = true;
    mark("lists");
    finish_precond(H, s);
    mark("precond");
  } catch (...) {
    for (cudaStream_t x : {H.lu_hi, H.lu_small, H.aux, H.side, s})
      if (x) cudaStreamSynchronize(x);
    H.pc_lu_phase.reset();
    H.has_tree = H.has_precond = false;
    throw;
  }
}

void do_build(Handle& H, cudaStream_t s) {
  build_tree(H, s);
  lists_and_precond(H, s, [](const char*) {});
}

template <typename T>
void h2d(DBuf<T>& buf, const T* src, size_t n, cudaStream_t s) {
  buf.alloc(std::max<size_t>(n, 1));
  TABI_CUDA(cudaMemcpyAsync(buf.p, src, sizeof(T) * n, cudaMemcpyHostToDevice, s));
}

constexpr int kBatchStats = TABI_BATCH_STATS;

struct MolDev {
  int nspt;
  const double* sptpos;
  const double* sptnrm;
  int nface;
  const int* nvert;
  int nchr;
  const double* chrpos;
  const double* atmchr;
};

template <typename M>
void check_mol(const M& m) {
  TABI_REQUIRE(m.nspt > 0 && m.nface > 0 && m.nchr > 0, TABI_ERR_ARG, "sizes must be positive");
  TABI_REQUIRE(m.sptpos && m.sptnrm && m.nvert && m.chrpos && m.atmchr, TABI_ERR_ARG,
               "null input");
}

// The whole main.f90 sequence for one molecule on device inputs: form_matrix,
// tree, interaction lists, leaf LU, initial guess (zero, or the warm-start
// network's prediction), solve, energy.  x_dev (tree order) may be null.
void run_molecule(Handle& H, WsNet* ws, const MolDev& m, double* x_dev, double* stats,
                  cudaStream_t s) {
  check_mol(m);
  const int nface = m.nface, nchr = m.nchr;
  // TABI_TRACE=1 prints host wall time per phase (synchronising between them)
  static const bool trace = getenv("TABI_TRACE") && getenv("TABI_TRACE")[0] == '1';
  auto t_last = std::chrono::steady_clock::now();
  auto mark = [&](const char* what) {
    if (!trace) return;
    cudaStreamSynchronize(s);
    auto t = std::chrono::steady_clock::now();
    fprintf(stderr, "[tabi] %-12s %9.3f ms\n", what,
            std::chrono::duration<double, std::milli>(t - t_last).count());
    t_last = t;
  };
  alloc_surface(H, nface);
  pack_atoms_dev(H, nchr, m.chrpos, m.atmchr, s);
  DBuf<double>& b0 = H.rn_b0;
  DBuf<double>& b = H.rn_b;
  b0.alloc(2 * (size_t)nface);
  b.alloc(2 * (size_t)nface);
  launch_form_matrix(H, m.nspt, m.sptpos, m.sptnrm, nface, m.nvert, nchr, H.d_atoms.p, b0.p, s);
  H.has_surface = true;
  mark("form_matrix");
  build_tree(H, s);
  mark("tree");
  lists_and_precond(H, s, mark);
  { TABI_K(K_FORM, s); permute_b_kernel<<<ceil_div(nface, 256), 256, 0, s>>>(H.d_perm.p, nface, b0.p, b.p); }
  DBuf<double>& xl = H.rn_x;
  double* x = x_dev;
  if (!x) {
    xl.alloc(2 * (size_t)nface);
    x = xl.p;
  }
  if (ws) {
    // learned initial guess (tree order), GMRES from there: the network
    // corrects the leaf-block preconditioner's solution z = M^-1 b
    DBuf<double>& z = H.rn_z;
    z.alloc(2 * (size_t)nface);
    msolve_dev(H, b.p, z.p, s);
    WsInput in;
    in.n = nface;
    in.px = H.d_x.p;
    in.py = H.d_y.p;
    in.pz = H.d_z.p;
    in.qx = H.d_nx.p;
    in.qy = H.d_ny.p;
    in.qz = H.d_nz.p;
    in.area = H.d_area.p;
    in.b = b.p;
    in.z = z.p;
    ws->forward(in, x, nullptr, s);
    mark("warm start");
  } else {
    TABI_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * 2 * nface, s));
  }
  int iter = 0, ierr = 0;
  double err = 0.0, se = 0.0, ce = 0.0;
  solve_dev(H, b.p, x, &iter, &err, &ierr, nullptr, nullptr, s);
  mark("gmres");
  energy_dev(H, nchr, nullptr, nullptr, x, &se, &ce, s);
  mark("energy");
  if (stats) {
    stats[0] = iter;
    stats[1] = err;
    stats[2] = ierr;
    stats[3] = se;
    stats[4] = ce;
    stats[5] = (double)H.tree.n_near_pairs;
    stats[6] = (double)H.tree.n_far;
    stats[7] = H.tree.nleaf;
  }
}

WsInput ws_input(int nface, const double* tr_xyz, const double* tr_q, const double* tr_area,
                 const double* bvct, const double* zprec) {
  TABI_REQUIRE(nface > 0 && tr_xyz && tr_q && tr_area && bvct, TABI_ERR_ARG, "null argument");
  WsInput in;
  in.n = nface;
  in.px = tr_xyz;
  in.py = tr_xyz + 1;
  in.pz = tr_xyz + 2;
  in.ps = 3;
  in.qx = tr_q;
  in.qy = tr_q + 1;
  in.qz = tr_q + 2;
  in.qs = 3;
  in.area = tr_area;
  in.b = bvct;
  in.z = zprec;
  return in;
}

}  // namespace

extern "C" {

void tabi_default_params(tabi_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->order = 3;
  p->maxparnode = 500;
  p->theta = 0.8;
  p->eps0 = 1.0;
  p->eps1 = 80.0;
  p->kappa = tabi_kappa(0.15, 80.0);
  p->iprcd = 1;
  p->tol = 1e-4;
  p->maxl = 10;
  p->nrmax = 10;
  p->precision = TABI_PREC_FP64;
}

double tabi_kappa(double bulk_strength, double eps1) {
  return std::sqrt((double)(float)8.430325455 * bulk_strength / eps1);
}

int tabi_create(tabi_h* h, const tabi_params* p) {
  if (!h || !p) return TABI_ERR_ARG;
  *h = nullptr;
  tabi_h nh = nullptr;
  int rc = guarded(nullptr, [&] {
    check_params(*p);
    int ndev = 0;
    TABI_CUDA(cudaGetDeviceCount(&ndev));
    TABI_REQUIRE(ndev > 0, TABI_ERR_CUDA, "no CUDA device");
    nh = new tabi_handle_s();
    nh->H.prm = *p;
    nh->H.mv_prec = p->precision;
    TABI_CUDA(cudaGetDevice(&nh->H.device));
    TABI_CUDA(cudaStreamCreateWithFlags(&nh->H.stream, cudaStreamNonBlocking));
    TABI_CUDA(cudaStreamCreateWithFlags(&nh->H.side, cudaStreamNonBlocking));
    TABI_CUDA(cudaEventCreateWithFlags(&nh->H.ev_fork, cudaEventDisableTiming));
    TABI_CUDA(cudaEventCreateWithFlags(&nh->H.ev_join, cudaEventDisableTiming));
    int prio_lo = 0, prio_hi = 0;
    TABI_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    // the large-block chain first; the trailing updates beside it (the chain
    // waits for them one outer block later) and the small-block group (a
    // shorter chain of its own) share the SMs the chain leaves free
    const int prio_mid = (prio_lo + prio_hi) / 2;
    TABI_CUDA(cudaStreamCreateWithPriority(&nh->H.lu_hi, cudaStreamNonBlocking, prio_hi));
    TABI_CUDA(cudaStreamCreateWithPriority(&nh->H.aux, cudaStreamNonBlocking, prio_mid));
    TABI_CUDA(cudaStreamCreateWithPriority(&nh->H.lu_small, cudaStreamNonBlocking, prio_mid));
    TABI_CUDA(cudaEventCreateWithFlags(&nh->H.ev_la, cudaEventDisableTiming));
    TABI_CUDA(cudaEventCreateWithFlags(&nh->H.ev_rest, cudaEventDisableTiming));
    TABI_CUDA(cudaEventCreateWithFlags(&nh->H.ev_lu_join, cudaEventDisableTiming));
    TABI_CUDA(cudaMallocHost(&nh->H.h_pinned, sizeof(double) * 256));
  });
  if (rc != TABI_OK) {
    if (nh) tabi_destroy(nh);
    return rc;
  }
  *h = nh;
  return TABI_OK;
}

int tabi_destroy(tabi_h h) {
  if (!h) return TABI_OK;
  cudaSetDevice(h->H.device);
  if (h->H.stream) cudaStreamSynchronize(h->H.stream);
  if (h->H.h_pinned) cudaFreeHost(h->H.h_pinned);
  if (h->H.side) cudaStreamSynchronize(h->H.side);
  for (cudaStream_t x : {h->H.aux, h->H.lu_hi, h->H.lu_small})
    if (x) cudaStreamSynchronize(x);
  cudaStream_t st[] = {h->H.stream, h->H.side, h->H.aux, h->H.lu_hi, h->H.lu_small};
  cudaEvent_t ev[] = {h->H.ev_fork, h->H.ev_join, h->H.ev_la, h->H.ev_rest, h->H.ev_lu_join};
  delete h;
  for (cudaStream_t x : st)
    if (x) cudaStreamDestroy(x);
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  return TABI_OK;
}

const char* tabi_last_error(tabi_h h) { return h ? h->H.err.c_str() : g_err.c_str(); }

int tabi_form_matrix(tabi_h h, int nspt, const double* sptpos, const double* sptnrm, int nface,
                     const int* nvert, int nchr, const double* chrpos, const double* atmchr,
                     double* tr_xyz, double* tr_q, double* tr_area, double* bvct) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(nspt > 0 && nface > 0 && nchr >= 0, TABI_ERR_ARG, "sizes must be positive");
    TABI_REQUIRE(sptpos && sptnrm && nvert && (nchr == 0 || (chrpos && atmchr)), TABI_ERR_ARG,
                 "null input array");
    for (int k = 0; k < 3 * nface; ++k)
      TABI_REQUIRE(nvert[k] >= 1 && nvert[k] <= nspt, TABI_ERR_ARG,
                   "face vertex index out of range");
    set_device(H);
    cudaStream_t s = H.stream;
    alloc_surface(H, nface);
    DBuf<double>& dpos = H.st_pos;
    DBuf<double>& dnrm = H.st_nrm;
    DBuf<double>& dcp = H.st_cp;
    DBuf<double>& dq = H.st_q;
    DBuf<int>& dfv = H.st_fv;
    h2d(dpos, sptpos, 3 * (size_t)nspt, s);
    h2d(dnrm, sptnrm, 3 * (size_t)nspt, s);
    h2d(dfv, nvert, 3 * (size_t)nface, s);
    if (nchr > 0) {
      h2d(dcp, chrpos, 3 * (size_t)nchr, s);
      h2d(dq, atmchr, (size_t)nchr, s);
    }
    pack_atoms_dev(H, nchr, dcp.p, dq.p, s);
    DBuf<double>& db = H.st_b;
    db.alloc(2 * (size_t)nface);
    launch_form_matrix(H, nspt, dpos.p, dnrm.p, nface, dfv.p, nchr, H.d_atoms.p, db.p, s);
    if (tr_xyz || tr_q) {
      DBuf<double>& axyz = H.st_axyz;
      DBuf<double>& aq = H.st_aq;
      axyz.alloc(3 * (size_t)nface);
      aq.alloc(3 * (size_t)nface);
      { TABI_K(K_FORM, s); aos_from_soa_kernel<<<ceil_div(nface, 256), 256, 0, s>>>(
          H.d_x.p, H.d_y.p, H.d_z.p, H.d_nx.p, H.d_ny.p, H.d_nz.p, nface, axyz.p, aq.p); }
      if (tr_xyz)
        TABI_CUDA(cudaMemcpyAsync(tr_xyz, axyz.p, sizeof(double) * 3 * nface,
                                  cudaMemcpyDeviceToHost, s));
      if (tr_q)
        TABI_CUDA(cudaMemcpyAsync(tr_q, aq.p, sizeof(double) * 3 * nface,
                                  cudaMemcpyDeviceToHost, s));
      TABI_CUDA(cudaStreamSynchronize(s));
    }
    if (tr_area)
      TABI_CUDA(cudaMemcpyAsync(tr_area, H.d_area.p, sizeof(double) * nface,
                                cudaMemcpyDeviceToHost, s));
    if (bvct)
      TABI_CUDA(cudaMemcpyAsync(bvct, db.p, sizeof(double) * 2 * nface, cudaMemcpyDeviceToHost,
                                s));
    TABI_CUDA(cudaStreamSynchronize(s));
    H.has_surface = true;
  });
}

int tabi_set_surface(tabi_h h, int nface, const double* tr_xyz, const double* tr_q,
                     const double* tr_area) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(nface > 0 && tr_xyz && tr_q && tr_area, TABI_ERR_ARG, "bad surface arrays");
    set_device(H);
    cudaStream_t s = H.stream;
    alloc_surface(H, nface);
    DBuf<double>& a = H.st_axyz;
    DBuf<double>& b = H.st_aq;
    DBuf<double>& c = H.st_b;
    h2d(a, tr_xyz, 3 * (size_t)nface, s);
    h2d(b, tr_q, 3 * (size_t)nface, s);
    h2d(c, tr_area, (size_t)nface, s);
    { TABI_K(K_FORM, s); soa_from_aos_kernel<<<ceil_div(nface, 256), 256, 0, s>>>(a.p, b.p, c.p, nface, H.d_x.p,
                                                             H.d_y.p, H.d_z.p, H.d_nx.p,
                                                             H.d_ny.p, H.d_nz.p, H.d_area.p); }
    TABI_CUDA(cudaStreamSynchronize(s));
    H.has_surface = true;
  });
}

int tabi_rhs(tabi_h h, int nchr, const double* chrpos, const double* atmchr, double* bvct) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_surface, TABI_ERR_STATE, "no surface loaded");
    TABI_REQUIRE(nchr > 0 && chrpos && atmchr && bvct, TABI_ERR_ARG, "bad atom arrays");
    set_device(H);
    cudaStream_t s = H.stream;
    DBuf<double>& dcp = H.st_cp;
    DBuf<double>& dq = H.st_q;
    DBuf<double>& db = H.st_b;
    h2d(dcp, chrpos, 3 * (size_t)nchr, s);
    h2d(dq, atmchr, (size_t)nchr, s);
    pack_atoms_dev(H, nchr, dcp.p, dq.p, s);
    db.alloc(2 * (size_t)H.n);
    launch_rhs(H, nchr, H.d_atoms.p, db.p, s);
    TABI_CUDA(cudaMemcpyAsync(bvct, db.p, sizeof(double) * 2 * H.n, cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

int tabi_build_tree(tabi_h h, int* orderarr, int* nleaf) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_surface, TABI_ERR_STATE, "no surface loaded");
    TABI_REQUIRE(!H.has_tree, TABI_ERR_STATE, "tree already built for this surface");
    set_device(H);
    do_build(H, H.stream);
    if (orderarr)
      for (int i = 0; i < H.n; ++i) orderarr[i] = H.h_perm[i] + 1;
    if (nleaf) *nleaf = H.tree.nleaf;
  });
}

int tabi_matvec_dev(tabi_h h, int n2, const double* x_dev, double* y_dev, void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    require_tree(H, n2);
    TABI_REQUIRE(x_dev && y_dev && x_dev != y_dev, TABI_ERR_ARG, "bad vectors");
    set_device(H);
    matvec_dev(H, x_dev, y_dev, pick(H, stream), true);
  });
}

int tabi_matvec(tabi_h h, int n2, const double* x, double* y) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    require_tree(H, n2);
    TABI_REQUIRE(x && y, TABI_ERR_ARG, "null vector");
    set_device(H);
    cudaStream_t s = H.stream;
    H.d_b.alloc(n2);
    H.d_xio.alloc(n2);
    TABI_CUDA(cudaMemcpyAsync(H.d_b.p, x, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    matvec_dev(H, H.d_b.p, H.d_xio.p, s, true);
    TABI_CUDA(cudaMemcpyAsync(y, H.d_xio.p, sizeof(double) * n2, cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

int tabi_msolve_dev(tabi_h h, int n2, const double* r_dev, double* z_dev, void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    require_tree(H, n2);
    TABI_REQUIRE(r_dev && z_dev, TABI_ERR_ARG, "bad vectors");
    set_device(H);
    msolve_dev(H, r_dev, z_dev, pick(H, stream));
  });
}

int tabi_msolve(tabi_h h, int n2, const double* r, double* z) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    require_tree(H, n2);
    TABI_REQUIRE(r && z, TABI_ERR_ARG, "null vector");
    set_device(H);
    cudaStream_t s = H.stream;
    H.d_b.alloc(n2);
    H.d_xio.alloc(n2);
    TABI_CUDA(cudaMemcpyAsync(H.d_b.p, r, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    msolve_dev(H, H.d_b.p, H.d_xio.p, s);
    TABI_CUDA(cudaMemcpyAsync(z, H.d_xio.p, sizeof(double) * n2, cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

int tabi_solve_dev(tabi_h h, int n2, const double* b_dev, double* x_dev, int* iter, double* err,
                   int* ierr, double* err_hist, int* n_hist, void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    require_tree(H, n2);
    TABI_REQUIRE(b_dev && x_dev && iter && err && ierr, TABI_ERR_ARG, "null argument");
    set_device(H);
    solve_dev(H, b_dev, x_dev, iter, err, ierr, err_hist, n_hist, pick(H, stream));
  });
}

int tabi_solve(tabi_h h, int n2, const double* b, double* x, int* iter, double* err, int* ierr,
               double* err_hist, int* n_hist) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    require_tree(H, n2);
    TABI_REQUIRE(b && x && iter && err && ierr, TABI_ERR_ARG, "null argument");
    set_device(H);
    cudaStream_t s = H.stream;
    H.d_b.alloc(n2);
    H.d_xio.alloc(n2);
    TABI_CUDA(cudaMemcpyAsync(H.d_b.p, b, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    TABI_CUDA(cudaMemcpyAsync(H.d_xio.p, x, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    solve_dev(H, H.d_b.p, H.d_xio.p, iter, err, ierr, err_hist, n_hist, s);
    TABI_CUDA(cudaMemcpyAsync(x, H.d_xio.p, sizeof(double) * n2, cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

int tabi_energy_dev(tabi_h h, int nchr, const double* chrpos_dev, const double* atmchr_dev,
                    const double* x_dev, double* soleng, double* couleng, void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_surface, TABI_ERR_STATE, "no surface loaded");
    TABI_REQUIRE(nchr > 0 && chrpos_dev && atmchr_dev && x_dev && soleng && couleng,
                 TABI_ERR_ARG, "bad energy arguments");
    set_device(H);
    cudaStream_t s = pick(H, stream);
    pack_atoms_dev(H, nchr, chrpos_dev, atmchr_dev, s);
    energy_dev(H, nchr, nullptr, nullptr, x_dev, soleng, couleng, s);
  });
}

int tabi_energy(tabi_h h, int nchr, const double* chrpos, const double* atmchr, const double* x,
                double* soleng, double* couleng) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_surface, TABI_ERR_STATE, "no surface loaded");
    TABI_REQUIRE(nchr > 0 && chrpos && atmchr && x && soleng && couleng, TABI_ERR_ARG,
                 "bad energy arguments");
    set_device(H);
    cudaStream_t s = H.stream;
    DBuf<double>& dcp = H.st_cp;
    DBuf<double>& dq = H.st_q;
    DBuf<double>& dx = H.st_x;
    h2d(dcp, chrpos, 3 * (size_t)nchr, s);
    h2d(dq, atmchr, (size_t)nchr, s);
    h2d(dx, x, 2 * (size_t)H.n, s);
    pack_atoms_dev(H, nchr, dcp.p, dq.p, s);
    energy_dev(H, nchr, nullptr, nullptr, dx.p, soleng, couleng, s);
  });
}

int tabi_energy_noalloc(int nface, const double* tr_xyz_dev, const double* tr_q_dev,
                        const double* tr_area_dev, const double* x_dev, int nchr,
                        const double* chrpos_dev, const double* atmchr_dev, double kappa,
                        double eps0, double eps1, double* out_dev, void* stream) {
  return guarded(nullptr, [&] {
    energy_noalloc(nface, tr_xyz_dev, tr_q_dev, tr_area_dev, x_dev, nchr, chrpos_dev, atmchr_dev,
                   kappa, eps0, eps1, out_dev, (cudaStream_t)stream);
  });
}

int tabi_run_dev(tabi_h h, int nspt, const double* sptpos_dev, const double* sptnrm_dev,
                 int nface, const int* nvert_dev, int nchr, const double* chrpos_dev,
                 const double* atmchr_dev, double* x_dev, double* stats, void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    set_device(H);
    cudaStream_t s = pick(H, stream);
    cudaStream_t keep = H.stream;
    H.stream = s;
    struct Restore {
      Handle& H;
      cudaStream_t k;
      ~Restore() { H.stream = k; }
    } restore{H, keep};
    MolDev m{nspt, sptpos_dev, sptnrm_dev, nface, nvert_dev, nchr, chrpos_dev, atmchr_dev};
    run_molecule(H, h->ws, m, x_dev, stats, s);
  });
}

int tabi_counts(tabi_h h, int64_t* near_pairs, int64_t* far_interactions) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_tree, TABI_ERR_STATE, "no tree");
    if (near_pairs) *near_pairs = H.tree.n_near_pairs;
    if (far_interactions) *far_interactions = H.tree.n_far;
  });
}

int tabi_face_filter_dev(tabi_h h, int nspt, const double* sptpos_dev, int nface,
                         const int* nvert_dev, int* nvert_out_dev, int* nkept, double* s_area,
                         void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(nspt > 0 && nface > 0 && sptpos_dev && nvert_dev && nvert_out_dev && nkept &&
                     s_area,
                 TABI_ERR_ARG, "bad arguments");
    TABI_REQUIRE(nvert_out_dev != nvert_dev, TABI_ERR_ARG, "the output must not alias the input");
    set_device(H);
    face_filter_dev(H, nspt, sptpos_dev, nface, nvert_dev, nvert_out_dev, nkept, s_area,
                    pick(H, stream));
  });
}

int tabi_pivoted_leaves(tabi_h h, int* count) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_precond && H.prm.iprcd == 1, TABI_ERR_STATE,
                 "no leaf-block preconditioner built");
    TABI_REQUIRE(count != nullptr, TABI_ERR_ARG, "null argument");
    *count = H.pc_pv_leaves;
  });
}

int tabi_tree_nodes(tabi_h h, int* nnodes, int* ibeg, int* numpar, int* level, int* nchild,
                    double* geo) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(H.has_tree, TABI_ERR_STATE, "no tree");
    Tree& T = H.tree;
    if (nnodes) *nnodes = T.nnodes;
    if (!ibeg && !numpar && !level && !nchild && !geo) return;
    // depth-first (creation) order of the reference
    std::vector<int> order, stack = {0};
    while (!stack.empty()) {
      int c = stack.back();
      stack.pop_back();
      order.push_back(c);
      for (int k = T.nchild[c] - 1; k >= 0; --k) stack.push_back(T.child0[c] + k);
    }
    for (size_t k = 0; k < order.size(); ++k) {
      int c = order[k];
      if (ibeg) ibeg[k] = T.ibeg[c] + 1;
      if (numpar) numpar[k] = T.num[c];
      if (level) level[k] = T.level[c];
      if (nchild) nchild[k] = T.nchild[c];
      if (geo) {
        geo[4 * k] = T.mid[3 * c];
        geo[4 * k + 1] = T.mid[3 * c + 1];
        geo[4 * k + 2] = T.mid[3 * c + 2];
        geo[4 * k + 3] = T.rad[c];
      }
    }
  });
}

int tabi_profile_enable(tabi_h h, int enable) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    H.prof.reset();
    H.prof.on = enable != 0;
  });
}

int tabi_profile_read(tabi_h h, int kclass, double* ms, int64_t* launches) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(kclass >= -1 && kclass < K_NCLASS, TABI_ERR_ARG, "bad kernel class");
    H.prof.resolve();
    double t = 0.0;
    int64_t l = 0;
    for (int k = 0; k < K_NCLASS; ++k)
      if ((kclass == -1 && k < K_PHASE_MATVEC) || kclass == k) {
        t += H.prof.ms[k];
        l += H.prof.launches[k];
      }
    if (ms) *ms = t;
    if (launches) *launches = l;
  });
}

int tabi_profile_nclasses(void) { return K_NCLASS; }

const char* tabi_profile_class_name(int kclass) {
  static const char* names[K_NCLASS] = {"form_matrix", "tree",   "lists",     "moments",
                                        "far",         "near",   "reduce",    "assemble",
                                        "lu_panel",    "solve",  "vector",    "energy",
                                        "lu_update",   "lu_post",   "lu_strip",
                                        "lu_swap",     "matvec", "lu",       "apply"};
  return (kclass >= 0 && kclass < K_NCLASS) ? names[kclass] : "all";
}

int tabi_probe_fp64_peak(double ms, double* flops) { return probe_fma_peak<double>(ms, flops); }
int tabi_probe_fp32_peak(double ms, double* flops) { return probe_fma_peak<float>(ms, flops); }

// ---- accuracy reference
int tabi_direct_targets(tabi_h h, int nt, const int* targets, const double* x, double* y) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(nt > 0 && targets && x && y, TABI_ERR_ARG, "null argument");
    TABI_REQUIRE(H.has_surface, TABI_ERR_STATE, "no surface");
    for (int k = 0; k < nt; ++k)
      TABI_REQUIRE(targets[k] >= 0 && targets[k] < H.n, TABI_ERR_ARG, "target index out of range");
    set_device(H);
    cudaStream_t s = H.stream;
    H.st_fv.alloc(nt);
    TABI_CUDA(cudaMemcpyAsync(H.st_fv.p, targets, sizeof(int) * nt, cudaMemcpyHostToDevice, s));
    h2d(H.st_x, x, 2 * (size_t)H.n, s);
    H.d_tmp.alloc(2 * (size_t)nt);
    direct_targets_dev(H, nt, H.st_fv.p, H.st_x.p, H.d_tmp.p, s);
    TABI_CUDA(cudaMemcpyAsync(y, H.d_tmp.p, sizeof(double) * 2 * nt, cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

// ---- shards of the operator
int tabi_set_exchange(tabi_h h, tabi_exchange_fn fn, void* user) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    h->H.xchg = fn;
    h->H.xchg_user = fn ? user : nullptr;
  });
}

int tabi_set_target_range(tabi_h h, int t0, int t1) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    set_device(H);
    set_target_range(H, t0, t1, H.stream);
  });
}

// ---- output_potential (main.f90:226-326)
int tabi_output_potential_dev(tabi_h h, int nspt, const double* sptpos_dev, int nface,
                              const int* nvert_dev, const double* x_dev, double* x_orig_dev,
                              double* vert_ptl_dev, void* stream) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    set_device(H);
    output_potential_dev(H, nspt, sptpos_dev, nface, nvert_dev, x_dev, x_orig_dev, vert_ptl_dev,
                         pick(H, stream));
  });
}

int tabi_output_potential(tabi_h h, int nspt, const double* sptpos, int nface, const int* nvert,
                          const double* x, double* x_orig, double* vert_ptl) {
  if (!h) return TABI_ERR_ARG;
  return guarded(h, [&] {
    Handle& H = h->H;
    TABI_REQUIRE(sptpos && nvert && x && x_orig && vert_ptl && nspt > 0 && nface > 0,
                 TABI_ERR_ARG, "null argument");
    set_device(H);
    cudaStream_t s = H.stream;
    h2d(H.vp_pos, sptpos, 3 * (size_t)nspt, s);
    h2d(H.vp_nv, nvert, 3 * (size_t)nface, s);
    h2d(H.vp_xo, x, 2 * (size_t)nface, s);  // x in tree order
    H.vp_vert.alloc(2 * (size_t)nspt);
    H.d_tmp.alloc(2 * (size_t)nface);
    output_potential_dev(H, nspt, H.vp_pos.p, nface, H.vp_nv.p, H.vp_xo.p, H.d_tmp.p,
                         H.vp_vert.p, s);
    TABI_CUDA(cudaMemcpyAsync(x_orig, H.d_tmp.p, sizeof(double) * 2 * nface,
                              cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaMemcpyAsync(vert_ptl, H.vp_vert.p, sizeof(double) * 2 * nspt,
                              cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

// ---- learned warm start
// NULL = the CUDA default stream, as for any CUDA call
static cudaStream_t ws_stream(tabi_ws, void* stream) { return (cudaStream_t)stream; }

int tabi_ws_create(tabi_ws* w, int hidden, int layers, unsigned long long seed) {
  if (!w) return TABI_ERR_ARG;
  *w = nullptr;
  return guarded(nullptr, [&] {
    auto o = std::make_unique<tabi_ws_s>();
    o->net = new WsNet(hidden, layers, seed);
    *w = o.release();
  });
}

int tabi_ws_destroy(tabi_ws w) {
  if (!w) return TABI_ERR_ARG;
  delete w->net;
  delete w;
  return TABI_OK;
}

long long tabi_ws_nparams(tabi_ws w) { return (w && w->net) ? (long long)w->net->np : -1; }

int tabi_ws_get_params(tabi_ws w, float* theta, long long n) {
  if (!w || !theta) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    TABI_REQUIRE(n == w->net->np, TABI_ERR_ARG, "parameter count mismatch");
    w->net->get_params(theta);
  });
}

int tabi_ws_set_params(tabi_ws w, const float* theta, long long n) {
  if (!w || !theta) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    TABI_REQUIRE(n == w->net->np, TABI_ERR_ARG, "parameter count mismatch");
    w->net->set_params(theta);
  });
}

int tabi_ws_predict_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                        const double* tr_area, const double* bvct, const double* zprec,
                        double* x0, void* stream) {
  if (!w) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    TABI_REQUIRE(x0 != nullptr, TABI_ERR_ARG, "null output");
    cudaStream_t s = ws_stream(w, stream);
    w->net->forward(ws_input(nface, tr_xyz, tr_q, tr_area, bvct, zprec), x0, nullptr, s);
  });
}

int tabi_ws_loss_grad_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                          const double* tr_area, const double* bvct, const double* zprec,
                          const double* x_target, double* loss, float* grad, void* stream) {
  if (!w) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    TABI_REQUIRE(x_target && loss, TABI_ERR_ARG, "null argument");
    cudaStream_t s = ws_stream(w, stream);
    WsNet& N = *w->net;
    N.forward(ws_input(nface, tr_xyz, tr_q, tr_area, bvct, zprec), nullptr, x_target, s);
    N.backward(nface, s);
    *loss = N.read_loss(s);
    if (grad) {
      TABI_CUDA(cudaMemcpyAsync(grad, N.grad.p, sizeof(float) * N.np, cudaMemcpyDeviceToHost, s));
      TABI_CUDA(cudaStreamSynchronize(s));
    }
  });
}

int tabi_ws_train_step_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                           const double* tr_area, const double* bvct, const double* zprec,
                           const double* x_target, double lr, double* loss, void* stream) {
  if (!w) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    TABI_REQUIRE(x_target != nullptr, TABI_ERR_ARG, "null target");
    TABI_REQUIRE(lr > 0.0 && std::isfinite(lr), TABI_ERR_ARG, "learning rate must be > 0");
    cudaStream_t s = ws_stream(w, stream);
    WsNet& N = *w->net;
    N.forward(ws_input(nface, tr_xyz, tr_q, tr_area, bvct, zprec), nullptr, x_target, s);
    N.backward(nface, s);
    N.adam(lr, s);
    if (loss) *loss = N.read_loss(s);
  });
}

int tabi_ws_graph_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                      const double* tr_area, const double* bvct, const double* zprec, int* nbr,
                      float* feat, void* stream) {
  if (!w) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    cudaStream_t s = ws_stream(w, stream);
    WsNet& N = *w->net;
    N.graph(ws_input(nface, tr_xyz, tr_q, tr_area, bvct, zprec), s);
    TABI_REQUIRE(N.graph_exact(s), TABI_ERR_LIMIT,
                 "neighbour search: fewer than 16 other panels");
    if (nbr)
      TABI_CUDA(cudaMemcpyAsync(nbr, N.nbr.p, sizeof(int) * (size_t)nface * kWsK,
                                cudaMemcpyDeviceToHost, s));
    if (feat)
      TABI_CUDA(cudaMemcpyAsync(feat, N.feat.p, sizeof(float) * (size_t)nface * kWsF,
                                cudaMemcpyDeviceToHost, s));
    TABI_CUDA(cudaStreamSynchronize(s));
  });
}

int tabi_set_warmstart(tabi_h h, tabi_ws w) {
  if (!h) return TABI_ERR_ARG;
  h->ws = w ? w->net : nullptr;
  return TABI_OK;
}

// ---- batched solves
int tabi_batch_run_dev(const tabi_params* p, int nmol, const tabi_mol_dev* mols, tabi_ws ws,
                       int nworkers, double* stats) {
  if (!p || !mols || nmol <= 0) return TABI_ERR_ARG;
  return guarded(nullptr, [&] {
    check_params(*p);
    TABI_REQUIRE(nworkers >= 1 && nworkers <= 64, TABI_ERR_ARG, "nworkers must be in 1..64");
    for (int k = 0; k < nmol; ++k) {
      check_mol(mols[k]);
      TABI_REQUIRE(mols[k].maxparnode >= 0 && mols[k].order >= 0 && mols[k].order <= kMaxOrder,
                   TABI_ERR_ARG, "per-molecule maxparnode / order out of range");
    }
    int dev = 0;
    TABI_CUDA(cudaGetDevice(&dev));
    // largest first (longest-processing-time order over the workers)
    std::vector<int> order(nmol);
    for (int k = 0; k < nmol; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return mols[a].nface > mols[b].nface; });
    std::atomic<int> next{0};
    std::atomic<bool> stop{false};
    std::vector<std::string> errs(nworkers);
    std::vector<int> codes(nworkers, TABI_OK);
    const auto t0 = std::chrono::steady_clock::now();
    auto ms_since = [&](std::chrono::steady_clock::time_point a,
                        std::chrono::steady_clock::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    auto worker = [&](int w) {
      tabi_h h = nullptr;
      try {
        TABI_CUDA(cudaSetDevice(dev));
        int rc = tabi_create(&h, p);
        TABI_REQUIRE(rc == TABI_OK, rc, "batch worker: cannot create a handle");
        std::unique_ptr<WsNet> own;
        if (ws) own = ws->net->clone();
        for (;;) {
          if (stop.load()) break;
          const int k = next.fetch_add(1);
          if (k >= nmol) break;
          const tabi_mol_dev& md = mols[order[k]];
          Handle& H = h->H;
          H.prm = *p;
          if (md.maxparnode > 0) H.prm.maxparnode = md.maxparnode;
          if (md.order > 0) H.prm.order = md.order;
          H.mv_prec = H.prm.precision;
          double* st = stats ? stats + (size_t)kBatchStats * order[k] : nullptr;
          const auto ta = std::chrono::steady_clock::now();
          MolDev m{md.nspt, md.sptpos, md.sptnrm, md.nface, md.nvert, md.nchr, md.chrpos,
                   md.atmchr};
          run_molecule(H, own.get(), m, nullptr, st, H.stream);
          TABI_CUDA(cudaStreamSynchronize(H.stream));
          const auto tb = std::chrono::steady_clock::now();
          if (st) {
            st[8] = ms_since(ta, tb);
            st[9] = ms_since(t0, tb);
            st[10] = w;
            st[11] = H.prm.maxparnode;
          }
        }
      } catch (const Error& e) {
        errs[w] = e.what();
        codes[w] = e.code;
        stop = true;
      } catch (const std::exception& e) {
        errs[w] = e.what();
        codes[w] = TABI_ERR_CUDA;
        stop = true;
      }
      if (h) tabi_destroy(h);
    };
    std::vector<std::thread> th;
    for (int w = 0; w < nworkers; ++w) th.emplace_back(worker, w);
    for (auto& t : th) t.join();
    for (int w = 0; w < nworkers; ++w)
      TABI_REQUIRE(codes[w] == TABI_OK, codes[w],
                   "batch worker " + std::to_string(w) + ": " + errs[w]);
  });
}

}  // extern "C"
