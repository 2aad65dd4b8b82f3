/*
 * tabi_gpu.h -- C ABI of the B200 TABI-PB solve path (libtabi_gpu.so).
 *
 * The reference (gengwh/TABI-PB, Fortran) solves the boundary-integral
 * Poisson-Boltzmann system with a treecode matvec, a leaf-block-diagonal
 * preconditioner and SLATEC GMRES, all driven from module globals by
 * src/main.f90.  Each entry point below replaces one reference interface; the
 * citation is given with each.  A Fortran caller binds them with
 * ISO_C_BINDING (interface blocks with bind(C), value arguments, c_double
 * arrays); see INTEGRATION.md.
 *
 * Conventions
 *  - All arrays are host arrays unless the name ends in _dev (device
 *    pointers, with a cudaStream_t passed as void*; NULL = the handle's own
 *    stream).
 *  - Layouts are the reference's: coordinates are column-major 3 x N
 *    (point i at [3i, 3i+2]); face vertex lists and orderarr are 1-based;
 *    vectors of length 2N are [x1 ; x2] (potential ; normal derivative).
 *  - After tabi_build_tree, every length-N / 2N vector exchanged with the
 *    library is in TREE ORDER, exactly as the reference's bvct/xvct are after
 *    treecode_initialization (main.f90:447-453).
 *  - Every function returns 0 on success or a negative TABI_ERR_* code;
 *    tabi_last_error() gives the message.  A handle is not thread-safe.
 */
#ifndef TABI_GPU_H
#define TABI_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TABI_OK 0
#define TABI_ERR_ARG (-1)       /* invalid argument */
#define TABI_ERR_CUDA (-2)      /* CUDA runtime error */
#define TABI_ERR_NOMEM (-3)     /* device or host allocation failed */
#define TABI_ERR_STATE (-4)     /* call out of order (e.g. matvec before tree) */
#define TABI_ERR_SINGULAR (-5)  /* a leaf block LU hit an exact zero pivot */
#define TABI_ERR_LIMIT (-6)     /* an internal size limit was exceeded */

#define TABI_PREC_FP64 0 /* plain FP64 treecode (the reference's arithmetic) */
/* Mixed precision (no counterpart in the reference): the treecode operator
 * (moments contraction, Taylor recurrences, near-field kernels, per-leaf and
 * per-cluster sums) in FP32, the per-target sum over leaves and clusters in
 * FP64; tabi_matvec applies that FP32 operator.  tabi_solve wraps GMRES on it
 * in FP64 iterative refinement: the residual b - A x with the FP64 operator,
 * the preconditioner (FP64 leaf LU), Arnoldi, Givens and the energy stay FP64,
 * and the stopping test is the FP64 |M^-1 (b - A x)| / |M^-1 b| <= tol. */
#define TABI_PREC_MIXED 1

typedef struct tabi_handle_s* tabi_h;

/* usrdata.in parameters (main.f90:39-50) and the hard-coded solver settings
 * (main.f90:55-58, 93-97).  kappa is the inverse Debye length as main.f90:62-63
 * computes it (see tabi_kappa).  theta must be in (0, 1): the reference's
 * self-interaction removal (treecode3d_pb.f:1169-1172) relies on the MAC
 * failing for every cluster that contains the target. */
typedef struct {
  int order;       /* Taylor order p (1..8) */
  int maxparnode;  /* leaf size L */
  double theta;    /* MAC */
  double kappa;    /* 1/A */
  double eps0;     /* interior dielectric (epsp) */
  double eps1;     /* exterior dielectric (epsw) */
  int iprcd;       /* 1 = leaf-block preconditioner, else diagonal scaling */
  double tol;      /* GMRES tolerance (reference: 1e-4) */
  int maxl;        /* GMRES restart length (reference: 10) */
  int nrmax;       /* max restarts (reference: 10) */
  int precision;   /* TABI_PREC_* */
  int flags;       /* TABI_FLAG_* bits, 0 for the defaults */
} tabi_params;

/* The leaf blocks are factored by a blocked LU without row interchanges whose
 * every multiplier is checked against |l| <= 1 - 2^-20: when that holds,
 * DGETRF2's partial pivoting (treecode3d_pb.f:1530, dgetrf_dep.f:757-900)
 * keeps the diagonal row at every column and the factors are its factors;
 * a leaf that fails the check is factored again with partial pivoting.  This
 * flag factors every leaf with partial pivoting from the start (the same
 * factors, slower). */
#define TABI_FLAG_PIVOTED_LU 1

/* Fills p with the reference defaults: order 3, maxparnode 500, theta 0.8,
 * eps 1/80, 0.15 M (kappa from tabi_kappa), iprcd 1, tol 1e-4, maxl 10,
 * nrmax 10, FP64. */
void tabi_default_params(tabi_params* p);

/* main.f90:62-63: kappa = sqrt(8.430325455 * I / eps1) with the literal
 * rounded to REAL*4 as the Fortran does. */
double tabi_kappa(double bulk_strength, double eps1);

int tabi_create(tabi_h* h, const tabi_params* p);
int tabi_destroy(tabi_h h);
const char* tabi_last_error(tabi_h h);

/* main.f90:546-610 form_matrix.  sptpos/sptnrm: 3 x nspt vertices and
 * vertex normals (MSMS .vert), nvert: 3 x nface 1-based (MSMS .face, already
 * filtered by readin.f90:264-333 surface_area), chrpos: 3 x nchr, atmchr:
 * nchr.  Outputs (original face order): tr_xyz, tr_q (3 x nface centroids and
 * unit normals), tr_area (nface), bvct (2 nface).  Any output may be NULL.
 * Also loads the surface into the handle (replaces tabi_set_surface). */
int tabi_form_matrix(tabi_h h, int nspt, const double* sptpos,
                     const double* sptnrm, int nface, const int* nvert,
                     int nchr, const double* chrpos, const double* atmchr,
                     double* tr_xyz, double* tr_q, double* tr_area,
                     double* bvct);

/* readin.f90:264-333 surface_area on device arrays: drops the faces whose
 * Heron area is below 1e-5 or whose centroid lies within sqrt(1e-5) of one of
 * the 10 faces before it in the given list.  nvert_dev: 3 x nface, 1-based;
 * nvert_out_dev (capacity 3 x nface, not aliasing the input) receives the kept
 * faces in their order, *nkept their number and *s_area the total area of all
 * faces (summed by blocks: it differs from the reference's running sum in
 * rounding only).  Returns after the counts are on the host. */
int tabi_face_filter_dev(tabi_h h, int nspt, const double* sptpos_dev, int nface,
                         const int* nvert_dev, int* nvert_out_dev, int* nkept,
                         double* s_area, void* stream);

/* Loads centroids, unit normals and areas (original order) when the caller
 * already has them (the state form_matrix leaves in module treecode). */
int tabi_set_surface(tabi_h h, int nface, const double* tr_xyz,
                     const double* tr_q, const double* tr_area);

/* main.f90:597-607: the RHS of form_matrix alone, for the loaded surface,
 * in the CURRENT order of the handle (original order before
 * tabi_build_tree, tree order after). */
int tabi_rhs(tabi_h h, int nchr, const double* chrpos, const double* atmchr,
             double* bvct);

/* main.f90:400-441 SETUP + CREATE_TREE (treecode3d_pb.f:54-356): builds the
 * tree on the device (same node sets, boxes and children order as the
 * reference), the interaction lists and the preconditioner factors.
 * orderarr (may be NULL) receives, per tree slot, the 1-based original face
 * index; the caller then permutes its arrays as main.f90:447-453 does.  The
 * order of faces inside a leaf may differ from the reference's (its
 * PARTITION is not stable); node sets are identical. */
int tabi_build_tree(tabi_h h, int* orderarr, int* nleaf);

/* main.f90:467-488 MATVECmain -> TREE_COMPP_PB (treecode3d_pb.f:1130-1189):
 * y = A x with A the treecode BIE operator; an x with sum|x| < 1e-10 gives
 * y = x as in the reference.  n2 = 2 nface. */
int tabi_matvec(tabi_h h, int n2, const double* x, double* y);
int tabi_matvec_dev(tabi_h h, int n2, const double* x_dev, double* y_dev,
                    void* stream);

/* main.f90:511-529 MSOLVEdric -> LEAFMATVECpara (treecode3d_pb.f:1393-1542)
 * when iprcd == 1, else main.f90:532-542 MSOLVEprec.  The leaf blocks are
 * factored once in tabi_build_tree (the reference re-factors the same blocks
 * on every call; the factors are identical). */
int tabi_msolve(tabi_h h, int n2, const double* r, double* z);
int tabi_msolve_dev(tabi_h h, int n2, const double* r_dev, double* z_dev,
                    void* stream);

/* main.f90:92-139 + dgmres_dep.f DGMRES (ITOL = 2, JPRE = -1, JSCAL = 0,
 * KMP = MAXL): x holds x0 on entry (the reference uses 0).  iter, err, ierr
 * as DGMRES returns them (ierr 0 converged, 1 iteration limit, 2 stagnation,
 * -1/-2 as in dgmres_dep.f:840-851).  err_hist (may be NULL, capacity
 * (nrmax+1)*maxl) receives the per-iteration error estimates the reference
 * prints at dgmres_dep.f:1796; *n_hist their count. */
int tabi_solve(tabi_h h, int n2, const double* b, double* x, int* iter,
               double* err, int* ierr, double* err_hist, int* n_hist);
int tabi_solve_dev(tabi_h h, int n2, const double* b_dev, double* x_dev,
                   int* iter, double* err, int* ierr, double* err_hist,
                   int* n_hist, void* stream);

/* main.f90:144-157 + potential_molecule (main.f90:614-657): solvation energy
 * soleng and Coulomb energy couleng (kcal/mol) for the solution x (tree
 * order, as tabi_solve returns it). */
int tabi_energy(tabi_h h, int nchr, const double* chrpos,
                const double* atmchr, const double* x, double* soleng,
                double* couleng);
int tabi_energy_dev(tabi_h h, int nchr, const double* chrpos_dev,
                    const double* atmchr_dev, const double* x_dev,
                    double* soleng, double* couleng, void* stream);

/* Solvation and Coulomb energy as tabi_energy, for callers that cannot
 * allocate device memory (device memory owned and budgeted by another
 * allocator, or a pipeline that cannot absorb the device-wide
 * synchronisation of cudaFree).  No counterpart in the reference.
 * Allocates nothing: needs no handle; its scratch is a file-scope static
 * device array of 2^20 doubles (8 MiB) that every GPU which loads the library
 * holds until exit.  All pointers are device pointers on the current device:
 * the surface in the reference's layout (tr_xyz, tr_q 3 x nface, tr_area),
 * x (2 nface, same face order), atoms (chrpos 3 x nchr, atmchr); out receives
 * [soleng, couleng] (kcal/mol).  nchr <= 524288, else TABI_ERR_LIMIT.  The
 * first call on a device looks up the scratch address (cudaGetSymbolAddress)
 * and should come before any stream capture.  The address is cached for the
 * life of the process: do not call this after cudaDeviceReset (or anything
 * else that recreates the device's primary context), which reloads the module
 * at another address.  Every call writes the scratch
 * it reads, nothing needs clearing; calls that overlap on the GPU (on
 * different streams) share the scratch and race. */
int tabi_energy_noalloc(int nface, const double* tr_xyz_dev,
                        const double* tr_q_dev, const double* tr_area_dev,
                        const double* x_dev, int nchr,
                        const double* chrpos_dev, const double* atmchr_dev,
                        double kappa, double eps0, double eps1,
                        double* out_dev, void* stream);

/* Whole path on device-resident inputs (form_matrix, tree, preconditioner,
 * GMRES, energy) -- one call per molecule.  Inputs as tabi_form_matrix but
 * device pointers; x_dev (2 nface, tree order on return) may be NULL.
 * stats (may be NULL) receives: [0] iter, [1] err, [2] ierr, [3] soleng,
 * [4] couleng, [5] near pairs per matvec, [6] far interactions per matvec,
 * [7] nleaf. */
int tabi_run_dev(tabi_h h, int nspt, const double* sptpos_dev,
                 const double* sptnrm_dev, int nface, const int* nvert_dev,
                 int nchr, const double* chrpos_dev, const double* atmchr_dev,
                 double* x_dev, double* stats, void* stream);

/* Interaction counts of the current tree (per matvec): near-field pairs and
 * far-field (target, cluster) evaluations; as the reference's traversal
 * would perform them. */
int tabi_counts(tabi_h h, int64_t* near_pairs, int64_t* far_interactions);

/* Leaf blocks of the current tree that were factored with partial pivoting:
 * those whose no-interchange check failed (see TABI_FLAG_PIVOTED_LU), or all
 * of them when that flag is set.  No counterpart in the reference. */
int tabi_pivoted_leaves(tabi_h h, int* count);

/* Node table of the current tree in depth-first (reference creation) order:
 * ibeg (1-based), numpar, level, num_children, and geo = x_mid, y_mid,
 * z_mid, radius per node.  Pass NULL arrays to get *nnodes only. */
int tabi_tree_nodes(tabi_h h, int* nnodes, int* ibeg, int* numpar,
                    int* level, int* nchild, double* geo);

/* Instrumentation (no counterpart in the reference, which only prints
 * cpu_time totals): every kernel launch of the library is counted per kernel
 * class; while profiling is enabled each launch is also timed with CUDA
 * events recorded on the stream it is launched on.  tabi_profile_enable
 * resets the counters.  kclass -1 reads the sum over all classes. */
int tabi_profile_enable(tabi_h h, int enable);
int tabi_profile_read(tabi_h h, int kclass, double* ms, int64_t* launches);
int tabi_profile_nclasses(void);
const char* tabi_profile_class_name(int kclass);

/* FP64 pipe peak probe: runs a DFMA loop for about `ms` milliseconds and
 * returns the achieved FP64 FLOP/s (2 per FMA). */
int tabi_probe_fp64_peak(double ms, double* flops);
/* The same for the FP32 pipe (FFMA loop), the denominator of the
 * mixed-precision operator's roofline. */
int tabi_probe_fp32_peak(double ms, double* flops);

/* Accuracy reference (no counterpart in the reference, whose treecode is
 * checked against a direct sum only in its papers): the operator evaluated
 * by an FP64 direct sum over every source (COMPP_DIRECT_PB's kernels,
 * treecode3d_pb.f:919-1008, self term excluded) at nt targets of the current
 * face order (0-based; the tree order after tabi_build_tree).  x is 2 nface;
 * y receives [y1 of the targets; y2 of the targets] (2 nt).  Cost nt x nface
 * pair evaluations on the GPU. */
int tabi_direct_targets(tabi_h h, int nt, const int* targets, const double* x, double* y);

/* One shard of the operator (no counterpart in the reference, which is serial):
 * after tabi_build_tree, restricts tabi_matvec(_dev) and tabi_msolve(_dev) to
 * the targets [t0, t1) of the tree order (0-based, half-open, starting and
 * ending on leaf boundaries): only those entries of y / z are written, the
 * far and near interactions and the leaf blocks of other targets are not
 * computed (the cluster moments still are: every shard needs all of them).
 * The shards' slices then assemble the full vector (an all-gather), and the
 * solve runs across shards: tabi_solve / tabi_solve_dev on a restricted
 * handle need an exchange (tabi_set_exchange) and are refused
 * (TABI_ERR_STATE) without one.  (0, nface) lifts the restriction. */
int tabi_set_target_range(tabi_h h, int t0, int t1);

/* The exchange of a target-sharded solve (one handle per rank, each restricted
 * by tabi_set_target_range to its own leaf-aligned range): after every
 * operator and preconditioner application inside tabi_solve /
 * tabi_solve_dev, the library calls fn(user, v_dev, n2, t0, t1, stream) with
 * the device vector v_dev (n2 = 2 nface doubles) whose entries [t0, t1) and
 * [nface + t0, nface + t1) this rank has just computed, and the stream the
 * solve runs on; fn completes v_dev in place with the other ranks' slices
 * (an all-gather, ordered on that stream) and returns 0, or non-zero on
 * failure (the solve then fails with TABI_ERR_STATE).  Every rank then runs
 * the same GMRES on identical vectors, so all ranks take the same steps and
 * end with the same solution, which equals the unsharded solve's.  The
 * reference has no counterpart (its solve is one process, main.f90:87-124);
 * this replaces tabipb.sharded's host-side GMRES.  fn NULL removes it. */
typedef int (*tabi_exchange_fn)(void* user, double* v_dev, int n2, int t0, int t1,
                                void* stream);
int tabi_set_exchange(tabi_h h, tabi_exchange_fn fn, void* user);

/* main.f90:226-326 output_potential, after tabi_build_tree: x (2 nface) is
 * the solution in tree order as tabi_solve returns it; x_orig receives it in
 * the original face order and vert_ptl (2 per vertex: potential, normal
 * derivative) the inverse-distance weighted average over the faces that use
 * each vertex (at most 14, the first in face order, as the reference's
 * 15-row table), both scaled by 332.0716 * 4 pi.  sptpos 3 x nspt, nvert
 * 3 x nface 1-based (the faces given to tabi_form_matrix).  A vertex that no
 * face uses gets 0/0 (NaN), as in the reference.  The writer of
 * surface_potential.dat stays with the caller (main.f90:307-318). */
int tabi_output_potential(tabi_h h, int nspt, const double* sptpos, int nface,
                          const int* nvert, const double* x, double* x_orig,
                          double* vert_ptl);
int tabi_output_potential_dev(tabi_h h, int nspt, const double* sptpos_dev, int nface,
                              const int* nvert_dev, const double* x_dev, double* x_orig_dev,
                              double* vert_ptl_dev, void* stream);

/* ---- Learned warm start (no counterpart in the reference, which starts
 * GMRES from zero, main.f90:133).  A rotation- and translation-invariant
 * point-cloud network over the panels (16 nearest neighbours per panel,
 * `layers` residual message-passing layers of width `hidden`, bfloat16 weight
 * matrices with FP32 accumulation) predicts x0 = [phi; dphi/dn] from the
 * panel geometry and the right-hand side; GMRES on the true residual then
 * runs from x0, so the prediction changes the iteration count only.  The
 * network corrects zprec = M^-1 bvct, the leaf-block preconditioner's solution
 * (tabi_msolve of the right-hand side; it solves the equations exactly within
 * each leaf), which is also one of its inputs; zprec may be NULL, the
 * baseline is then [0; b2].  The
 * network trains on the GPU (its own forward, backward and Adam kernels) on
 * solutions of this solver.  All surface arrays are device pointers in the
 * reference's layout (tr_xyz, tr_q 3 x nface, tr_area nface, bvct and x
 * 2 nface), in any one face order.  The _dev calls are ordered on `stream`
 * (NULL = the CUDA default stream); the loss / graph calls return after their
 * results are on the host.  A network object is not thread-safe. */
typedef struct tabi_ws_s* tabi_ws;

/* hidden: multiple of 32 in 32..256; layers 1..8; deterministic init from
 * seed (output layer zero: an untrained network predicts the baseline). */
int tabi_ws_create(tabi_ws* w, int hidden, int layers, unsigned long long seed);
int tabi_ws_destroy(tabi_ws w);
/* number of FP32 parameters (-1 for a NULL network) */
long long tabi_ws_nparams(tabi_ws w);
/* FP32 master parameters (host arrays of tabi_ws_nparams floats); set also
 * resets the optimiser state */
int tabi_ws_get_params(tabi_ws w, float* theta, long long n);
int tabi_ws_set_params(tabi_ws w, const float* theta, long long n);
/* x0 (device, 2 nface) = the network's prediction */
int tabi_ws_predict_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                        const double* tr_area, const double* bvct, const double* zprec,
                        double* x0, void* stream);
/* loss against a solution x_target (device, 2 nface) and, if grad != NULL,
 * its gradient with respect to the parameters (host, tabi_ws_nparams) */
int tabi_ws_loss_grad_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                          const double* tr_area, const double* bvct, const double* zprec,
                          const double* x_target, double* loss, float* grad,
                          void* stream);
/* one Adam step (beta 0.9 / 0.999) on one molecule; *loss (may be NULL) =
 * the loss before the step */
int tabi_ws_train_step_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                           const double* tr_area, const double* bvct, const double* zprec,
                           const double* x_target, double lr, double* loss,
                           void* stream);
/* the network's input: neighbour lists (host, nface x 16) and node features
 * (host, nface x 10); either may be NULL */
int tabi_ws_graph_dev(tabi_ws w, int nface, const double* tr_xyz, const double* tr_q,
                      const double* tr_area, const double* bvct, const double* zprec,
                      int* nbr, float* feat, void* stream);
/* attaches a network to a solve handle (NULL detaches): tabi_run_dev then
 * applies the preconditioner to the right-hand side and starts GMRES from the
 * network's correction of it instead of zero.  The handle does not own the
 * network. */
int tabi_set_warmstart(tabi_h h, tabi_ws w);

/* ---- Batched solves (no counterpart in the reference, which solves one
 * molecule per run).  One molecule: device inputs as tabi_run_dev takes them,
 * plus per-molecule overrides of the leaf size and Taylor order (0 = the batch
 * parameters'), e.g. from an autotuned table. */
typedef struct {
  int nspt;
  const double* sptpos;  /* 3 x nspt */
  const double* sptnrm;  /* 3 x nspt */
  int nface;
  const int* nvert;      /* 3 x nface, 1-based, already face-filtered */
  int nchr;
  const double* chrpos;  /* 3 x nchr */
  const double* atmchr;  /* nchr */
  int maxparnode;
  int order;
} tabi_mol_dev;

#define TABI_BATCH_STATS 12
/* Solves nmol molecules with nworkers host threads, each owning a handle (and
 * its two streams) on the current device, so that the latency-bound phases of
 * one molecule (panel factorisations, triangular solves, GMRES reductions)
 * overlap the work of others; molecules are taken largest first.  With a
 * warm-start network each worker uses its own copy.  stats (may be NULL)
 * receives TABI_BATCH_STATS doubles per molecule, in input order: the 8 of
 * tabi_run_dev, the molecule's wall time (ms), its completion time since the
 * batch started (ms), the worker index and the leaf size used. */
int tabi_batch_run_dev(const tabi_params* p, int nmol, const tabi_mol_dev* mols, tabi_ws ws,
                       int nworkers, double* stats);

#ifdef __cplusplus
}
#endif
#endif /* TABI_GPU_H */
