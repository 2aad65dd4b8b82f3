/*
 * tabi_oracle.h -- CPU oracle for the TABI-PB solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Fortran solver (gengwh/TABI-PB, src/main.f90, src/treecode3d_pb.f,
 * src/dgmres_dep.f, src/dgetrf_dep.f, src/readin.f90).  Only the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker / CPU baseline -- the product path (libtabi_gpu.so)
 * never calls into it.
 *
 * Parity status: the reference is Fortran and no Fortran compiler exists in
 * the build image, and the reference ships no golden outputs, so agreement of
 * this restatement with the reference binary's own output is UNPINNED.  It is
 * checked instead against the analytic Kirkwood/Born energy and against an
 * FP64 O(N^2) direct sum (tests/test_oracle.py).
 *
 * Conventions: arrays are column-major like the Fortran (tr_xyz is 3 x N,
 * point i at tr_xyz[3*i..3*i+2]); face vertex indices (nvert) and orderarr are
 * 1-based like the reference; vectors of length 2N are [x1 ; x2].
 */
#ifndef TABI_ORACLE_H
#define TABI_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_tree or_tree;

/* readin.f90:264-333 surface_area: drops faces with Heron area < 1e-5 or a
 * centroid within squared distance 1e-5 of one of the 10 previous faces.
 * nvert (3 x nface, 1-based) is compacted in place; returns the new nface. */
int or_surface_area(int nspt, const double* sptpos, int nface, int* nvert,
                    double* s_area);

/* main.f90:546-610 form_matrix: centroids, unit normals, Heron areas, RHS. */
void or_form_matrix(int nspt, const double* sptpos, const double* sptnrm,
                    int nface, const int* nvert, int nchr,
                    const double* chrpos, const double* atmchr, double eps0,
                    double* tr_xyz, double* tr_q, double* tr_area,
                    double* bvct, int nthreads);

/* main.f90:329-464 treecode_initialization: SETUP + CREATE_TREE (with the
 * reference's in-place PARTITION, so orderarr matches the reference's), then
 * the tree-order permutation of tr_xyz, tr_q, tr_area and bvct (in place).
 * bvct may be NULL. */
or_tree* or_tree_create(int nface, double* tr_xyz, double* tr_q,
                        double* tr_area, double* bvct, int order,
                        int maxparnode, double theta, int* orderarr,
                        int* nleaf);
void or_tree_free(or_tree* t);
int or_tree_num_nodes(const or_tree* t);
/* Node table in creation (depth-first) order: per node ibeg,iend (1-based),
 * level, num_children; geo = x_mid,y_mid,z_mid,radius. */
void or_tree_nodes(const or_tree* t, int* ibeg, int* iend, int* level,
                   int* nchild, double* geo);

/* main.f90:467-488 MATVECmain -> treecode3d_pb.f:1130-1189 TREE_COMPP_PB.
 * counts (may be NULL): [0] near-field pairs, [1] far (target, cluster)
 * interactions.  nthreads > 1 splits the target loop over OpenMP threads. */
void or_matvec(or_tree* t, double kappa, double eps, const double* x,
               double* y, int64_t* counts, int nthreads);
/* Same operator on a subset of targets [i0, i1) (0-based, tree order);
 * y receives entries i and N+i for those targets only.  Used to time a
 * bounded sample of a matvec. */
void or_matvec_range(or_tree* t, double kappa, double eps, const double* x,
                     double* y, int i0, int i1, int64_t* counts,
                     int nthreads);

/* The two halves of or_matvec_range: pb_kernel + moments, then the target
 * loop over [i0, i1) (used to time a bounded sample). */
void or_matvec_prepare(or_tree* t, const double* x);
void or_matvec_targets(or_tree* t, double kappa, double eps, const double* x,
                       double* y, int i0, int i1, int64_t* counts,
                       int nthreads);

/* FP64 O(N^2) direct sum of the same four kernels (no treecode). */
void or_matvec_direct(int n, const double* tr_xyz, const double* tr_q,
                      const double* tr_area, double kappa, double eps,
                      const double* x, double* y, int nthreads);

/* treecode3d_pb.f:1393-1542 LEAFMATVECpara (block-diagonal preconditioner:
 * assemble each leaf block, DGETRF + DGETRS).  Returns the number of leaves
 * whose DGETRF reported info != 0.  leaf0/leaf1 restrict to a leaf range
 * (pass 0, -1 for all). */
int or_msolve_block(or_tree* t, double kappa, double eps, const double* r,
                    double* z, int leaf0, int leaf1, int nthreads);
/* main.f90:532-542 MSOLVEprec (diagonal scaling). */
void or_msolve_diag(int n2, double eps, const double* r, double* z);
int or_tree_num_leaves(const or_tree* t);
/* leaf ibeg (1-based) and size, leaves in tree order. */
void or_tree_leaves(const or_tree* t, int* ibeg, int* nrow);

/* dgetrf_dep.f:757-900 DGETRF2 and :346-445 DGETRS (column-major, 1-based
 * pivots).  Exposed for unit tests. */
int or_dgetrf(int m, int n, double* a, int lda, int* ipiv);
void or_dgetrs(int n, int nrhs, const double* a, int lda, const int* ipiv,
               double* b, int ldb);

/* dgmres_dep.f DGMRES driven by the tree operator: main.f90:92-139
 * settings (ITOL=2, JPRE=-1 (iprcd=1) or JPRE=-1 with diagonal MSOLVE,
 * JSCAL=0, MAXL, NRMAX, tol).  x holds x0 on entry.  err_hist (may be NULL,
 * length >= (nrmax+1)*maxl+1) receives the 'LL err=' values printed by
 * dgmres_dep.f:1796; n_hist its count.  Returns IERR. */
int or_dgmres(or_tree* t, double kappa, double eps, int iprcd,
              const double* b, double* x, double tol, int maxl, int nrmax,
              int* iter, double* err, double* err_hist, int* n_hist,
              int64_t* n_matvec, int64_t* n_msolve, int nthreads);

/* main.f90:144-157 + 614-657: solvation energy (kcal/mol) and Coulomb energy
 * from the converged x (tree order, with the tree's permuted surface). */
void or_energy(const or_tree* t, int nchr, const double* chrpos,
               const double* atmchr, double kappa, double eps, double eps0,
               const double* x, double* soleng, double* couleng,
               int nthreads);
/* Same with explicit surface arrays (any order). */
void or_energy_surface(int nface, const double* tr_xyz, const double* tr_q,
                       const double* tr_area, int nchr, const double* chrpos,
                       const double* atmchr, double kappa, double eps,
                       double eps0, const double* x, double* soleng,
                       double* couleng, int nthreads);

/* main.f90:62-65 constants: kappa from the REAL*4 literal 8.430325455. */
double or_kappa(double bulk_strength, double eps1);

/* main.f90:226-326 output_potential (vertex potentials; see tabi_oracle.c) */
void or_output_potential(int nspt, const double* sptpos, int nface, const int* nvert,
                         const double* tr_xyz, const double* x_orig, double* vert_ptl,
                         double* x_scaled);

#ifdef __cplusplus
}
#endif
#endif
