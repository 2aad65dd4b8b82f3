/*
 * tabi_oracle.c -- CPU oracle for the TABI-PB solve path.
 *
 * TEST INFRASTRUCTURE ONLY (see tabi_oracle.h): a plain-C restatement of the
 * reference Fortran (gengwh/TABI-PB).  Each function cites the reference
 * lines it follows.  Parity with the reference binary is UNPINNED (no
 * Fortran compiler in the build image, no golden outputs in the reference);
 * the restatement is checked against the analytic Born energy and an FP64
 * direct sum.
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp (oracle/Makefile).  The
 * reference is built by gfortran -O2 on x86-64 (src/Makefile:6-7), which
 * emits no fused multiply-adds and does not reassociate; -ffp-contract=off
 * keeps this file to the same IEEE evaluation, and every expression keeps the
 * Fortran's left-to-right operand order.
 */
#include "tabi_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_F (acos(-1.0))

static double dot3(const double* a, const double* b) {
  /* gfortran dot_product of length 3: (a1*b1 + a2*b2) + a3*b3 */
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* readin.f90:336-340 */
static double triangle_area(double aa, double bb, double cc) {
  double s = 0.5 * (aa + bb + cc);
  return sqrt(s * (s - aa) * (s - bb) * (s - cc));
}

static double dist3(const double* p, const double* q) {
  double d[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
  return sqrt(dot3(d, d));
}

/* readin.f90:264-333 */
int or_surface_area(int nspt, const double* sptpos, int nface, int* nvert,
                    double* s_area) {
  (void)nspt;
  const double third = 1.0 / 3.0;
  int* copy = (int*)malloc(sizeof(int) * 3 * (size_t)(nface > 0 ? nface : 1));
  int nnew = 0;
  double area_sum = 0.0;
  for (int i = 0; i < nface; ++i) {
    double face[3][3], xx[3] = {0, 0, 0};
    for (int j = 0; j < 3; ++j) {
      const double* p = sptpos + 3 * (size_t)(nvert[3 * i + j] - 1);
      for (int d = 0; d < 3; ++d) {
        face[j][d] = p[d];
        xx[d] = xx[d] + third * p[d];
      }
    }
    double aa = dist3(face[0], face[1]);
    double bb = dist3(face[0], face[2]);
    double cc = dist3(face[1], face[2]);
    double area_local = triangle_area(aa, bb, cc);
    int alert = 0;
    /* the reference compares against the previous 10 faces of the ORIGINAL
     * list (deleted ones included) */
    for (int ii = (i - 10 > 0 ? i - 10 : 0); ii < i; ++ii) {
      double yy[3] = {0, 0, 0};
      for (int j = 0; j < 3; ++j) {
        const double* p = sptpos + 3 * (size_t)(nvert[3 * ii + j] - 1);
        for (int d = 0; d < 3; ++d) yy[d] = yy[d] + third * p[d];
      }
      double df[3] = {xx[0] - yy[0], xx[1] - yy[1], xx[2] - yy[2]};
      if (dot3(df, df) < 1e-5) alert = 1;
    }
    if (!(area_local < 1e-5 || alert)) {
      copy[3 * nnew + 0] = nvert[3 * i + 0];
      copy[3 * nnew + 1] = nvert[3 * i + 1];
      copy[3 * nnew + 2] = nvert[3 * i + 2];
      ++nnew;
    }
    area_sum = area_sum + area_local;
  }
  memcpy(nvert, copy, sizeof(int) * 3 * (size_t)nnew);
  free(copy);
  if (s_area) *s_area = area_sum;
  return nnew;
}

/* main.f90:546-610 */
void or_form_matrix(int nspt, const double* sptpos, const double* sptnrm,
                    int nface, const int* nvert, int nchr,
                    const double* chrpos, const double* atmchr, double eps0,
                    double* tr_xyz, double* tr_q, double* tr_area,
                    double* bvct, int nthreads) {
  (void)nspt;
  const double pi = PI_F;
  const double third = 1.0 / 3.0;
  for (int i = 0; i < 2 * nface; ++i) bvct[i] = 0.0;
  /* faces are independent: threads change nothing in the results */
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static)
  for (int i = 0; i < nface; ++i) {
    double r0[3] = {0, 0, 0}, v0[3] = {0, 0, 0}, r[3][3];
    for (int k = 0; k < 3; ++k) {
      int id = nvert[3 * i + k] - 1;
      for (int d = 0; d < 3; ++d) {
        r0[d] = r0[d] + third * sptpos[3 * (size_t)id + d];
        v0[d] = v0[d] + third * sptnrm[3 * (size_t)id + d];
        r[k][d] = sptpos[3 * (size_t)id + d];
      }
    }
    double nv = sqrt(dot3(v0, v0));
    for (int d = 0; d < 3; ++d) v0[d] = v0[d] / nv;
    for (int d = 0; d < 3; ++d) {
      tr_xyz[3 * (size_t)i + d] = r0[d];
      tr_q[3 * (size_t)i + d] = v0[d];
    }
    double aa = dist3(r[0], r[1]);
    double bb = dist3(r[0], r[2]);
    double cc = dist3(r[1], r[2]);
    tr_area[i] = triangle_area(aa, bb, cc);
    double b1 = 0.0, b2 = 0.0;
    for (int j = 0; j < nchr; ++j) {
      const double* rr = chrpos + 3 * (size_t)j;
      double d[3] = {rr[0] - r0[0], rr[1] - r0[1], rr[2] - r0[2]};
      double rs = sqrt(dot3(d, d));
      double G0 = 1.0 / (4.0 * pi * rs);
      double cos_theta = dot3(v0, d) / rs;
      double G1 = cos_theta / (rs * rs) / 4.0 / pi;
      b1 = b1 + atmchr[j] * G0 / eps0;
      b2 = b2 + atmchr[j] * G1 / eps0;
    }
    bvct[i] = b1;
    bvct[nface + i] = b2;
  }
}

double or_kappa(double bulk_strength, double eps1) {
  /* main.f90:62-63: the literal 8.430325455 is default REAL (REAL*4) */
  double kappa2 = (double)(float)8.430325455 * bulk_strength / eps1;
  return sqrt(kappa2);
}

/* ------------------------------------------------------------------ */
/* tree (treecode3d_pb.f:38-47 tnode, :54-356 SETUP/CREATE_TREE/PARTITION_8,
 * :1677-1759 PARTITION)                                                */

typedef struct {
  int numpar, ibeg, iend; /* 1-based */
  double x_min, y_min, z_min, x_max, y_max, z_max;
  double x_mid, y_mid, z_mid, radius;
  int level, num_children;
  int child[8];
  int mslot; /* moment slot, -1 if numpar <= 40 */
} or_node;

struct or_tree {
  int n, order, maxparnode;
  double theta;
  int torder, torderlim;
  double *x, *y, *z, *q; /* tree order, 1-based access via X(i) */
  double* tq;            /* 3 x n normals, tree order */
  double* area;          /* n, tree order */
  int* orderarr;         /* 1-based original index per tree slot */
  or_node* nodes;
  int nnodes, cap;
  int nleaf;
  int *leaf_ibeg, *leaf_n;
  double *cf1, *cf2, *cf3;
  double* der_cof; /* [idx][k][j][i], (order+1)^3 x 16 */
  int kk[16][3];
  int nmslot;
  double* ms; /* [slot][16][(torder+1)^3] */
  double* schg; /* 16 x n (idx-major) source charges, tree order */
  double* tchg; /* 16 x n target charges */
};

/* PARTITION (treecode3d_pb.f:1677-1759): in-place, 1-based indices */
static void partition(double* a, double* b, double* c, double* q, int* ind,
                      int ibeg, int iend, double val, int* midind) {
#define A_(i) a[(i)-1]
#define B_(i) b[(i)-1]
#define C_(i) c[(i)-1]
#define Q_(i) q[(i)-1]
#define I_(i) ind[(i)-1]
  if (ibeg < iend) {
    double ta = A_(ibeg), tb = B_(ibeg), tc = C_(ibeg), tq = Q_(ibeg);
    int tind = I_(ibeg);
    A_(ibeg) = val;
    int upper = ibeg, lower = iend;
    while (upper != lower) {
      while (upper < lower && val < A_(lower)) lower = lower - 1;
      if (upper != lower) {
        A_(upper) = A_(lower);
        B_(upper) = B_(lower);
        C_(upper) = C_(lower);
        Q_(upper) = Q_(lower);
        I_(upper) = I_(lower);
      }
      while (upper < lower && val >= A_(upper)) upper = upper + 1;
      if (upper != lower) {
        A_(lower) = A_(upper);
        B_(lower) = B_(upper);
        C_(lower) = C_(upper);
        Q_(lower) = Q_(upper);
        I_(lower) = I_(upper);
      }
    }
    *midind = upper;
    if (ta > val) *midind = upper - 1;
    A_(upper) = ta;
    B_(upper) = tb;
    C_(upper) = tc;
    Q_(upper) = tq;
    I_(upper) = tind;
  } else if (ibeg == iend) {
    *midind = (A_(ibeg) <= val) ? ibeg : ibeg - 1;
  } else {
    *midind = ibeg - 1;
  }
#undef A_
#undef B_
#undef C_
#undef Q_
#undef I_
}

/* PARTITION_8 (treecode3d_pb.f:284-356); ind[8][2], xyzmms[8][6] */
static void partition_8(or_tree* t, double xyzmms[8][6], double xl, double yl,
                        double zl, double lmax, int* numposchild,
                        double x_mid, double y_mid, double z_mid,
                        int ind[8][2]) {
  int temp_ind;
  int npc = 1;
  double critlen = lmax / sqrt(2.0);
  if (xl >= critlen) {
    partition(t->x, t->y, t->z, t->q, t->orderarr, ind[0][0], ind[0][1],
              x_mid, &temp_ind);
    ind[1][0] = temp_ind + 1;
    ind[1][1] = ind[0][1];
    ind[0][1] = temp_ind;
    memcpy(xyzmms[1], xyzmms[0], sizeof(double) * 6);
    xyzmms[0][1] = x_mid;
    xyzmms[1][0] = x_mid;
    npc = 2 * npc;
  }
  if (yl >= critlen) {
    for (int i = 0; i < npc; ++i) {
      partition(t->y, t->x, t->z, t->q, t->orderarr, ind[i][0], ind[i][1],
                y_mid, &temp_ind);
      ind[npc + i][0] = temp_ind + 1;
      ind[npc + i][1] = ind[i][1];
      ind[i][1] = temp_ind;
      memcpy(xyzmms[npc + i], xyzmms[i], sizeof(double) * 6);
      xyzmms[i][3] = y_mid;
      xyzmms[npc + i][2] = y_mid;
    }
    npc = 2 * npc;
  }
  if (zl >= critlen) {
    for (int i = 0; i < npc; ++i) {
      partition(t->z, t->x, t->y, t->q, t->orderarr, ind[i][0], ind[i][1],
                z_mid, &temp_ind);
      ind[npc + i][0] = temp_ind + 1;
      ind[npc + i][1] = ind[i][1];
      ind[i][1] = temp_ind;
      memcpy(xyzmms[npc + i], xyzmms[i], sizeof(double) * 6);
      xyzmms[i][5] = z_mid;
      xyzmms[npc + i][4] = z_mid;
    }
    npc = 2 * npc;
  }
  *numposchild = npc;
}

static int new_node(or_tree* t) {
  if (t->nnodes == t->cap) {
    t->cap = t->cap ? 2 * t->cap : 64;
    t->nodes = (or_node*)realloc(t->nodes, sizeof(or_node) * (size_t)t->cap);
  }
  memset(&t->nodes[t->nnodes], 0, sizeof(or_node));
  return t->nnodes++;
}

static void minmax(const double* v, int i0, int i1, double* mn, double* mx) {
  double a = v[i0 - 1], b = v[i0 - 1];
  for (int i = i0; i <= i1; ++i) {
    if (v[i - 1] < a) a = v[i - 1];
    if (v[i - 1] > b) b = v[i - 1];
  }
  *mn = a;
  *mx = b;
}

/* CREATE_TREE (treecode3d_pb.f:142-281) */
static int create_tree(or_tree* t, int ibeg, int iend, const double* xyzmm,
                       int level) {
  int id = new_node(t);
  or_node* p = &t->nodes[id];
  p->numpar = iend - ibeg + 1;
  p->x_min = xyzmm[0];
  p->x_max = xyzmm[1];
  p->y_min = xyzmm[2];
  p->y_max = xyzmm[3];
  p->z_min = xyzmm[4];
  p->z_max = xyzmm[5];
  double xl = p->x_max - p->x_min;
  double yl = p->y_max - p->y_min;
  double zl = p->z_max - p->z_min;
  double lmax = xl;
  if (yl > lmax) lmax = yl;
  if (zl > lmax) lmax = zl;
  p->x_mid = (p->x_max + p->x_min) / 2.0;
  p->y_mid = (p->y_max + p->y_min) / 2.0;
  p->z_mid = (p->z_max + p->z_min) / 2.0;
  double t1 = p->x_max - p->x_mid;
  double t2 = p->y_max - p->y_mid;
  double t3 = p->z_max - p->z_mid;
  p->radius = sqrt(t1 * t1 + t2 * t2 + t3 * t3);
  p->ibeg = ibeg;
  p->iend = iend;
  p->level = level;
  p->num_children = 0;
  p->mslot = -1;
  if (p->numpar > t->maxparnode) {
    double xyzmms[8][6];
    int ind[8][2];
    memset(ind, 0, sizeof(ind));
    xyzmms[0][0] = p->x_min;
    xyzmms[0][1] = p->x_max;
    xyzmms[0][2] = p->y_min;
    xyzmms[0][3] = p->y_max;
    xyzmms[0][4] = p->z_min;
    xyzmms[0][5] = p->z_max;
    ind[0][0] = ibeg;
    ind[0][1] = iend;
    int numposchild;
    partition_8(t, xyzmms, xl, yl, zl, lmax, &numposchild, p->x_mid,
                p->y_mid, p->z_mid, ind);
    /* shrink the boxes of children holding >= 2 particles (:249-258) */
    for (int i = 0; i < 8; ++i) {
      if (ind[i][0] < ind[i][1]) {
        minmax(t->x, ind[i][0], ind[i][1], &xyzmms[i][0], &xyzmms[i][1]);
        minmax(t->y, ind[i][0], ind[i][1], &xyzmms[i][2], &xyzmms[i][3]);
        minmax(t->z, ind[i][0], ind[i][1], &xyzmms[i][4], &xyzmms[i][5]);
      }
    }
    int kids[8], nk = 0;
    for (int i = 0; i < numposchild; ++i) {
      if (ind[i][0] <= ind[i][1]) {
        kids[nk++] = create_tree(t, ind[i][0], ind[i][1], xyzmms[i],
                                 level + 1);
      }
    }
    p = &t->nodes[id]; /* realloc may have moved the table */
    p->num_children = nk;
    for (int i = 0; i < nk; ++i) p->child[i] = kids[i];
  } else {
    t->nleaf++;
  }
  return id;
}

static void collect_leaves(or_tree* t, int id, int* k) {
  or_node* p = &t->nodes[id];
  if (p->num_children == 0) {
    t->leaf_ibeg[*k] = p->ibeg;
    t->leaf_n[*k] = p->numpar;
    (*k)++;
  } else {
    for (int i = 0; i < p->num_children; ++i)
      collect_leaves(t, p->child[i], k);
  }
}

/* main.f90:329-464 treecode_initialization + treecode3d_pb.f:54-139 SETUP */
or_tree* or_tree_create(int nface, double* tr_xyz, double* tr_q,
                        double* tr_area, double* bvct, int order,
                        int maxparnode, double theta, int* orderarr,
                        int* nleaf) {
  or_tree* t = (or_tree*)calloc(1, sizeof(or_tree));
  int n = nface;
  t->n = n;
  t->order = order;
  t->maxparnode = maxparnode;
  t->theta = theta;
  t->torder = order + 2;
  t->torderlim = t->torder + 1; /* iflag is never set: orderoffset = 1 */
  t->x = (double*)malloc(sizeof(double) * (size_t)n);
  t->y = (double*)malloc(sizeof(double) * (size_t)n);
  t->z = (double*)malloc(sizeof(double) * (size_t)n);
  t->q = (double*)malloc(sizeof(double) * (size_t)n);
  t->orderarr = (int*)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; ++i) {
    t->x[i] = tr_xyz[3 * (size_t)i + 0];
    t->y[i] = tr_xyz[3 * (size_t)i + 1];
    t->z[i] = tr_xyz[3 * (size_t)i + 2];
    t->q[i] = 1.0;
    t->orderarr[i] = i + 1;
  }
  /* Taylor tables (SETUP :107-116) */
  t->cf1 = (double*)calloc((size_t)t->torderlim + 1, sizeof(double));
  t->cf2 = (double*)calloc((size_t)t->torderlim + 1, sizeof(double));
  t->cf3 = (double*)calloc((size_t)t->torderlim + 1, sizeof(double));
  for (int i = 1; i <= t->torderlim; ++i) {
    double t1 = 1.0 / (double)i;
    t->cf1[i] = t1;
    t->cf2[i] = 1.0 - 0.5 * t1;
    t->cf3[i] = 1.0 - t1;
  }
  /* kk and der_cof (main.f90:357-399) */
  static const int kk[16][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                {1, 1, 0}, {1, 0, 1}, {1, 1, 0}, {0, 2, 0},
                                {0, 1, 1}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};
  memcpy(t->kk, kk, sizeof(kk));
  int P1 = order + 1;
  t->der_cof = (double*)malloc(sizeof(double) * 16 * (size_t)P1 * P1 * P1);
  const double one_over_4pi = 0.25 / PI_F;
  for (int idx = 0; idx < 16; ++idx)
    for (int k = 0; k <= order; ++k)
      for (int j = 0; j <= order; ++j)
        for (int i = 0; i <= order; ++i) {
          double v = 1.0;
          if (i + j + k <= order) {
            int ijk[3] = {i, j, k};
            for (int mm = 0; mm < 3; ++mm)
              for (int nn = 1; nn <= kk[idx][mm]; ++nn)
                v = v * (double)(ijk[mm] + nn);
          }
          t->der_cof[(((size_t)idx * P1 + k) * P1 + j) * P1 + i] =
              v * one_over_4pi;
        }
  /* bounding box (SETUP :120-125) and tree */
  double xyzmm[6];
  minmax(t->x, 1, n, &xyzmm[0], &xyzmm[1]);
  minmax(t->y, 1, n, &xyzmm[2], &xyzmm[3]);
  minmax(t->z, 1, n, &xyzmm[4], &xyzmm[5]);
  t->nleaf = 0;
  create_tree(t, 1, n, xyzmm, 0);
  t->leaf_ibeg = (int*)malloc(sizeof(int) * (size_t)t->nleaf);
  t->leaf_n = (int*)malloc(sizeof(int) * (size_t)t->nleaf);
  int k = 0;
  collect_leaves(t, 0, &k);
  /* moment slots for every node that can pass the MAC (numpar > 40) */
  t->nmslot = 0;
  for (int i = 0; i < t->nnodes; ++i)
    if (t->nodes[i].numpar > 40) t->nodes[i].mslot = t->nmslot++;
  int T1 = t->torder + 1;
  t->ms = (double*)calloc((size_t)(t->nmslot > 0 ? t->nmslot : 1) * 16 * T1 *
                              T1 * T1,
                          sizeof(double));
  t->schg = (double*)malloc(sizeof(double) * 16 * (size_t)n);
  t->tchg = (double*)malloc(sizeof(double) * 16 * (size_t)n);
  /* permutation (main.f90:443-453) */
  t->tq = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  t->area = (double*)malloc(sizeof(double) * (size_t)n);
  double* tmpb = bvct ? (double*)malloc(sizeof(double) * 2 * (size_t)n) : 0;
  if (bvct) memcpy(tmpb, bvct, sizeof(double) * 2 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    int o = t->orderarr[i] - 1;
    t->area[i] = tr_area[o];
    for (int d = 0; d < 3; ++d) t->tq[3 * (size_t)i + d] = tr_q[3 * (size_t)o + d];
    if (bvct) {
      bvct[i] = tmpb[o];
      bvct[i + n] = tmpb[o + n];
    }
  }
  for (int i = 0; i < n; ++i) {
    tr_area[i] = t->area[i];
    for (int d = 0; d < 3; ++d) tr_q[3 * (size_t)i + d] = t->tq[3 * (size_t)i + d];
    tr_xyz[3 * (size_t)i + 0] = t->x[i];
    tr_xyz[3 * (size_t)i + 1] = t->y[i];
    tr_xyz[3 * (size_t)i + 2] = t->z[i];
  }
  free(tmpb);
  if (orderarr) memcpy(orderarr, t->orderarr, sizeof(int) * (size_t)n);
  if (nleaf) *nleaf = t->nleaf;
  return t;
}

void or_tree_free(or_tree* t) {
  if (!t) return;
  free(t->x);
  free(t->y);
  free(t->z);
  free(t->q);
  free(t->tq);
  free(t->area);
  free(t->orderarr);
  free(t->nodes);
  free(t->leaf_ibeg);
  free(t->leaf_n);
  free(t->cf1);
  free(t->cf2);
  free(t->cf3);
  free(t->der_cof);
  free(t->ms);
  free(t->schg);
  free(t->tchg);
  free(t);
}

int or_tree_num_nodes(const or_tree* t) { return t->nnodes; }
int or_tree_num_leaves(const or_tree* t) { return t->nleaf; }

void or_tree_nodes(const or_tree* t, int* ibeg, int* iend, int* level,
                   int* nchild, double* geo) {
  for (int i = 0; i < t->nnodes; ++i) {
    const or_node* p = &t->nodes[i];
    ibeg[i] = p->ibeg;
    iend[i] = p->iend;
    level[i] = p->level;
    nchild[i] = p->num_children;
    geo[4 * i + 0] = p->x_mid;
    geo[4 * i + 1] = p->y_mid;
    geo[4 * i + 2] = p->z_mid;
    geo[4 * i + 3] = p->radius;
  }
}

void or_tree_leaves(const or_tree* t, int* ibeg, int* nrow) {
  memcpy(ibeg, t->leaf_ibeg, sizeof(int) * (size_t)t->nleaf);
  memcpy(nrow, t->leaf_n, sizeof(int) * (size_t)t->nleaf);
}

/* ------------------------------------------------------------------ */
/* matvec                                                              */

/* main.f90:664-694 pb_kernel: 16 target and source charges (tree order).
 * Both kappa slots of the reference hold identical values, one is kept. */
static void pb_kernel(or_tree* t, const double* phi) {
  int n = t->n;
  for (int i = 0; i < n; ++i) {
    double A = t->area[i], x1 = phi[i], x2 = phi[n + i];
    const double* v = t->tq + 3 * (size_t)i;
    int idx = 0;
    t->tchg[(size_t)idx * n + i] = 1.0;
    t->schg[(size_t)idx * n + i] = A * x2;
    idx++;
    for (int iknl = 1; iknl <= 2; ++iknl)
      for (int d = 0; d < 3; ++d) {
        t->tchg[(size_t)idx * n + i] =
            1.0 * (double)(2 - iknl) + v[d] * (double)(iknl - 1);
        double phiv = (iknl == 1) ? x1 : x2;
        t->schg[(size_t)idx * n + i] =
            (v[d] * (double)(2 - iknl) + 1.0 * (double)(iknl - 1)) * A * phiv;
        idx++;
      }
    for (int ixyz = 0; ixyz < 3; ++ixyz)
      for (int jxyz = 0; jxyz < 3; ++jxyz) {
        t->tchg[(size_t)idx * n + i] = v[jxyz];
        t->schg[(size_t)idx * n + i] = -(v[ixyz] * A * x1);
        idx++;
      }
  }
}

#define MSI(t, k1, k2, k3) \
  ((((size_t)(k3) * ((t)->torder + 1) + (k2)) * ((t)->torder + 1)) + (k1))

/* COMP_MS (treecode3d_pb.f:859-916), done for every node that can pass the
 * MAC before the target loop (the reference computes the same values
 * lazily on first acceptance). */
static void comp_ms(or_tree* t, const or_node* p) {
  int T1 = t->torder + 1;
  size_t T3 = (size_t)T1 * T1 * T1;
  double* ms = t->ms + (size_t)p->mslot * 16 * T3;
  memset(ms, 0, sizeof(double) * 16 * T3);
  int n = t->n;
  static const int comp[10] = {0, 1, 2, 3, 4, 5, 6, 7, 10, 13};
  for (int i = p->ibeg; i <= p->iend; ++i) {
    double dx = t->x[i - 1] - p->x_mid;
    double dy = t->y[i - 1] - p->y_mid;
    double dz = t->z[i - 1] - p->z_mid;
    double tz = 1.0;
    for (int k3 = 0; k3 <= t->torder; ++k3) {
      double ty = 1.0;
      for (int k2 = 0; k2 <= t->torder - k3; ++k2) {
        double tx = 1.0;
        for (int k1 = 0; k1 <= t->torder - k3 - k2; ++k1) {
          double txyz = tx * ty * tz;
          for (int c = 0; c < 10; ++c) {
            int idx = comp[c];
            ms[(size_t)idx * T3 + MSI(t, k1, k2, k3)] +=
                t->schg[(size_t)idx * n + (i - 1)] * txyz;
          }
          tx = tx * dx;
        }
        ty = ty * dy;
      }
      tz = tz * dz;
    }
  }
  memcpy(ms + 8 * T3, ms + 7 * T3, sizeof(double) * T3);
  memcpy(ms + 9 * T3, ms + 7 * T3, sizeof(double) * T3);
  memcpy(ms + 11 * T3, ms + 10 * T3, sizeof(double) * T3);
  memcpy(ms + 12 * T3, ms + 10 * T3, sizeof(double) * T3);
  memcpy(ms + 14 * T3, ms + 13 * T3, sizeof(double) * T3);
  memcpy(ms + 15 * T3, ms + 13 * T3, sizeof(double) * T3);
}

typedef struct {
  int L;     /* torderlim */
  int D;     /* L + 3 (index range -2..L) */
  double *a, *b;
  double tarpos[3], tarq[3];
  double tempq[16];
  int64_t near_pairs, far_inter;
  int self; /* target index (1-based) */
} or_scratch;

#define AB(s, i, j, k) \
  ((((size_t)((k) + 2) * (s)->D + ((j) + 2)) * (s)->D) + ((i) + 2))

/* COMP_TCOEFF (treecode3d_pb.f:684-855) */
static void comp_tcoeff(const or_tree* t, or_scratch* s, const or_node* p,
                        double kappa) {
  double* a = s->a;
  double* b = s->b;
  int L = t->torderlim;
  const double *cf1 = t->cf1, *cf2 = t->cf2, *cf3 = t->cf3;
  double cf1_new[64];
  for (int i = 1; i <= L; ++i) cf1_new[i] = cf1[i] * kappa;
#define a_(i, j, k) a[AB(s, i, j, k)]
#define b_(i, j, k) b[AB(s, i, j, k)]
  double dx = s->tarpos[0] - p->x_mid;
  double dy = s->tarpos[1] - p->y_mid;
  double dz = s->tarpos[2] - p->z_mid;
  double ddx = 2.0 * dx, ddy = 2.0 * dy, ddz = 2.0 * dz;
  double kappax = kappa * dx, kappay = kappa * dy, kappaz = kappa * dz;
  double dist = dx * dx + dy * dy + dz * dz;
  double fac = 1.0 / dist;
  dist = sqrt(dist);
  b_(0, 0, 0) = exp(-kappa * dist);
  a_(0, 0, 0) = b_(0, 0, 0) / dist;
  b_(1, 0, 0) = kappax * a_(0, 0, 0);
  b_(0, 1, 0) = kappay * a_(0, 0, 0);
  b_(0, 0, 1) = kappaz * a_(0, 0, 0);
  a_(1, 0, 0) = fac * dx * (a_(0, 0, 0) + kappa * b_(0, 0, 0));
  a_(0, 1, 0) = fac * dy * (a_(0, 0, 0) + kappa * b_(0, 0, 0));
  a_(0, 0, 1) = fac * dz * (a_(0, 0, 0) + kappa * b_(0, 0, 0));
  for (int i = 2; i <= L; ++i) {
    b_(i, 0, 0) = cf1_new[i] * (dx * a_(i - 1, 0, 0) - a_(i - 2, 0, 0));
    b_(0, i, 0) = cf1_new[i] * (dy * a_(0, i - 1, 0) - a_(0, i - 2, 0));
    b_(0, 0, i) = cf1_new[i] * (dz * a_(0, 0, i - 1) - a_(0, 0, i - 2));
    a_(i, 0, 0) = fac * (ddx * cf2[i] * a_(i - 1, 0, 0) -
                         cf3[i] * a_(i - 2, 0, 0) +
                         cf1_new[i] * (dx * b_(i - 1, 0, 0) - b_(i - 2, 0, 0)));
    a_(0, i, 0) = fac * (ddy * cf2[i] * a_(0, i - 1, 0) -
                         cf3[i] * a_(0, i - 2, 0) +
                         cf1_new[i] * (dy * b_(0, i - 1, 0) - b_(0, i - 2, 0)));
    a_(0, 0, i) = fac * (ddz * cf2[i] * a_(0, 0, i - 1) -
                         cf3[i] * a_(0, 0, i - 2) +
                         cf1_new[i] * (dz * b_(0, 0, i - 1) - b_(0, 0, i - 2)));
  }
  b_(1, 1, 0) = kappax * a_(0, 1, 0);
  b_(1, 0, 1) = kappax * a_(0, 0, 1);
  b_(0, 1, 1) = kappay * a_(0, 0, 1);
  a_(1, 1, 0) = fac * (dx * a_(0, 1, 0) + ddy * a_(1, 0, 0) + kappax * b_(0, 1, 0));
  a_(1, 0, 1) = fac * (dx * a_(0, 0, 1) + ddz * a_(1, 0, 0) + kappax * b_(0, 0, 1));
  a_(0, 1, 1) = fac * (dy * a_(0, 0, 1) + ddz * a_(0, 1, 0) + kappay * b_(0, 0, 1));
  for (int i = 2; i <= L - 1; ++i) {
    b_(1, 0, i) = kappax * a_(0, 0, i);
    b_(0, 1, i) = kappay * a_(0, 0, i);
    b_(0, i, 1) = kappaz * a_(0, i, 0);
    b_(1, i, 0) = kappax * a_(0, i, 0);
    b_(i, 1, 0) = kappay * a_(i, 0, 0);
    b_(i, 0, 1) = kappaz * a_(i, 0, 0);
    a_(1, 0, i) = fac * (dx * a_(0, 0, i) + ddz * a_(1, 0, i - 1) -
                         a_(1, 0, i - 2) + kappax * b_(0, 0, i));
    a_(0, 1, i) = fac * (dy * a_(0, 0, i) + ddz * a_(0, 1, i - 1) -
                         a_(0, 1, i - 2) + kappay * b_(0, 0, i));
    a_(0, i, 1) = fac * (dz * a_(0, i, 0) + ddy * a_(0, i - 1, 1) -
                         a_(0, i - 2, 1) + kappaz * b_(0, i, 0));
    a_(1, i, 0) = fac * (dx * a_(0, i, 0) + ddy * a_(1, i - 1, 0) -
                         a_(1, i - 2, 0) + kappax * b_(0, i, 0));
    a_(i, 1, 0) = fac * (dy * a_(i, 0, 0) + ddx * a_(i - 1, 1, 0) -
                         a_(i - 2, 1, 0) + kappay * b_(i, 0, 0));
    a_(i, 0, 1) = fac * (dz * a_(i, 0, 0) + ddx * a_(i - 1, 0, 1) -
                         a_(i - 2, 0, 1) + kappaz * b_(i, 0, 0));
  }
  for (int i = 2; i <= L - 2; ++i) {
    for (int j = 2; j <= L - i; ++j) {
      b_(i, j, 0) = cf1_new[i] * (dx * a_(i - 1, j, 0) - a_(i - 2, j, 0));
      b_(i, 0, j) = cf1_new[i] * (dx * a_(i - 1, 0, j) - a_(i - 2, 0, j));
      b_(0, i, j) = cf1_new[i] * (dy * a_(0, i - 1, j) - a_(0, i - 2, j));
      a_(i, j, 0) = fac * (ddx * cf2[i] * a_(i - 1, j, 0) + ddy * a_(i, j - 1, 0) -
                           cf3[i] * a_(i - 2, j, 0) - a_(i, j - 2, 0) +
                           cf1_new[i] * (dx * b_(i - 1, j, 0) - b_(i - 2, j, 0)));
      a_(i, 0, j) = fac * (ddx * cf2[i] * a_(i - 1, 0, j) + ddz * a_(i, 0, j - 1) -
                           cf3[i] * a_(i - 2, 0, j) - a_(i, 0, j - 2) +
                           cf1_new[i] * (dx * b_(i - 1, 0, j) - b_(i - 2, 0, j)));
      a_(0, i, j) = fac * (ddy * cf2[i] * a_(0, i - 1, j) + ddz * a_(0, i, j - 1) -
                           cf3[i] * a_(0, i - 2, j) - a_(0, i, j - 2) +
                           cf1_new[i] * (dy * b_(0, i - 1, j) - b_(0, i - 2, j)));
    }
  }
  b_(1, 1, 1) = kappax * a_(0, 1, 1);
  a_(1, 1, 1) = fac * (dx * a_(0, 1, 1) + ddy * a_(1, 0, 1) + ddz * a_(1, 1, 0) +
                       kappax * b_(0, 1, 1));
  for (int i = 2; i <= L - 2; ++i) {
    b_(1, 1, i) = kappax * a_(0, 1, i);
    b_(1, i, 1) = kappax * a_(0, i, 1);
    b_(i, 1, 1) = kappay * a_(i, 0, 1);
    a_(1, 1, i) = fac * (dx * a_(0, 1, i) + ddy * a_(1, 0, i) + ddz * a_(1, 1, i - 1) -
                         a_(1, 1, i - 2) + kappax * b_(0, 1, i));
    a_(1, i, 1) = fac * (dx * a_(0, i, 1) + ddy * a_(1, i - 1, 1) + ddz * a_(1, i, 0) -
                         a_(1, i - 2, 1) + kappax * b_(0, i, 1));
    a_(i, 1, 1) = fac * (dy * a_(i, 0, 1) + ddx * a_(i - 1, 1, 1) + ddz * a_(i, 1, 0) -
                         a_(i - 2, 1, 1) + kappay * b_(i, 0, 1));
  }
  for (int i = 2; i <= L - 3; ++i) {
    for (int j = 2; j <= L - i; ++j) {
      b_(1, i, j) = kappax * a_(0, i, j);
      b_(i, 1, j) = kappay * a_(i, 0, j);
      b_(i, j, 1) = kappaz * a_(i, j, 0);
      a_(1, i, j) = fac * (dx * a_(0, i, j) + ddy * a_(1, i - 1, j) + ddz * a_(1, i, j - 1) -
                           a_(1, i - 2, j) - a_(1, i, j - 2) + kappax * b_(0, i, j));
      a_(i, 1, j) = fac * (dy * a_(i, 0, j) + ddx * a_(i - 1, 1, j) + ddz * a_(i, 1, j - 1) -
                           a_(i - 2, 1, j) - a_(i, 1, j - 2) + kappay * b_(i, 0, j));
      a_(i, j, 1) = fac * (dz * a_(i, j, 0) + ddx * a_(i - 1, j, 1) + ddy * a_(i, j - 1, 1) -
                           a_(i - 2, j, 1) - a_(i, j - 2, 1) + kappaz * b_(i, j, 0));
    }
  }
  for (int k = 2; k <= L - 4; ++k)
    for (int j = 2; j <= L - 2 - k; ++j)
      for (int i = 2; i <= L - k - j; ++i) {
        b_(i, j, k) = cf1_new[i] * (dx * a_(i - 1, j, k) - a_(i - 2, j, k));
        a_(i, j, k) = fac * (ddx * cf2[i] * a_(i - 1, j, k) + ddy * a_(i, j - 1, k) +
                             ddz * a_(i, j, k - 1) - cf3[i] * a_(i - 2, j, k) -
                             a_(i, j - 2, k) - a_(i, j, k - 2) +
                             cf1_new[i] * (dx * b_(i - 1, j, k) - b_(i - 2, j, k)));
      }
#undef a_
#undef b_
}

/* COMPP_TREE_PB (treecode3d_pb.f:439-486) */
static void compp_tree_pb(const or_tree* t, or_scratch* s, const or_node* p,
                          double kappa, double eps, double* peng) {
  int T1 = t->torder + 1;
  size_t T3 = (size_t)T1 * T1 * T1;
  const double* ms = t->ms + (size_t)p->mslot * 16 * T3;
  int P = t->order, P1 = P + 1;
  double pt_comp[16][2];
  double kapa[2] = {0.0, kappa};
  for (int ikp = 0; ikp < 2; ++ikp) {
    comp_tcoeff(t, s, p, kapa[ikp]);
    for (int indx = 0; indx < 16; ++indx) {
      double pg = 0.0;
      const int* kk = t->kk[indx];
      for (int k = 0; k <= P; ++k)
        for (int j = 0; j <= P - k; ++j)
          for (int i = 0; i <= P - k - j; ++i) {
            double dc = t->der_cof[(((size_t)indx * P1 + k) * P1 + j) * P1 + i];
            pg = pg + dc * s->a[AB(s, i + kk[0], j + kk[1], k + kk[2])] *
                          ms[(size_t)indx * T3 + MSI(t, i, j, k)];
          }
      pt_comp[indx][ikp] = s->tempq[indx] * pg;
    }
  }
  double sl1 = pt_comp[0][0] - pt_comp[0][1];
  double s24_2 = pt_comp[1][1] + pt_comp[2][1] + pt_comp[3][1];
  double s24_1 = pt_comp[1][0] + pt_comp[2][0] + pt_comp[3][0];
  double sl2 = eps * s24_2 - s24_1;
  double s57_1 = pt_comp[4][0] + pt_comp[5][0] + pt_comp[6][0];
  double s57_2 = pt_comp[4][1] + pt_comp[5][1] + pt_comp[6][1];
  double sl3 = -(s57_1 - 1.0 / eps * s57_2);
  double s816_2 = 0.0, s816_1 = 0.0;
  for (int i = 7; i < 16; ++i) {
    s816_2 = s816_2 + pt_comp[i][1];
    s816_1 = s816_1 + pt_comp[i][0];
  }
  double sl4 = s816_2 - s816_1;
  peng[0] = sl1 + sl2;
  peng[1] = sl3 + sl4;
}

/* COMPP_DIRECT_PB (treecode3d_pb.f:919-1008); the target's own term is the
 * one the reference zeroes by shifting x(i) and setting tr_area(i)=0
 * (:1169-1172), which adds exactly +-0 -- skipping it is bit-identical. */
static void compp_direct_pb(const or_tree* t, or_scratch* s, int ibeg,
                            int iend, const double* tpoten, double kappa,
                            double eps, double* peng) {
  const double one_over_4pi = 0.25 / PI_F;
  int n = t->n;
  double p1 = 0.0, p2 = 0.0;
  const double* sp = s->tarpos;
  const double* v0 = s->tarq;
  for (int j = ibeg; j <= iend; ++j) {
    if (j == s->self) continue;
    s->near_pairs++;
    double r[3] = {t->x[j - 1], t->y[j - 1], t->z[j - 1]};
    const double* v = t->tq + 3 * (size_t)(j - 1);
    double d[3] = {r[0] - sp[0], r[1] - sp[1], r[2] - sp[2]};
    double rs = sqrt(dot3(d, d));
    double G0 = one_over_4pi / rs;
    double kappa_rs = kappa * rs;
    double exp_kappa_rs = exp(-kappa_rs);
    double Gk = exp_kappa_rs * G0;
    double cos_theta = dot3(v, d) / rs;
    double cos_theta0 = dot3(v0, d) / rs;
    double tp1 = G0 / rs;
    double tp2 = (1.0 + kappa_rs) * exp_kappa_rs;
    double G10 = cos_theta0 * tp1;
    double G20 = tp2 * G10;
    double G1 = cos_theta * tp1;
    double G2 = tp2 * G1;
    double G3 = (dot3(v0, v) - 3.0 * cos_theta0 * cos_theta) / rs * tp1;
    double G4 = tp2 * G3 - kappa * kappa * cos_theta0 * cos_theta * Gk;
    double L1 = G1 - eps * G2;
    double L2 = G0 - Gk;
    double L3 = G4 - G3;
    double L4 = G10 - G20 / eps;
    double x1 = tpoten[j - 1], x2 = tpoten[j - 1 + n];
    double area = t->area[j - 1];
    p1 = p1 + (L1 * x1 + L2 * x2) * area;
    p2 = p2 + (L3 * x1 + L4 * x2) * area;
  }
  peng[0] = p1;
  peng[1] = p2;
}

/* COMPP_TREE (treecode3d_pb.f:359-436) */
static void compp_tree(const or_tree* t, or_scratch* s, int id,
                       const double* tpoten, double kappa, double eps,
                       double* peng) {
  const or_node* p = &t->nodes[id];
  double tx = p->x_mid - s->tarpos[0];
  double ty = p->y_mid - s->tarpos[1];
  double tz = p->z_mid - s->tarpos[2];
  double dist = sqrt(tx * tx + ty * ty + tz * tz);
  peng[0] = peng[1] = 0.0;
  if (p->radius < dist * t->theta && p->numpar > 40) {
    s->far_inter++;
    compp_tree_pb(t, s, p, kappa, eps, peng);
  } else if (p->num_children == 0) {
    compp_direct_pb(t, s, p->ibeg, p->iend, tpoten, kappa, eps, peng);
  } else {
    for (int i = 0; i < p->num_children; ++i) {
      double pl[2];
      compp_tree(t, s, p->child[i], tpoten, kappa, eps, pl);
      peng[0] = peng[0] + pl[0];
      peng[1] = peng[1] + pl[1];
    }
  }
}

static void prepare_matvec(or_tree* t, const double* x) {
  pb_kernel(t, x);
  for (int i = 0; i < t->nnodes; ++i)
    if (t->nodes[i].mslot >= 0) comp_ms(t, &t->nodes[i]);
}

static void matvec_targets(or_tree* t, double kappa, double eps,
                           const double* x, double* y, int i0, int i1,
                           int64_t* counts, int nthreads) {
  int n = t->n;
  double pre1 = 0.5 * (1.0 + eps);
  double pre2 = 0.5 * (1.0 + 1.0 / eps);
  int64_t np = 0, nf = 0;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads) reduction(+ : np, nf)
#endif
  {
    or_scratch s;
    s.L = t->torderlim;
    s.D = s.L + 3;
    size_t D3 = (size_t)s.D * s.D * s.D;
    s.a = (double*)calloc(D3, sizeof(double));
    s.b = (double*)calloc(D3, sizeof(double));
    s.near_pairs = s.far_inter = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (int i = i0; i < i1; ++i) {
      s.tarpos[0] = t->x[i];
      s.tarpos[1] = t->y[i];
      s.tarpos[2] = t->z[i];
      for (int d = 0; d < 3; ++d) s.tarq[d] = t->tq[3 * (size_t)i + d];
      for (int idx = 0; idx < 16; ++idx)
        s.tempq[idx] = t->tchg[(size_t)idx * n + i];
      s.self = i + 1;
      double peng[2];
      compp_tree(t, &s, 0, x, kappa, eps, peng);
      y[i] = pre1 * x[i] - peng[0];
      y[n + i] = pre2 * x[n + i] - peng[1];
    }
    np += s.near_pairs;
    nf += s.far_inter;
    free(s.a);
    free(s.b);
  }
  if (counts) {
    counts[0] = np;
    counts[1] = nf;
  }
}

/* MATVECmain (main.f90:467-488) -> TREE_COMPP_PB (:1130-1189) */
void or_matvec(or_tree* t, double kappa, double eps, const double* x,
               double* y, int64_t* counts, int nthreads) {
  int n2 = 2 * t->n;
  double sa = 0.0;
  for (int i = 0; i < n2; ++i) sa = sa + fabs(x[i]);
  if (sa < 1e-10) {
    for (int i = 0; i < n2; ++i) y[i] = x[i];
    if (counts) counts[0] = counts[1] = 0;
    return;
  }
  prepare_matvec(t, x);
  matvec_targets(t, kappa, eps, x, y, 0, t->n, counts, nthreads);
}

void or_matvec_range(or_tree* t, double kappa, double eps, const double* x,
                     double* y, int i0, int i1, int64_t* counts,
                     int nthreads) {
  prepare_matvec(t, x);
  matvec_targets(t, kappa, eps, x, y, i0, i1, counts, nthreads);
}

void or_matvec_prepare(or_tree* t, const double* x) { prepare_matvec(t, x); }

void or_matvec_targets(or_tree* t, double kappa, double eps, const double* x,
                       double* y, int i0, int i1, int64_t* counts,
                       int nthreads) {
  matvec_targets(t, kappa, eps, x, y, i0, i1, counts, nthreads);
}

void or_matvec_direct(int n, const double* tr_xyz, const double* tr_q,
                      const double* tr_area, double kappa, double eps,
                      const double* x, double* y, int nthreads) {
  const double one_over_4pi = 0.25 / PI_F;
  double pre1 = 0.5 * (1.0 + eps);
  double pre2 = 0.5 * (1.0 + 1.0 / eps);
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 16)
#endif
  for (int i = 0; i < n; ++i) {
    const double* s = tr_xyz + 3 * (size_t)i;
    const double* v0 = tr_q + 3 * (size_t)i;
    double p1 = 0.0, p2 = 0.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double* r = tr_xyz + 3 * (size_t)j;
      const double* v = tr_q + 3 * (size_t)j;
      double d[3] = {r[0] - s[0], r[1] - s[1], r[2] - s[2]};
      double rs = sqrt(dot3(d, d));
      double G0 = one_over_4pi / rs;
      double kappa_rs = kappa * rs;
      double e = exp(-kappa_rs);
      double Gk = e * G0;
      double c = dot3(v, d) / rs;
      double c0 = dot3(v0, d) / rs;
      double tp1 = G0 / rs;
      double tp2 = (1.0 + kappa_rs) * e;
      double G10 = c0 * tp1, G20 = tp2 * G10;
      double G1 = c * tp1, G2 = tp2 * G1;
      double G3 = (dot3(v0, v) - 3.0 * c0 * c) / rs * tp1;
      double G4 = tp2 * G3 - kappa * kappa * c0 * c * Gk;
      double L1 = G1 - eps * G2, L2 = G0 - Gk, L3 = G4 - G3,
             L4 = G10 - G20 / eps;
      p1 = p1 + (L1 * x[j] + L2 * x[n + j]) * tr_area[j];
      p2 = p2 + (L3 * x[j] + L4 * x[n + j]) * tr_area[j];
    }
    y[i] = pre1 * x[i] - p1;
    y[n + i] = pre2 * x[n + i] - p2;
  }
  (void)nthreads;
}

/* ------------------------------------------------------------------ */
/* dense LU: DGETRF2 (dgetrf_dep.f:757-900), DLASWP, DTRSM, DGEMM, DGETRS */

#define M_(a, lda, i, j) (a)[(size_t)((j)-1) * (lda) + ((i)-1)]

static void dlaswp(int n, double* a, int lda, int k1, int k2,
                   const int* ipiv) {
  /* incx = 1: rows k1..k2 swapped with ipiv(k) in increasing k */
  for (int i = k1; i <= k2; ++i) {
    int ip = ipiv[i - 1];
    if (ip != i)
      for (int j = 1; j <= n; ++j) {
        double tmp = M_(a, lda, i, j);
        M_(a, lda, i, j) = M_(a, lda, ip, j);
        M_(a, lda, ip, j) = tmp;
      }
  }
}

/* DTRSM Left, Lower, No transpose, Unit */
static void dtrsm_llnu(int m, int n, const double* a, int lda, double* b,
                       int ldb) {
  for (int j = 1; j <= n; ++j)
    for (int k = 1; k <= m; ++k)
      if (M_(b, ldb, k, j) != 0.0)
        for (int i = k + 1; i <= m; ++i)
          M_(b, ldb, i, j) = M_(b, ldb, i, j) - M_(b, ldb, k, j) * M_(a, lda, i, k);
}

/* DTRSM Left, Upper, No transpose, Non-unit */
static void dtrsm_lunn(int m, int n, const double* a, int lda, double* b,
                       int ldb) {
  for (int j = 1; j <= n; ++j)
    for (int k = m; k >= 1; --k)
      if (M_(b, ldb, k, j) != 0.0) {
        M_(b, ldb, k, j) = M_(b, ldb, k, j) / M_(a, lda, k, k);
        for (int i = 1; i <= k - 1; ++i)
          M_(b, ldb, i, j) = M_(b, ldb, i, j) - M_(b, ldb, k, j) * M_(a, lda, i, k);
      }
}

/* DGEMM N,N with alpha = -1, beta = 1 */
static void dgemm_nn_m1(int m, int n, int k, const double* a, int lda,
                        const double* b, int ldb, double* c, int ldc) {
  for (int j = 1; j <= n; ++j)
    for (int l = 1; l <= k; ++l) {
      double temp = -1.0 * M_(b, ldb, l, j);
      for (int i = 1; i <= m; ++i)
        M_(c, ldc, i, j) = M_(c, ldc, i, j) + temp * M_(a, lda, i, l);
    }
}

static int dgetrf2(int m, int n, double* a, int lda, int* ipiv) {
  int info = 0;
  if (m == 0 || n == 0) return 0;
  if (m == 1) {
    ipiv[0] = 1;
    if (M_(a, lda, 1, 1) == 0.0) info = 1;
  } else if (n == 1) {
    double sfmin = DBL_MIN; /* DLAMCH('S') for IEEE double */
    int imax = 1;
    double vmax = fabs(M_(a, lda, 1, 1));
    for (int i = 2; i <= m; ++i)
      if (fabs(M_(a, lda, i, 1)) > vmax) {
        vmax = fabs(M_(a, lda, i, 1));
        imax = i;
      }
    ipiv[0] = imax;
    if (M_(a, lda, imax, 1) != 0.0) {
      if (imax != 1) {
        double temp = M_(a, lda, 1, 1);
        M_(a, lda, 1, 1) = M_(a, lda, imax, 1);
        M_(a, lda, imax, 1) = temp;
      }
      if (fabs(M_(a, lda, 1, 1)) >= sfmin) {
        double r = 1.0 / M_(a, lda, 1, 1);
        for (int i = 2; i <= m; ++i) M_(a, lda, i, 1) = r * M_(a, lda, i, 1);
      } else {
        for (int i = 2; i <= m; ++i)
          M_(a, lda, i, 1) = M_(a, lda, i, 1) / M_(a, lda, 1, 1);
      }
    } else {
      info = 1;
    }
  } else {
    int mn = m < n ? m : n;
    int n1 = mn / 2;
    int n2 = n - n1;
    int iinfo = dgetrf2(m, n1, a, lda, ipiv);
    if (info == 0 && iinfo > 0) info = iinfo;
    dlaswp(n2, &M_(a, lda, 1, n1 + 1), lda, 1, n1, ipiv);
    dtrsm_llnu(n1, n2, a, lda, &M_(a, lda, 1, n1 + 1), lda);
    dgemm_nn_m1(m - n1, n2, n1, &M_(a, lda, n1 + 1, 1), lda,
                &M_(a, lda, 1, n1 + 1), lda, &M_(a, lda, n1 + 1, n1 + 1), lda);
    iinfo = dgetrf2(m - n1, n2, &M_(a, lda, n1 + 1, n1 + 1), lda, ipiv + n1);
    if (info == 0 && iinfo > 0) info = iinfo + n1;
    for (int i = n1 + 1; i <= mn; ++i) ipiv[i - 1] = ipiv[i - 1] + n1;
    dlaswp(n1, a, lda, n1 + 1, mn, ipiv);
  }
  return info;
}

/* DGETRF (dgetrf_dep.f:107-220): the vendored testing ILAENV returns an
 * unset COMMON value (NB = 0), so DGETRF always takes DGETRF2. */
int or_dgetrf(int m, int n, double* a, int lda, int* ipiv) {
  return dgetrf2(m, n, a, lda, ipiv);
}

/* DGETRS 'N' (dgetrf_dep.f:346-445) */
void or_dgetrs(int n, int nrhs, const double* a, int lda, const int* ipiv,
               double* b, int ldb) {
  dlaswp(nrhs, b, ldb, 1, n, ipiv);
  dtrsm_llnu(n, nrhs, a, lda, b, ldb);
  dtrsm_lunn(n, nrhs, a, lda, b, ldb);
}

/* LEAFMATVECpara (treecode3d_pb.f:1393-1542).  NOTE: the reference puts
 * -A*(G0-Gk) (the operator's x2-coefficient of equation 1) in block
 * (row 2, col 1) and -A*(G4-G3) in block (row 1, col 2) -- the transpose of
 * where the operator has them; restated as is. */
int or_msolve_block(or_tree* t, double kappa, double eps, const double* rhs,
                    double* sol, int leaf0, int leaf1, int nthreads) {
  const double one_over_4pi = 0.25 / PI_F;
  int N = t->n;
  double pre1 = 0.5 * (1.0 + eps);
  double pre2 = 0.5 * (1.0 + 1.0 / eps);
  if (leaf1 < 0 || leaf1 > t->nleaf) leaf1 = t->nleaf;
  int nbad = 0;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) reduction(+ : nbad)
#endif
  for (int il = leaf0; il < leaf1; ++il) {
    int ibeg = t->leaf_ibeg[il];
    int nrow = t->leaf_n[il];
    int iend = ibeg + nrow - 1;
    int nrow2 = 2 * nrow;
    double* A = (double*)calloc((size_t)nrow2 * nrow2, sizeof(double));
    double* r2s = (double*)malloc(sizeof(double) * (size_t)nrow2);
    int* ipiv = (int*)malloc(sizeof(int) * (size_t)nrow2);
    for (int i = 0; i < nrow; ++i) {
      r2s[i] = rhs[ibeg - 1 + i];
      r2s[nrow + i] = rhs[ibeg - 1 + N + i];
    }
    for (int i = ibeg; i <= iend; ++i) {
      double tx[3] = {t->x[i - 1], t->y[i - 1], t->z[i - 1]};
      const double* tc = t->tq + 3 * (size_t)(i - 1);
      for (int j = ibeg; j <= iend; ++j) {
        if (j == i) continue;
        double r[3] = {t->x[j - 1], t->y[j - 1], t->z[j - 1]};
        const double* v = t->tq + 3 * (size_t)(j - 1);
        double d[3] = {r[0] - tx[0], r[1] - tx[1], r[2] - tx[2]};
        double rs = sqrt(dot3(d, d));
        double G0 = one_over_4pi / rs;
        double kappa_rs = kappa * rs;
        double e = exp(-kappa_rs);
        double Gk = e * G0;
        double c = dot3(v, d) / rs;
        double c0 = dot3(tc, d) / rs;
        double tp1 = G0 / rs;
        double tp2 = (1.0 + kappa_rs) * e;
        double G10 = c0 * tp1, G20 = tp2 * G10;
        double G1 = c * tp1, G2 = tp2 * G1;
        double G3 = (dot3(tc, v) - 3.0 * c0 * c) / rs * tp1;
        double G4 = tp2 * G3 - kappa * kappa * c0 * c * Gk;
        double aj = t->area[j - 1];
        size_t m1 = (size_t)(j - ibeg) * nrow2 + (i - ibeg);
        size_t m2 = (size_t)(j - ibeg) * nrow2 + (i - ibeg + nrow);
        size_t m3 = (size_t)(j - ibeg + nrow) * nrow2 + (i - ibeg);
        size_t m4 = (size_t)(j - ibeg + nrow) * nrow2 + (i - ibeg + nrow);
        A[m1] = -(G1 - eps * G2) * aj;
        A[m2] = -(G0 - Gk) * aj;
        A[m3] = -(G4 - G3) * aj;
        A[m4] = -(G10 - G20 / eps) * aj;
      }
      A[(size_t)(i - ibeg) * (nrow2 + 1)] = pre1;
      A[(size_t)(i - ibeg + nrow) * (nrow2 + 1)] = pre2;
    }
    int info = or_dgetrf(nrow2, nrow2, A, nrow2, ipiv);
    if (info != 0) nbad++;
    or_dgetrs(nrow2, 1, A, nrow2, ipiv, r2s, nrow2);
    for (int i = 0; i < nrow; ++i) {
      sol[ibeg - 1 + i] = r2s[i];
      sol[ibeg - 1 + N + i] = r2s[nrow + i];
    }
    free(A);
    free(r2s);
    free(ipiv);
  }
  (void)nthreads;
  return nbad;
}

/* MSOLVEprec (main.f90:532-542) */
void or_msolve_diag(int n2, double eps, const double* r, double* z) {
  double scale1 = 0.5 * (1.0 + eps);
  double scale2 = 0.5 * (1.0 + 1.0 / eps);
  for (int i = 0; i < n2 / 2; ++i) z[i] = r[i] / scale1;
  for (int i = n2 / 2; i < n2; ++i) z[i] = r[i] / scale2;
}

/* ------------------------------------------------------------------ */
/* GMRES: DGMRES (dgmres_dep.f:689-853), DPIGMR (:1652-1864), DORTH
 * (:1376-1415), DHEQR (:1031-1128), DHELS (:925-950), DRLCAL (:1948-1979),
 * ISDGMR (:2532-2650).  JSCAL = 0, KMP = MAXL, ITOL = 2.                */

typedef struct {
  or_tree* t;
  double kappa, eps;
  int iprcd, nthreads;
  int64_t nmv, nms;
} or_op;

static void op_matvec(or_op* op, const double* x, double* y) {
  or_matvec(op->t, op->kappa, op->eps, x, y, NULL, op->nthreads);
  op->nmv++;
}
static void op_msolve(or_op* op, const double* r, double* z) {
  if (op->iprcd == 1)
    or_msolve_block(op->t, op->kappa, op->eps, r, z, 0, -1, op->nthreads);
  else
    or_msolve_diag(2 * op->t->n, op->eps, r, z);
  op->nms++;
}

static double dnrm2(int n, const double* x) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + x[i] * x[i];
  return sqrt(s);
}
static double ddot(int n, const double* x, const double* y) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + x[i] * y[i];
  return s;
}
static void daxpy(int n, double a, const double* x, double* y) {
  if (a == 0.0) return;
  for (int i = 0; i < n; ++i) y[i] = y[i] + a * x[i];
}

#define HES_(i, j) hes[(size_t)((j)-1) * ldh + ((i)-1)]
#define V_(j) (v + (size_t)((j)-1) * n)

static void dorth(int n, double* vnew, const double* v, double* hes, int ldh,
                  int ll, int kmp, double* snormw) {
  double vnrm = dnrm2(n, vnew);
  int i0 = ll - kmp + 1 > 1 ? ll - kmp + 1 : 1;
  for (int i = i0; i <= ll; ++i) {
    HES_(i, ll) = ddot(n, V_(i), vnew);
    daxpy(n, -HES_(i, ll), V_(i), vnew);
  }
  *snormw = dnrm2(n, vnew);
  if (vnrm + 0.001 * (*snormw) != vnrm) return;
  double sumdsq = 0.0;
  for (int i = i0; i <= ll; ++i) {
    double tem = -ddot(n, V_(i), vnew);
    if (HES_(i, ll) + 0.001 * tem == HES_(i, ll)) continue;
    HES_(i, ll) = HES_(i, ll) - tem;
    daxpy(n, tem, V_(i), vnew);
    sumdsq = sumdsq + tem * tem;
  }
  if (sumdsq == 0.0) return;
  double arg = (*snormw) * (*snormw) - sumdsq;
  if (arg < 0.0) arg = 0.0;
  *snormw = sqrt(arg);
}

static void givens(double t1, double t2, double* c, double* s) {
  if (t2 == 0.0) {
    *c = 1.0;
    *s = 0.0;
  } else if (fabs(t2) >= fabs(t1)) {
    double tt = t1 / t2;
    *s = -1.0 / sqrt(1.0 + tt * tt);
    *c = -(*s) * tt;
  } else {
    double tt = t2 / t1;
    *c = 1.0 / sqrt(1.0 + tt * tt);
    *s = -(*c) * tt;
  }
}

/* DHEQR with IJOB = 1 for nn = 1, else IJOB = 2 (update of column nn) */
static int dheqr(double* hes, int ldh, int nn, double* q) {
  int info = 0;
  if (nn == 1) {
    double c, s, t1 = HES_(1, 1), t2 = HES_(2, 1);
    givens(t1, t2, &c, &s);
    q[0] = c;
    q[1] = s;
    HES_(1, 1) = c * t1 - s * t2;
    if (HES_(1, 1) == 0.0) info = 1;
    return info;
  }
  for (int k = 1; k <= nn - 1; ++k) {
    int i = 2 * (k - 1);
    double t1 = HES_(k, nn), t2 = HES_(k + 1, nn);
    double c = q[i], s = q[i + 1];
    HES_(k, nn) = c * t1 - s * t2;
    HES_(k + 1, nn) = s * t1 + c * t2;
  }
  double c, s, t1 = HES_(nn, nn), t2 = HES_(nn + 1, nn);
  givens(t1, t2, &c, &s);
  q[2 * nn - 2] = c;
  q[2 * nn - 1] = s;
  HES_(nn, nn) = c * t1 - s * t2;
  if (HES_(nn, nn) == 0.0) info = nn;
  return info;
}

static void dhels(const double* hes, int ldh, int nn, const double* q,
                  double* b) {
  for (int k = 1; k <= nn; ++k) {
    int iq = 2 * (k - 1);
    double c = q[iq], s = q[iq + 1];
    double t1 = b[k - 1], t2 = b[k];
    b[k - 1] = c * t1 - s * t2;
    b[k] = s * t1 + c * t2;
  }
  for (int kb = 1; kb <= nn; ++kb) {
    int k = nn + 1 - kb;
    b[k - 1] = b[k - 1] / HES_(k, k);
    double tt = -b[k - 1];
    for (int i = 1; i <= k - 1; ++i) b[i - 1] = b[i - 1] + tt * HES_(i, k);
  }
}

static void drlcal(int n, int kmp, int ll, int maxl, const double* v,
                   const double* q, double* rl, double snormw, double prod,
                   double r0nrm) {
  if (kmp == maxl) {
    memcpy(rl, V_(1), sizeof(double) * (size_t)n);
    for (int i = 1; i <= ll - 1; ++i) {
      double s = q[2 * i - 1], c = q[2 * i - 2];
      const double* vi = V_(i + 1);
      for (int k = 0; k < n; ++k) rl[k] = s * rl[k] + c * vi[k];
    }
    double s = q[2 * ll - 1], c = q[2 * ll - 2] / snormw;
    const double* vl = V_(ll + 1);
    for (int k = 0; k < n; ++k) rl[k] = s * rl[k] + c * vl[k];
  }
  double tem = r0nrm * prod;
  for (int k = 0; k < n; ++k) rl[k] = tem * rl[k];
}

#undef HES_
#undef V_

int or_dgmres(or_tree* t, double kappa, double eps, int iprcd,
              const double* b, double* x, double tol, int maxl, int nrmax,
              int* iter_out, double* err_out, double* err_hist, int* n_hist,
              int64_t* n_matvec, int64_t* n_msolve, int nthreads) {
  or_op op = {t, kappa, eps, iprcd, nthreads, 0, 0};
  int n = 2 * t->n;
  int nh = 0;
  if (maxl == 0) maxl = 10;
  if (maxl > n) maxl = n;
  int kmp = maxl;
  if (nrmax == 0) nrmax = 10;
  if (nrmax == -1) nrmax = 0;
  if (tol == 0.0) tol = 500 * 1e-20;
  int maxlp1 = maxl + 1;
  int ldh = maxlp1;
  double* v = (double*)calloc((size_t)n * maxlp1, sizeof(double));
  double* hes = (double*)calloc((size_t)maxlp1 * maxl, sizeof(double));
  double* q = (double*)calloc(2 * (size_t)maxl, sizeof(double));
  double* r = (double*)calloc((size_t)n + 1, sizeof(double));
  double* dl = (double*)calloc((size_t)n, sizeof(double));
  double* wk = (double*)calloc((size_t)n, sizeof(double));
  double* z = (double*)calloc((size_t)n, sizeof(double));
  int iter = 0, ierr = 0;
  double err = 0.0;
  int nrsts = 0;
  /* JPRE = -1: BNRM = |M^-1 b| (dgmres_dep.f:754-771) */
  op_msolve(&op, b, r);
  double bnrm = dnrm2(n, r);
  op_matvec(&op, x, r);
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  for (;;) {
    if (nrsts > nrmax) {
      ierr = 1;
      break;
    }
    if (nrsts > 0) memcpy(r, dl, sizeof(double) * (size_t)n);
    /* ---- DPIGMR ---- */
    int iflag = 0, lgmr = 0;
    double rhol = 0.0, snormw = 0.0, prod = 1.0, rho = 0.0;
    memset(z, 0, sizeof(double) * (size_t)n);
    if (nrsts == 0) {
      memcpy(wk, r, sizeof(double) * (size_t)n);
      op_msolve(&op, wk, r);
    }
    memcpy(v, r, sizeof(double) * (size_t)n);
    double r0nrm = dnrm2(n, v);
    /* ISDGMR with LGMR = 0: ERR = |V(:,1)| / BNRM */
    err = dnrm2(n, v) / bnrm;
    int conv_now = (err <= tol);
    int goto200 = 0, goto120 = 0;
    if (conv_now) {
      /* DPIGMR returns at once with IFLAG = 0, LGMR = 0, Z = 0 */
      iflag = 0;
      lgmr = 0;
    } else {
      double tem = 1.0 / r0nrm;
      for (int i = 0; i < n; ++i) v[i] = tem * v[i];
      memset(hes, 0, sizeof(double) * (size_t)maxlp1 * maxl);
      prod = 1.0;
      int ll;
      for (ll = 1; ll <= maxl; ++ll) {
        lgmr = ll;
        double* vl = v + (size_t)(ll - 1) * n;
        double* vn = v + (size_t)ll * n;
        memcpy(wk, vl, sizeof(double) * (size_t)n);
        op_matvec(&op, wk, vn);
        memcpy(wk, vn, sizeof(double) * (size_t)n);
        op_msolve(&op, wk, vn);
        dorth(n, vn, v, hes, ldh, ll, kmp, &snormw);
        hes[(size_t)(ll - 1) * ldh + ll] = snormw;
        int info = dheqr(hes, ldh, ll, q);
        if (info == ll) {
          goto120 = 1;
          break;
        }
        prod = prod * q[2 * ll - 1];
        rho = fabs(prod * r0nrm);
        rhol = rho;
        drlcal(n, kmp, lgmr, maxl, v, q, dl, snormw, prod, r0nrm);
        err = dnrm2(n, dl) / bnrm;
        if (err_hist) err_hist[nh] = err;
        nh++;
        if (err <= tol) {
          goto200 = 1;
          break;
        }
        if (ll == maxl) break;
        tem = 1.0 / snormw;
        for (int i = 0; i < n; ++i) vn[i] = tem * vn[i];
      }
      if (!goto200 && !goto120) {
        if (rho < r0nrm) {
          iflag = 1;
          if (nrmax > 0)
            drlcal(n, kmp, maxl, maxl, v, q, dl, snormw, prod, r0nrm);
          goto200 = 1;
        } else {
          goto120 = 1;
        }
      }
      if (goto120) {
        iflag = 2;
        memset(z, 0, sizeof(double) * (size_t)n);
      } else if (goto200) {
        int l = lgmr;
        double* r0 = r;
        for (int k = 0; k <= l; ++k) r0[k] = 0.0;
        r0[0] = r0nrm;
        dhels(hes, ldh, l, q, r0);
        memset(z, 0, sizeof(double) * (size_t)n);
        for (int i = 1; i <= l; ++i)
          daxpy(n, r0[i - 1], v + (size_t)(i - 1) * n, z);
      }
    }
    (void)rhol;
    /* ---- back in DGMRES (dgmres_dep.f:796-814) ---- */
    iter += lgmr;
    for (int i = 0; i < n; ++i) x[i] = x[i] + z[i];
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
  free(v);
  free(hes);
  free(q);
  free(r);
  free(dl);
  free(wk);
  free(z);
  if (iter_out) *iter_out = iter;
  if (err_out) *err_out = err;
  if (n_hist) *n_hist = nh;
  if (n_matvec) *n_matvec = op.nmv;
  if (n_msolve) *n_msolve = op.nms;
  return ierr;
}

/* ------------------------------------------------------------------ */
/* energy: potential_molecule (main.f90:614-657) + main.f90:144-157      */

void or_energy_surface(int nface, const double* tr_xyz, const double* tr_q,
                       const double* tr_area, int nchr, const double* chrpos,
                       const double* atmchr, double kappa, double eps,
                       double eps0, const double* x, double* soleng,
                       double* couleng, int nthreads) {
  const double pi = PI_F;
  const double one_over_4pi = 0.25 / pi;
  const double para = 332.0716;
  double* ptl = (double*)malloc(sizeof(double) * (size_t)(nchr > 0 ? nchr : 1));
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
#endif
  for (int k = 0; k < nchr; ++k) {
    const double* r0 = chrpos + 3 * (size_t)k;
    double p = 0.0;
    for (int j = 0; j < nface; ++j) {
      const double* r = tr_xyz + 3 * (size_t)j;
      const double* v = tr_q + 3 * (size_t)j;
      double d[3] = {r[0] - r0[0], r[1] - r0[1], r[2] - r0[2]};
      double rs = sqrt(dot3(d, d));
      double G0 = one_over_4pi / rs;
      double kappa_rs = kappa * rs;
      double e = exp(-kappa_rs);
      double Gk = e * G0;
      double cos_theta = dot3(v, d) / rs;
      double tp1 = G0 / rs;
      double tp2 = (1.0 + kappa_rs) * e;
      double G1 = cos_theta * tp1;
      double G2 = tp2 * G1;
      double H1 = G1 - eps * G2;
      double H2 = G0 - Gk;
      p = p + tr_area[j] * H1 * x[j];
      p = p + tr_area[j] * H2 * x[nface + j];
    }
    ptl[k] = p;
  }
  (void)nthreads;
  double se = 0.0, ce = 0.0;
  for (int k = 0; k < nchr; ++k) {
    se = se + atmchr[k] * ptl[k];
    const double* r0 = chrpos + 3 * (size_t)k;
    for (int l = k + 1; l < nchr; ++l) {
      double dist = dist3(r0, chrpos + 3 * (size_t)l);
      ce = ce + 1.0 / eps0 / dist * atmchr[k] * atmchr[l];
    }
  }
  free(ptl);
  *soleng = se * 0.5 * para * 4.0 * pi;
  *couleng = ce * para;
}

void or_energy(const or_tree* t, int nchr, const double* chrpos,
               const double* atmchr, double kappa, double eps, double eps0,
               const double* x, double* soleng, double* couleng,
               int nthreads) {
  int n = t->n;
  double* xyz = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    xyz[3 * (size_t)i + 0] = t->x[i];
    xyz[3 * (size_t)i + 1] = t->y[i];
    xyz[3 * (size_t)i + 2] = t->z[i];
  }
  or_energy_surface(n, xyz, t->tq, t->area, nchr, chrpos, atmchr, kappa, eps,
                    eps0, x, soleng, couleng, nthreads);
  free(xyz);
}

/* main.f90:226-326 output_potential: x_orig (2 nface, original face order)
 * and the face centroids tr_xyz (3 x nface, original order) in; per vertex
 * the first 14 faces using it in face order (the 15-row ind_vert table,
 * :243,255-266), weighted by the inverse centroid distance (:268-281), then
 * both vertex and face values times para*4*pi (:297-298). */
void or_output_potential(int nspt, const double* sptpos, int nface, const int* nvert,
                         const double* tr_xyz, const double* x_orig, double* vert_ptl,
                         double* x_scaled) {
  const int nface_vert = 15;
  int* ind = (int*)calloc((size_t)nface_vert * (size_t)nspt, sizeof(int));
  for (int i = 0; i < nface; ++i)
    for (int j = 0; j < 3; ++j) {
      int v = nvert[3 * i + j] - 1;
      for (int k = 0; k < nface_vert - 1; ++k)
        if (ind[(size_t)v * nface_vert + k] == 0) {
          ind[(size_t)v * nface_vert + k] = i + 1;
          ind[(size_t)v * nface_vert + nface_vert - 1] += 1;
          break;
        }
    }
  const double pi = acos(-1.0);
  const double para_temp = 332.0716 * 4 * pi;
  for (int i = 0; i < nspt; ++i) {
    double tot = 0.0, v1 = 0.0, v2 = 0.0;
    for (int j = 0; j < ind[(size_t)i * nface_vert + nface_vert - 1]; ++j) {
      int f = ind[(size_t)i * nface_vert + j] - 1;
      double aa[3];
      for (int d = 0; d < 3; ++d) aa[d] = tr_xyz[3 * (size_t)f + d] - sptpos[3 * (size_t)i + d];
      double ll = sqrt(dot3(aa, aa));
      v1 = v1 + 1.0 / ll * x_orig[f];
      v2 = v2 + 1.0 / ll * x_orig[f + nface];
      tot = tot + 1.0 / ll;
    }
    vert_ptl[2 * (size_t)i] = v1 / tot * para_temp;
    vert_ptl[2 * (size_t)i + 1] = v2 / tot * para_temp;
  }
  for (int i = 0; i < 2 * nface; ++i) x_scaled[i] = x_orig[i] * para_temp;
  free(ind);
}
