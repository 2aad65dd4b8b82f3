"""ctypes wrapper of the CPU oracle (oracle/tabi_oracle.c).

TEST INFRASTRUCTURE ONLY: a CPU restatement of the reference Fortran TABI-PB
solve path (gengwh/TABI-PB).  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py may import this module; the product path
(libtabi_gpu.so through tabipb) never does.  Parity of the restatement with
the reference binary is unpinned (no Fortran compiler, no reference golden
outputs); it is checked against the analytic Born energy and an FP64 direct
sum.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtabi_oracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc only, seconds)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH)
        < max(os.path.getmtime(os.path.join(_HERE, f)) for f in ("tabi_oracle.c", "tabi_oracle.h"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.or_surface_area.argtypes = [C.c_int, _dp, C.c_int, _ip, C.POINTER(C.c_double)]
        L.or_surface_area.restype = C.c_int
        L.or_form_matrix.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, C.c_int, _dp, _dp,
                                     C.c_double, _dp, _dp, _dp, _dp, C.c_int]
        L.or_form_matrix.restype = None
        L.or_tree_create.argtypes = [C.c_int, _dp, _dp, _dp, C.c_void_p, C.c_int, C.c_int,
                                     C.c_double, _ip, C.POINTER(C.c_int)]
        L.or_tree_create.restype = C.c_void_p
        L.or_tree_free.argtypes = [C.c_void_p]
        L.or_tree_num_nodes.argtypes = [C.c_void_p]
        L.or_tree_num_nodes.restype = C.c_int
        L.or_tree_num_leaves.argtypes = [C.c_void_p]
        L.or_tree_num_leaves.restype = C.c_int
        L.or_tree_nodes.argtypes = [C.c_void_p, _ip, _ip, _ip, _ip, _dp]
        L.or_tree_leaves.argtypes = [C.c_void_p, _ip, _ip]
        L.or_matvec.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp, _i64p, C.c_int]
        L.or_matvec_range.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp, C.c_int,
                                      C.c_int, _i64p, C.c_int]
        L.or_matvec_prepare.argtypes = [C.c_void_p, _dp]
        L.or_matvec_targets.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp, C.c_int,
                                        C.c_int, _i64p, C.c_int]
        L.or_matvec_direct.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, _dp,
                                       _dp, C.c_int]
        L.or_msolve_block.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, _dp, C.c_int,
                                      C.c_int, C.c_int]
        L.or_msolve_block.restype = C.c_int
        L.or_msolve_diag.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.or_dgetrf.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _ip]
        L.or_dgetrf.restype = C.c_int
        L.or_dgetrs.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _ip, _dp, C.c_int]
        L.or_dgmres.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, _dp, _dp,
                                C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int),
                                C.POINTER(C.c_double), _dp, C.POINTER(C.c_int), _i64p, _i64p,
                                C.c_int]
        L.or_dgmres.restype = C.c_int
        L.or_energy.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_double, C.c_double,
                                C.c_double, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                C.c_int]
        L.or_output_potential.argtypes = [C.c_int, _dp, C.c_int, _ip, _dp, _dp, _dp, _dp]
        L.or_output_potential.restype = None
        L.or_energy_surface.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, _dp, _dp, C.c_double,
                                        C.c_double, C.c_double, _dp, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.c_int]
        L.or_kappa.argtypes = [C.c_double, C.c_double]
        L.or_kappa.restype = C.c_double
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def kappa(bulk_strength: float, eps1: float) -> float:
    """main.f90:62-63 (REAL*4 literal 8.430325455)."""
    return lib().or_kappa(bulk_strength, eps1)


def surface_area(sptpos, nvert):
    """readin.f90:264-333.  nvert: (nface, 3) 1-based.  Returns (nvert_kept, s_area)."""
    sp = _d(sptpos).reshape(-1, 3)
    nv = _i(nvert).reshape(-1, 3).copy()
    s = C.c_double()
    nnew = lib().or_surface_area(sp.shape[0], sp.ravel(), nv.shape[0], nv.ravel(), C.byref(s))
    return nv[:nnew].copy(), s.value


def form_matrix(sptpos, sptnrm, nvert, chrpos, atmchr, eps0, nthreads=1):
    """main.f90:546-610.  Returns tr_xyz (N,3), tr_q (N,3), tr_area (N,), bvct (2N,)."""
    sp = _d(sptpos).reshape(-1, 3)
    sn = _d(sptnrm).reshape(-1, 3)
    nv = _i(nvert).reshape(-1, 3)
    cp = _d(chrpos).reshape(-1, 3)
    q = _d(atmchr).ravel()
    n = nv.shape[0]
    xyz = np.zeros((n, 3))
    tq = np.zeros((n, 3))
    ar = np.zeros(n)
    b = np.zeros(2 * n)
    lib().or_form_matrix(sp.shape[0], sp.ravel(), sn.ravel(), n, nv.ravel(), cp.shape[0],
                         cp.ravel(), q, float(eps0), xyz.ravel(), tq.ravel(), ar, b,
                         int(nthreads))
    return xyz, tq, ar, b


class Tree:
    """Tree-order state of treecode_initialization (main.f90:329-464)."""

    def __init__(self, tr_xyz, tr_q, tr_area, bvct, order, maxparnode, theta):
        self.xyz = _d(tr_xyz).reshape(-1, 3).copy()
        self.tq = _d(tr_q).reshape(-1, 3).copy()
        self.area = _d(tr_area).ravel().copy()
        self.n = self.xyz.shape[0]
        self.bvct = None if bvct is None else _d(bvct).ravel().copy()
        self.orderarr = np.zeros(self.n, dtype=np.int32)
        nleaf = C.c_int()
        bp = None if self.bvct is None else self.bvct.ctypes.data_as(C.c_void_p)
        self._h = lib().or_tree_create(self.n, self.xyz.ravel(), self.tq.ravel(), self.area, bp,
                                       int(order), int(maxparnode), float(theta), self.orderarr,
                                       C.byref(nleaf))
        self.nleaf = nleaf.value
        self.order, self.maxparnode, self.theta = order, maxparnode, theta

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().or_tree_free(h)
            self._h = None

    def nodes(self):
        nn = lib().or_tree_num_nodes(self._h)
        ib = np.zeros(nn, np.int32)
        ie = np.zeros(nn, np.int32)
        lv = np.zeros(nn, np.int32)
        nc = np.zeros(nn, np.int32)
        geo = np.zeros(4 * nn)
        lib().or_tree_nodes(self._h, ib, ie, lv, nc, geo)
        return dict(ibeg=ib, iend=ie, level=lv, nchild=nc, geo=geo.reshape(nn, 4))

    def leaves(self):
        ib = np.zeros(self.nleaf, np.int32)
        nr = np.zeros(self.nleaf, np.int32)
        lib().or_tree_leaves(self._h, ib, nr)
        return ib, nr

    def matvec(self, kappa, eps, x, nthreads=1, return_counts=False):
        x = _d(x).ravel()
        y = np.zeros_like(x)
        cnt = np.zeros(2, np.int64)
        lib().or_matvec(self._h, kappa, eps, x, y, cnt, int(nthreads))
        return (y, cnt) if return_counts else y

    def matvec_range(self, kappa, eps, x, i0, i1, nthreads=1):
        x = _d(x).ravel()
        y = np.zeros_like(x)
        cnt = np.zeros(2, np.int64)
        lib().or_matvec_range(self._h, kappa, eps, x, y, int(i0), int(i1), cnt, int(nthreads))
        return y, cnt

    def matvec_prepare(self, x):
        self._x = _d(x).ravel().copy()
        lib().or_matvec_prepare(self._h, self._x)

    def matvec_targets(self, kappa, eps, i0, i1, nthreads=1):
        """Target loop over [i0, i1) after matvec_prepare; returns (y, counts)."""
        y = np.zeros_like(self._x)
        cnt = np.zeros(2, np.int64)
        lib().or_matvec_targets(self._h, kappa, eps, self._x, y, int(i0), int(i1), cnt,
                                int(nthreads))
        return y, cnt

    def msolve(self, kappa, eps, r, iprcd=1, leaf0=0, leaf1=-1, nthreads=1):
        r = _d(r).ravel()
        z = np.zeros_like(r)
        if iprcd == 1:
            bad = lib().or_msolve_block(self._h, kappa, eps, r, z, int(leaf0), int(leaf1),
                                        int(nthreads))
            if bad:
                raise FloatingPointError(f"{bad} singular leaf blocks")
        else:
            lib().or_msolve_diag(r.size, eps, r, z)
        return z

    def dgmres(self, kappa, eps, b, iprcd=1, tol=1e-4, maxl=10, nrmax=10, x0=None,
               nthreads=1):
        b = _d(b).ravel()
        x = np.zeros_like(b) if x0 is None else _d(x0).ravel().copy()
        it = C.c_int()
        err = C.c_double()
        # DGMRES reads MAXL 0 as 10, NRMAX 0 as 10 and NRMAX -1 as no restart
        cap = ({0: 10, -1: 0}.get(nrmax, nrmax) + 1) * (maxl or 10)
        hist = np.zeros(cap + 2)
        nh = C.c_int()
        nmv = np.zeros(1, np.int64)
        nms = np.zeros(1, np.int64)
        ierr = lib().or_dgmres(self._h, kappa, eps, int(iprcd), b, x, float(tol), int(maxl),
                               int(nrmax), C.byref(it), C.byref(err), hist, C.byref(nh), nmv,
                               nms, int(nthreads))
        return dict(x=x, iter=it.value, err=err.value, ierr=ierr, err_hist=hist[: nh.value],
                    n_matvec=int(nmv[0]), n_msolve=int(nms[0]))

    def energy(self, chrpos, atmchr, kappa, eps, eps0, x, nthreads=1):
        cp = _d(chrpos).reshape(-1, 3)
        q = _d(atmchr).ravel()
        se = C.c_double()
        ce = C.c_double()
        lib().or_energy(self._h, cp.shape[0], cp.ravel(), q, kappa, eps, eps0, _d(x).ravel(),
                        C.byref(se), C.byref(ce), int(nthreads))
        return se.value, ce.value


def matvec_direct(tr_xyz, tr_q, tr_area, kappa, eps, x, nthreads=1):
    xyz = _d(tr_xyz).reshape(-1, 3)
    tq = _d(tr_q).reshape(-1, 3)
    ar = _d(tr_area).ravel()
    x = _d(x).ravel()
    y = np.zeros_like(x)
    lib().or_matvec_direct(xyz.shape[0], xyz.ravel(), tq.ravel(), ar, kappa, eps, x, y,
                           int(nthreads))
    return y


def energy_surface(tr_xyz, tr_q, tr_area, chrpos, atmchr, kappa, eps, eps0, x, nthreads=1):
    xyz = _d(tr_xyz).reshape(-1, 3)
    tq = _d(tr_q).reshape(-1, 3)
    cp = _d(chrpos).reshape(-1, 3)
    se = C.c_double()
    ce = C.c_double()
    lib().or_energy_surface(xyz.shape[0], xyz.ravel(), tq.ravel(), _d(tr_area).ravel(),
                            cp.shape[0], cp.ravel(), _d(atmchr).ravel(), kappa, eps, eps0,
                            _d(x).ravel(), C.byref(se), C.byref(ce), int(nthreads))
    return se.value, ce.value


def output_potential(sptpos, nvert, tr_xyz, x_orig):
    """main.f90:226-326: vertex potentials (nspt, 2) and the scaled face
    values (2 nface), from x and the centroids in the ORIGINAL face order."""
    sp = _d(sptpos).reshape(-1, 3)
    nv = _i(nvert).reshape(-1, 3)
    xyz = _d(tr_xyz).reshape(-1, 3)
    vert = np.zeros((sp.shape[0], 2))
    xs = np.zeros(2 * nv.shape[0])
    lib().or_output_potential(sp.shape[0], sp.ravel(), nv.shape[0], nv.ravel(), xyz.ravel(),
                              _d(x_orig).ravel(), vert.ravel(), xs)
    return vert, xs


def dgetrf(a):
    """DGETRF2 on a copy of a (square, numpy row-major input); returns (lu_colmajor, ipiv, info)."""
    a = np.asfortranarray(_d(a))
    m, n = a.shape
    buf = np.ascontiguousarray(a.T).ravel()  # column-major storage
    ipiv = np.zeros(min(m, n), np.int32)
    info = lib().or_dgetrf(m, n, buf, m, ipiv)
    return buf, ipiv, info


def dgetrs(lu, ipiv, n, b):
    b = _d(b).ravel().copy()
    lib().or_dgetrs(n, 1, lu, n, ipiv, b, n)
    return b
