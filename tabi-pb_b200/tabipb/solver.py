"""Host-side mirror of the reference's solve interface, over libtabi_gpu.so.

The reference keeps its state in Fortran modules and exposes the solve as
subroutines called from main.f90; ``TabiSolver`` mirrors that interface
method by method (same names, same argument meaning, same array layouts):

    form_matrix()              main.f90:546-610
    treecode_initialization()  main.f90:329-464 (tree + permutation)
    matvec(x)                  MATVECmain, main.f90:467-488
    msolve(r)                  MSOLVEdric / MSOLVEprec, main.f90:511-542
    dgmres(b)                  DGMRES call, main.f90:92-139
    energy(x)                  main.f90:144-159 (+ potential_molecule)
    output_potential(x)        main.f90:226-326

All numerics run on the GPU; errors from the library raise TabiError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import Params, TabiError, check, dptr, f64, i32, iptr


def kappa(bulk_strength: float, eps1: float) -> float:
    """main.f90:62-63."""
    return _lib.load().tabi_kappa(float(bulk_strength), float(eps1))


def default_params(**kw) -> Params:
    p = Params()
    _lib.load().tabi_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


class TabiSolver:
    """One molecule's solve state (the reference's module globals)."""

    def __init__(self, params: Params | None = None, **kw):
        self.L = _lib.load()
        self.params = params if params is not None else default_params(**kw)
        h = C.c_void_p()
        rc = self.L.tabi_create(C.byref(h), C.byref(self.params))
        if rc != 0:
            raise TabiError(rc, self.L.tabi_last_error(None).decode())
        self.h = h
        self.nface = 0
        self.orderarr = None
        self.nleaf = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.tabi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def eps(self):
        return self.params.eps1 / self.params.eps0

    # ---- main.f90:546-610
    def form_matrix(self, sptpos, sptnrm, nvert, chrpos, atmchr, out=None):
        """out: optional (tr_xyz (n,3), tr_q (n,3), tr_area (n), bvct (2n))
        float64 C-contiguous arrays to write into (e.g. page-locked ones)."""
        sp = f64(sptpos, (-1, 3))
        sn = f64(sptnrm, (-1, 3))
        nv = i32(nvert).reshape(-1, 3)
        cp = f64(chrpos, (-1, 3))
        q = f64(atmchr).ravel()
        n = nv.shape[0]
        if out is None:
            xyz, tq, ar, b = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(2 * n)
        else:
            xyz, tq, ar, b = out
            for a, shape in ((xyz, (n, 3)), (tq, (n, 3)), (ar, (n,)), (b, (2 * n,))):
                if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError(f"out array of shape {shape}, float64, C order expected")
        check(self.h, self.L.tabi_form_matrix(self.h, sp.shape[0], dptr(sp), dptr(sn), n,
                                              iptr(nv), cp.shape[0], dptr(cp), dptr(q),
                                              dptr(xyz), dptr(tq), dptr(ar), dptr(b)))
        self.nface = n
        return xyz, tq, ar, b

    def set_surface(self, tr_xyz, tr_q, tr_area):
        xyz = f64(tr_xyz, (-1, 3))
        tq = f64(tr_q, (-1, 3))
        ar = f64(tr_area).ravel()
        check(self.h, self.L.tabi_set_surface(self.h, xyz.shape[0], dptr(xyz), dptr(tq),
                                              dptr(ar)))
        self.nface = xyz.shape[0]

    def rhs(self, chrpos, atmchr):
        cp = f64(chrpos, (-1, 3))
        q = f64(atmchr).ravel()
        b = np.zeros(2 * self.nface)
        check(self.h, self.L.tabi_rhs(self.h, cp.shape[0], dptr(cp), dptr(q), dptr(b)))
        return b

    # ---- main.f90:400-453
    def build_tree(self):
        oa = np.zeros(self.nface, np.int32)
        nl = C.c_int()
        check(self.h, self.L.tabi_build_tree(self.h, iptr(oa), C.byref(nl)))
        self.orderarr = oa
        self.nleaf = nl.value
        return oa, nl.value

    def permute(self, tr_xyz=None, tr_q=None, tr_area=None, bvct=None):
        """main.f90:447-453: arrays in original order -> tree order."""
        o = self.orderarr - 1
        n = self.nface
        out = []
        for a in (tr_xyz, tr_q, tr_area):
            out.append(None if a is None else np.asarray(a)[o].copy())
        if bvct is not None:
            b = np.asarray(bvct)
            out.append(np.concatenate([b[:n][o], b[n:][o]]))
        else:
            out.append(None)
        return out

    def unpermute(self, v):
        """Tree-order 2N vector -> original order (output_potential, main.f90:249-253)."""
        o = self.orderarr - 1
        n = self.nface
        v = np.asarray(v)
        out = np.empty_like(v)
        out[o] = v[:n]
        out[n + o] = v[n:]
        return out

    # ---- operators
    def matvec(self, x):
        x = f64(x).ravel()
        y = np.zeros_like(x)
        check(self.h, self.L.tabi_matvec(self.h, x.size, dptr(x), dptr(y)))
        return y

    def msolve(self, r):
        r = f64(r).ravel()
        z = np.zeros_like(r)
        check(self.h, self.L.tabi_msolve(self.h, r.size, dptr(r), dptr(z)))
        return z

    def dgmres(self, b, x0=None, out=None):
        """out: optional float64 array of 2n for the solution (e.g. page-locked)."""
        b = f64(b).ravel()
        if out is None:
            x = np.zeros_like(b) if x0 is None else f64(x0).ravel().copy()
        else:
            if out.shape != b.shape or out.dtype != np.float64 or not out.flags.c_contiguous:
                raise ValueError("out must be a float64 C-order array like b")
            x = out
            x[:] = 0.0 if x0 is None else f64(x0).ravel()
        it, ierr, nh = C.c_int(), C.c_int(), C.c_int()
        err = C.c_double()
        # DGMRES reads MAXL 0 as 10, NRMAX 0 as 10 and NRMAX -1 as no restart
        maxl = self.params.maxl or 10
        nrmax = {0: 10, -1: 0}.get(self.params.nrmax, self.params.nrmax)
        hist = np.zeros((nrmax + 1) * maxl + 2)
        check(self.h, self.L.tabi_solve(self.h, b.size, dptr(b), dptr(x), C.byref(it),
                                        C.byref(err), C.byref(ierr), dptr(hist), C.byref(nh)))
        return dict(x=x, iter=it.value, err=err.value, ierr=ierr.value,
                    err_hist=hist[: nh.value].copy())

    def energy(self, chrpos, atmchr, x):
        cp = f64(chrpos, (-1, 3))
        q = f64(atmchr).ravel()
        x = f64(x).ravel()
        se, ce = C.c_double(), C.c_double()
        check(self.h, self.L.tabi_energy(self.h, cp.shape[0], dptr(cp), dptr(q), dptr(x),
                                         C.byref(se), C.byref(ce)))
        return se.value, ce.value

    # ---- accuracy reference
    def direct_targets(self, targets, x):
        """FP64 direct sum of the operator at the given targets (current face
        order, 0-based): returns (y1, y2) of those targets."""
        t = i32(targets).ravel()
        x = f64(x).ravel()
        y = np.zeros(2 * t.size)
        check(self.h, self.L.tabi_direct_targets(self.h, t.size, iptr(t), dptr(x), dptr(y)))
        return y[: t.size], y[t.size:]

    # ---- shards of the operator
    def leaves(self):
        """(start, size) of each leaf in tree order (0-based starts)."""
        t = self.tree_nodes()
        m = t["nchild"] == 0
        st = t["ibeg"][m] - 1
        o = np.argsort(st, kind="stable")
        return st[o].astype(np.int64), t["numpar"][m][o].astype(np.int64)

    def set_target_range(self, t0, t1):
        """Restrict matvec / msolve to the tree-order targets [t0, t1)
        (leaf-aligned): only that slice of y / z is written."""
        check(self.h, self.L.tabi_set_target_range(self.h, int(t0), int(t1)))

    def set_exchange(self, fn):
        """The exchange of a target-sharded solve (tabi_set_exchange):
        fn(v_dev_ptr, n2, t0, t1, stream_ptr) completes the device vector in
        place with the other ranks' slices and returns None, or raises.  None
        removes it.  The ctypes callback is kept alive by the solver."""
        if fn is None:
            self._xchg = None
            check(self.h, self.L.tabi_set_exchange(self.h, _lib.EXCHANGE_FN(), None))
            return

        def cb(user, v, n2, t0, t1, stream):
            try:
                fn(v, n2, t0, t1, stream)
                return 0
            except Exception as e:  # noqa: BLE001 -- reported through the return code
                self.exchange_error = e
                return 1

        self._xchg = _lib.EXCHANGE_FN(cb)
        self.exchange_error = None
        check(self.h, self.L.tabi_set_exchange(self.h, self._xchg, None))

    # ---- main.f90:226-326
    def output_potential(self, sptpos, nvert, x):
        """x (tree order, as dgmres returns it) -> (x in the original face order
        and vertex values (nspt, 2): potential, normal derivative), both scaled
        by 332.0716 * 4 pi as the reference writes them."""
        sp = f64(sptpos, (-1, 3))
        nv = i32(nvert).reshape(-1, 3)
        x = f64(x).ravel()
        xo = np.zeros_like(x)
        vert = np.zeros((sp.shape[0], 2))
        check(self.h, self.L.tabi_output_potential(self.h, sp.shape[0], dptr(sp), nv.shape[0],
                                                   iptr(nv), dptr(x), dptr(xo), dptr(vert)))
        return xo, vert

    def pivoted_leaves(self):
        """Leaf blocks factored with partial pivoting (tabi_pivoted_leaves)."""
        c = C.c_int()
        check(self.h, self.L.tabi_pivoted_leaves(self.h, C.byref(c)))
        return c.value

    def counts(self):
        a, b = C.c_int64(), C.c_int64()
        check(self.h, self.L.tabi_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def tree_nodes(self):
        nn = C.c_int()
        check(self.h, self.L.tabi_tree_nodes(self.h, C.byref(nn), None, None, None, None, None))
        k = nn.value
        ib = np.zeros(k, np.int32)
        nu = np.zeros(k, np.int32)
        lv = np.zeros(k, np.int32)
        nc = np.zeros(k, np.int32)
        geo = np.zeros(4 * k)
        check(self.h, self.L.tabi_tree_nodes(self.h, C.byref(nn), iptr(ib), iptr(nu), iptr(lv),
                                             iptr(nc), dptr(geo)))
        return dict(ibeg=ib, numpar=nu, level=lv, nchild=nc, geo=geo.reshape(k, 4))

    # ---- instrumentation
    def profile(self, enable=True):
        check(self.h, self.L.tabi_profile_enable(self.h, 1 if enable else 0))

    def profile_read(self):
        """{class: (ms, launches)} plus 'all'."""
        out = {}
        for k in list(range(self.L.tabi_profile_nclasses())) + [-1]:
            ms, nl = C.c_double(), C.c_int64()
            check(self.h, self.L.tabi_profile_read(self.h, k, C.byref(ms), C.byref(nl)))
            out[self.L.tabi_profile_class_name(k).decode()] = (ms.value, nl.value)
        return out

    # ---- device-pointer entry points (torch tensors or raw pointers)
    def matvec_dev(self, x_ptr, y_ptr, n2, stream=None):
        check(self.h, self.L.tabi_matvec_dev(self.h, n2, x_ptr, y_ptr, stream))

    def face_filter_dev(self, nspt, sptpos_ptr, nface, nvert_ptr, nvert_out_ptr, stream=None):
        """readin.f90:264-333 on device arrays (tabi_face_filter_dev): returns
        (kept face count, total area); the kept faces go to nvert_out_ptr."""
        nk, sa = C.c_int(), C.c_double()
        check(self.h, self.L.tabi_face_filter_dev(self.h, nspt, sptpos_ptr, nface, nvert_ptr,
                                                  nvert_out_ptr, C.byref(nk), C.byref(sa),
                                                  stream))
        return nk.value, sa.value

    def set_warmstart(self, ws):
        """Attach a warmstart.WarmStart (None detaches): run_dev then starts
        GMRES from the network's prediction (tabi_set_warmstart)."""
        check(self.h, self.L.tabi_set_warmstart(self.h, ws.h if ws is not None else None))
        self._ws = ws  # the handle does not own the network

    def run_dev(self, nspt, sptpos_ptr, sptnrm_ptr, nface, nvert_ptr, nchr, chrpos_ptr,
                atmchr_ptr, x_ptr=None, stream=None):
        st = np.zeros(8)
        check(self.h, self.L.tabi_run_dev(self.h, nspt, sptpos_ptr, sptnrm_ptr, nface,
                                          nvert_ptr, nchr, chrpos_ptr, atmchr_ptr, x_ptr,
                                          dptr(st), stream))
        self.nface = nface
        return dict(iter=int(st[0]), err=st[1], ierr=int(st[2]), soleng=st[3], couleng=st[4],
                    near_pairs=int(st[5]), far=int(st[6]), nleaf=int(st[7]))


def probe_fp64_peak(ms=200.0) -> float:
    f = C.c_double()
    rc = _lib.load().tabi_probe_fp64_peak(ms, C.byref(f))
    if rc != 0:
        raise TabiError(rc, "fp64 probe failed")
    return f.value


def probe_fp32_peak(ms=200.0) -> float:
    f = C.c_double()
    rc = _lib.load().tabi_probe_fp32_peak(ms, C.byref(f))
    if rc != 0:
        raise TabiError(rc, "fp32 probe failed")
    return f.value


def solve_molecule(sptpos, sptnrm, nvert, chrpos, atmchr, **params):
    """The whole main.f90 sequence for one molecule on host arrays:
    form_matrix -> tree -> DGMRES -> energy.  Returns a result dict with the
    solution in the ORIGINAL face order."""
    with TabiSolver(**params) as s:
        xyz, tq, ar, b = s.form_matrix(sptpos, sptnrm, nvert, chrpos, atmchr)
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b)
        res = s.dgmres(bt)
        se, ce = s.energy(chrpos, atmchr, res["x"])
        res.update(soleng=se, couleng=ce, x_orig=s.unpermute(res["x"]), nleaf=s.nleaf,
                   counts=s.counts())
        return res
