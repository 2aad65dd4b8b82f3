"""Learned warm start: the panel network of libtabi_gpu.so (tabi_ws_*).

The network predicts the initial guess x0 = [phi; dphi/dn] of a solve from
the panel geometry, the right-hand side b and z = M^-1 b, the leaf-block
preconditioner's solution, which it corrects; GMRES on the true residual runs
from there, so only the iteration count changes.  It is trained on the GPU by
the library's own forward, backward and Adam kernels, on solutions this solver
produces for synthetic molecules.

    ws = WarmStart(hidden=160, layers=3, seed=0)      # 238,402 parameters
    samples = [make_sample(natm, seed) for ...]      # solved molecules (device)
    train(ws, samples, epochs=20)
    ws.save("ws.npz");  ws = WarmStart.load("ws.npz")
    solver.set_warmstart(ws)                         # run_dev starts from x0

Device arrays are torch tensors (CUDA); all numerics run in the library.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from ._lib import TabiError, check

K_NEIGHBOURS = 16
NODE_FEATURES = 10  # per panel, as the library writes them (tabi_ws_graph_dev)
# atoms per A^3 of the globular benchmark molecule (2,000 atoms in 18 A)
GLOBULAR_DENSITY = 2000 / (4.0 / 3.0 * np.pi * 18.0 ** 3)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    """The stream a call runs on: the given one, else torch's current stream
    (so the call is ordered with the torch operations around it; torch's
    default stream is the CUDA default stream, NULL)."""
    if stream is not None:
        return C.c_void_p(stream)
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class WarmStart:
    """One network (tabi_ws); see include/tabi_gpu.h."""

    def __init__(self, hidden=160, layers=3, seed=0):
        self.L = _lib.load()
        h = C.c_void_p()
        rc = self.L.tabi_ws_create(C.byref(h), int(hidden), int(layers), int(seed))
        if rc != 0:
            raise TabiError(rc, self.L.tabi_last_error(None).decode())
        self.h = h
        self.hidden, self.layers = int(hidden), int(layers)

    def close(self):
        if getattr(self, "h", None):
            self.L.tabi_ws_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        return check(None, rc)

    @property
    def nparams(self):
        return int(self.L.tabi_ws_nparams(self.h))

    def params(self):
        th = np.zeros(self.nparams, np.float32)
        self._check(self.L.tabi_ws_get_params(self.h, th.ctypes.data_as(C.POINTER(C.c_float)),
                                              th.size))
        return th

    def set_params(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float32)
        self._check(self.L.tabi_ws_set_params(self.h, th.ctypes.data_as(C.POINTER(C.c_float)),
                                              th.size))

    def save(self, path, **meta):
        np.savez(path, theta=self.params(), hidden=self.hidden, layers=self.layers,
                 **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path):
        z = np.load(path)
        ws = cls(int(z["hidden"]), int(z["layers"]))
        ws.set_params(z["theta"])
        return ws

    # ---- device entry points (sample: dict of CUDA tensors, see make_sample;
    # its "z" = M^-1 b may be absent)
    def predict_dev(self, s, x_out, stream=None):
        self._check(self.L.tabi_ws_predict_dev(self.h, s["n"], _ptr(s["xyz"]), _ptr(s["tq"]),
                                               _ptr(s["area"]), _ptr(s["b"]), _ptr(s.get("z")),
                                               _ptr(x_out), _stream(stream)))

    def loss_grad_dev(self, s, want_grad=True, stream=None):
        loss = C.c_double()
        g = np.zeros(self.nparams, np.float32) if want_grad else None
        self._check(self.L.tabi_ws_loss_grad_dev(
            self.h, s["n"], _ptr(s["xyz"]), _ptr(s["tq"]), _ptr(s["area"]), _ptr(s["b"]),
            _ptr(s.get("z")), _ptr(s["x"]), C.byref(loss),
            g.ctypes.data_as(C.POINTER(C.c_float)) if g is not None else None, _stream(stream)))
        return loss.value, g

    def train_step_dev(self, s, lr, stream=None):
        loss = C.c_double()
        self._check(self.L.tabi_ws_train_step_dev(
            self.h, s["n"], _ptr(s["xyz"]), _ptr(s["tq"]), _ptr(s["area"]), _ptr(s["b"]),
            _ptr(s.get("z")), _ptr(s["x"]), float(lr), C.byref(loss), _stream(stream)))
        return loss.value

    def graph_dev(self, s, stream=None):
        n = s["n"]
        # the input layer is NODE_FEATURES x hidden (+ hidden biases) at the
        # head of the parameters: check the host buffers match the library
        w0 = self.params()[: NODE_FEATURES * self.hidden]
        if self.nparams != _expected_nparams(self.hidden, self.layers) or w0.size == 0:
            raise TabiError(-1, "network layout does not match this binding")
        nbr = np.zeros((n, K_NEIGHBOURS), np.int32)
        feat = np.zeros((n, NODE_FEATURES), np.float32)
        self._check(self.L.tabi_ws_graph_dev(
            self.h, n, _ptr(s["xyz"]), _ptr(s["tq"]), _ptr(s["area"]), _ptr(s["b"]),
            _ptr(s.get("z")), nbr.ctypes.data_as(C.POINTER(C.c_int)), feat.ctypes.data_as(C.POINTER(C.c_float)),
            _stream(stream)))
        return nbr, feat


def _expected_nparams(hidden, layers, radial=8):
    edge = radial + 3
    per_layer = 3 * hidden * hidden + edge * hidden + 2 * hidden
    return NODE_FEATURES * hidden + hidden + layers * per_layer + 2 * hidden + 2


def globular_radius(natm):
    """Sphere radius holding natm atoms at the benchmark molecule's density."""
    return (natm / (4.0 / 3.0 * np.pi * GLOBULAR_DENSITY)) ** (1.0 / 3.0)


def make_sample(natm, seed, density=10.0, tol=1e-6, precision=None, maxparnode=500, order=3,
                theta=0.8, device="cuda"):
    """One training / evaluation molecule: a synthetic globule (the benchmark
    generator at the benchmark density), its surface, and its solution by this
    solver (tree order, GMRES from zero to `tol`).  Returns a dict of CUDA
    tensors (xyz, tq: 3n interleaved; area: n; b, z = M^-1 b, x: 2n) plus n,
    natm, the iteration count and the host inputs needed to solve it again."""
    import torch

    from . import surface as S
    from ._lib import PREC_MIXED
    from .solver import TabiSolver, kappa

    xyz, q, r = S.synthetic_molecule(natm, globular_radius(natm), min_sep=2.0, seed=seed)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=density, probe=1.4)
    fc, _ = S.face_filter(pos, fc)
    prm = dict(order=order, maxparnode=maxparnode, theta=theta, kappa=kappa(0.15, 80.0),
               eps0=1.0, eps1=80.0, tol=tol,
               precision=PREC_MIXED if precision is None else precision)
    with TabiSolver(**prm) as s:
        txyz, ttq, tar, b = s.form_matrix(pos, nrm, fc, xyz, q)
        s.build_tree()
        txyz, ttq, tar, bt = s.permute(txyz, ttq, tar, b)
        zt = s.msolve(bt)
        res = s.dgmres(bt)
    dev = torch.device(device)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).ravel()).to(dev)
    return dict(n=len(tar), natm=natm, seed=seed, xyz=t(txyz), tq=t(ttq), area=t(tar), b=t(bt),
                z=t(zt), x=t(res["x"]), iters=res["iter"], ierr=res["ierr"],
                host=dict(sptpos=pos, sptnrm=nrm, nvert=fc, chrpos=xyz, atmchr=q), prm=prm)


def train(ws, samples, epochs=10, lr=1e-3, lr_final=1e-4, seed=0, log=None):
    """Adam over the samples whose solve converged, one molecule per step,
    shuffled each epoch, learning rate decayed geometrically from lr to
    lr_final.  Returns the per-epoch mean losses."""
    rng = np.random.default_rng(seed)
    samples = [s for s in samples if s.get("ierr", 0) == 0]  # converged solutions only
    steps = max(1, epochs * len(samples))
    gamma = (lr_final / lr) ** (1.0 / max(1, steps - 1))
    k = 0
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(samples))
        tot = 0.0
        t0 = time.perf_counter()
        for i in order:
            tot += ws.train_step_dev(samples[i], lr * gamma ** k)
            k += 1
        hist.append(tot / len(samples))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f} ({time.perf_counter() - t0:.2f} s)")
    return hist


def evaluate(ws, samples, tol=1e-6, precision=None):
    """GMRES iterations and solve time from x0 = 0 and from the network's x0
    for each sample (same tree, same tolerance), and the iterations from the
    network's baseline z = M^-1 b alone.  Returns a list of dicts."""
    import torch

    from .solver import TabiSolver

    out = []
    for s in samples:
        prm = dict(s["prm"], tol=tol)
        if precision is not None:
            prm["precision"] = precision
        h = s["host"]
        with TabiSolver(**prm) as sv:
            sv.form_matrix(h["sptpos"], h["sptnrm"], h["nvert"], h["chrpos"], h["atmchr"])
            sv.build_tree()
            b = s["b"].cpu().numpy()
            x0 = torch.empty_like(s["b"])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ws.predict_dev(s, x0)
            torch.cuda.synchronize()
            t_pred = time.perf_counter() - t0
            t1 = time.perf_counter()
            r_ws = sv.dgmres(b, x0.cpu().numpy())
            t2 = time.perf_counter()
            r_0 = sv.dgmres(b)
            t3 = time.perf_counter()
            r_z = sv.dgmres(b, s["z"].cpu().numpy()) if "z" in s else r_0
        xt = s["x"].cpu().numpy()
        out.append(dict(n=s["n"], natm=s["natm"], iters_zero=r_0["iter"], iters_ws=r_ws["iter"],
                        iters_baseline=r_z["iter"],
                        ierr=(r_0["ierr"], r_ws["ierr"]), predict_s=t_pred,
                        solve_s_ws=t2 - t1, solve_s_zero=t3 - t2,
                        x0_rel_err=float(np.linalg.norm(x0.cpu().numpy() - xt)
                                         / np.linalg.norm(xt))))
    return out
