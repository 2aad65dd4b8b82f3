"""Target-sharded solve across ranks (one process per GPU).

The targets of the tree order are split into contiguous, leaf-aligned ranges,
one per rank (`shard_bounds`).  Every rank holds the whole surface, tree and
cluster moments; its handle is restricted to its range
(`TabiSolver.set_target_range`), so a matvec computes the far and near
interactions of its own targets only and an apply of the leaf-block
preconditioner its own leaves only.  One all-gather of the slices then gives
every rank the full vector (`ShardedOperator`), and GMRES runs redundantly on
all ranks on identical data (`dgmres`, the DGMRES of dgmres_dep.f with
ITOL = 2, left preconditioning, MAXL = 10, KMP = MAXL, as the library's
single-GPU solve), so every rank takes the same steps and ends with the same
solution.

The exchange uses torch.distributed: NCCL between GPUs, gloo on the host.

Two drivers share that exchange.  `sharded_solve` runs the library's own
GMRES (tabi_solve) on every rank: the handle calls back after each operator
and preconditioner application (tabi_set_exchange) and `DeviceExchange`
completes the device vector in place on the library's stream, so the
vectors never leave the GPU with NCCL (gloo, a host backend, stages the
slices through host memory).  `ShardedOperator` + `dgmres` keep the
host-side form, which the CPU tests drive with the oracle's operator.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(leaf_starts, leaf_sizes, nshards):
    """Leaf-aligned [t0, t1) ranges of about equal face counts, in tree order.
    Returns an array of nshards + 1 boundaries."""
    starts = np.asarray(leaf_starts, np.int64)
    sizes = np.asarray(leaf_sizes, np.int64)
    o = np.argsort(starts, kind="stable")
    starts, sizes = starts[o], sizes[o]
    n = int(starts[-1] + sizes[-1])
    ends = starts + sizes
    bounds = [0]
    for k in range(1, nshards):
        target = n * k / nshards
        # the leaf end closest to the ideal cut, not before the previous bound
        j = int(np.argmin(np.abs(ends - target)))
        cut = int(ends[j])
        bounds.append(max(cut, bounds[-1]))
    bounds.append(n)
    return np.asarray(bounds, np.int64)


class ShardedOperator:
    """matvec / msolve of one rank's shard, completed by an all-gather.

    local_matvec(x) and local_msolve(r) return full-length vectors whose
    entries [t0, t1) and [n + t0, n + t1) are this rank's results (the rest is
    ignored); `allgather` assembles the full vector from every rank's slices.
    """

    def __init__(self, local_matvec, local_msolve, bounds, rank, group=None, device=None):
        self.local_matvec = local_matvec
        self.local_msolve = local_msolve
        self.bounds = np.asarray(bounds, np.int64)
        self.rank = rank
        self.group = group
        self.device = device
        self.n = int(self.bounds[-1])
        self.matvecs = 0
        self.msolves = 0

    def allgather(self, v):
        import torch
        import torch.distributed as dist

        n, b = self.n, self.bounds
        t0, t1 = int(b[self.rank]), int(b[self.rank + 1])
        width = int(np.max(np.diff(b)))
        mine = np.zeros(2 * width)
        mine[: t1 - t0] = v[t0:t1]
        mine[width: width + t1 - t0] = v[n + t0:n + t1]
        dev = self.device or "cpu"
        src = torch.from_numpy(mine).to(dev)
        parts = [torch.empty_like(src) for _ in range(len(b) - 1)]
        dist.all_gather(parts, src, group=self.group)
        out = np.empty(2 * n)
        for r, p in enumerate(parts):
            p = p.cpu().numpy()
            a0, a1 = int(b[r]), int(b[r + 1])
            out[a0:a1] = p[: a1 - a0]
            out[n + a0:n + a1] = p[width: width + a1 - a0]
        return out

    def matvec(self, x):
        self.matvecs += 1
        return self.allgather(self.local_matvec(x))

    def msolve(self, r):
        self.msolves += 1
        return self.allgather(self.local_msolve(r))


def _givens(t1, t2):
    # DHEQR (dgmres_dep.f:1031-1128) rotation coefficients
    if t2 == 0.0:
        return 1.0, 0.0
    if abs(t2) >= abs(t1):
        t = t1 / t2
        s = -1.0 / np.sqrt(1.0 + t * t)
        return -s * t, s
    t = t2 / t1
    c = 1.0 / np.sqrt(1.0 + t * t)
    return c, -c * t


def dgmres(matvec, msolve, b, x0=None, tol=1e-4, maxl=10, nrmax=10):
    """DGMRES (dgmres_dep.f:689-853 with DPIGMR, DORTH, DHEQR, DHELS, DRLCAL,
    ISDGMR) for ITOL = 2, left preconditioning, KMP = MAXL: stops when
    |M^-1 (b - A x)| / |M^-1 b| <= tol, the residual of a restart taken from
    the recurrence.  matvec follows MATVECmain's zero shortcut (the caller's
    operator does).  Returns dict(x, iter, err, ierr, err_hist)."""
    b = np.asarray(b, np.float64)
    n = b.size
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    maxl = min(maxl, n)
    kmp = maxl
    bnrm = np.linalg.norm(msolve(b))
    r = b - matvec(x)
    it, nrsts, err, ierr = 0, 0, 0.0, 0
    hist = []
    dl = None
    while True:
        if nrsts > nrmax:
            ierr = 1
            break
        if nrsts > 0:
            r = dl.copy()
        else:
            r = msolve(r)
        V = np.zeros((maxl + 1, n))
        V[0] = r
        r0nrm = np.linalg.norm(V[0])
        err = r0nrm / bnrm
        iflag, lgmr = 0, 0
        z = None
        if not err <= tol:
            V[0] /= r0nrm
            hes = np.zeros((maxl + 1, maxl))
            q = np.zeros(2 * maxl)
            prod, rho, snormw = 1.0, 0.0, 0.0
            go200 = go120 = False
            for ll in range(1, maxl + 1):
                lgmr = ll
                vn = msolve(matvec(V[ll - 1]))
                i0 = max(1, ll - kmp + 1)
                vnrm = np.linalg.norm(vn)
                for i in range(i0, ll + 1):
                    h = float(V[i - 1] @ vn)
                    hes[i - 1, ll - 1] = h
                    vn = vn - h * V[i - 1]
                snormw = np.linalg.norm(vn)
                if not (vnrm + 0.001 * snormw != vnrm):
                    sumdsq = 0.0
                    for i in range(i0, ll + 1):
                        tem = -float(V[i - 1] @ vn)
                        if hes[i - 1, ll - 1] + 0.001 * tem == hes[i - 1, ll - 1]:
                            continue
                        hes[i - 1, ll - 1] -= tem
                        vn = vn + tem * V[i - 1]
                        sumdsq += tem * tem
                    if sumdsq != 0.0:
                        snormw = np.sqrt(max(0.0, snormw * snormw - sumdsq))
                hes[ll, ll - 1] = snormw
                for k in range(1, ll):
                    t1, t2 = hes[k - 1, ll - 1], hes[k, ll - 1]
                    c, s = q[2 * (k - 1)], q[2 * (k - 1) + 1]
                    hes[k - 1, ll - 1] = c * t1 - s * t2
                    hes[k, ll - 1] = s * t1 + c * t2
                c, s = _givens(hes[ll - 1, ll - 1], hes[ll, ll - 1])
                q[2 * ll - 2], q[2 * ll - 1] = c, s
                hes[ll - 1, ll - 1] = c * hes[ll - 1, ll - 1] - s * hes[ll, ll - 1]
                if hes[ll - 1, ll - 1] == 0.0:
                    go120 = True
                    break
                prod *= q[2 * ll - 1]
                rho = abs(prod * r0nrm)
                # DRLCAL: the residual from the recurrence of the V columns
                cf = np.zeros(ll + 1)
                cf[0] = 1.0
                for i in range(1, ll):
                    si, ci = q[2 * i - 1], q[2 * i - 2]
                    cf[:i] *= si
                    cf[i] += ci
                cf[:ll] *= q[2 * ll - 1]
                cf[ll] += q[2 * ll - 2] / snormw
                cf *= r0nrm * prod
                V[ll] = vn
                dl = cf[: ll] @ V[:ll] + cf[ll] * vn
                err = np.linalg.norm(dl) / bnrm
                hist.append(err)
                if err <= tol:
                    go200 = True
                    break
                if ll == maxl:
                    break
                V[ll] = vn / snormw
            if not go200 and not go120:
                if rho < r0nrm:
                    iflag = 1
                    go200 = True
                else:
                    go120 = True
            if go120:
                iflag = 2
            else:
                l = lgmr
                y = np.zeros(l + 1)
                y[0] = r0nrm
                for k in range(1, l + 1):
                    c, s = q[2 * (k - 1)], q[2 * (k - 1) + 1]
                    t1, t2 = y[k - 1], y[k]
                    y[k - 1] = c * t1 - s * t2
                    y[k] = s * t1 + c * t2
                for kb in range(1, l + 1):
                    k = l + 1 - kb
                    y[k - 1] /= hes[k - 1, k - 1]
                    y[: k - 1] -= y[k - 1] * hes[: k - 1, k - 1]
                z = y[:l] @ V[:l] if l > 0 else np.zeros(n)
                # V[l] was overwritten by the unscaled vn above when l == maxl;
                # the update uses the first l columns only
        it += lgmr
        if z is not None:
            x = x + z
        if iflag == 0:
            ierr = 0
            break
        if iflag == 1:
            nrsts += 1
            continue
        ierr = 2
        break
    return dict(x=x, iter=it, err=err, ierr=ierr, err_hist=np.asarray(hist))


def _slice_index(bounds):
    """(width, index): the all-gather buffer holds rank r's slices at
    [r * 2 width, r * 2 width + t1 - t0) and [r * 2 width + width, ...); index
    maps every entry of the full 2n vector to its place in that buffer."""
    b = np.asarray(bounds, np.int64)
    n = int(b[-1])
    width = int(np.max(np.diff(b)))
    idx = np.empty(2 * n, np.int64)
    for r in range(len(b) - 1):
        a0, a1 = int(b[r]), int(b[r + 1])
        base = r * 2 * width
        idx[a0:a1] = base + np.arange(a1 - a0)
        idx[n + a0:n + a1] = base + width + np.arange(a1 - a0)
    return width, idx


def exchange_slices(v, bounds, rank, group=None, index=None):
    """Completes v (a torch tensor of 2n, on the host or the GPU) in place
    with every rank's slices [t0, t1) and [n + t0, n + t1) of the tree order:
    one all-gather of this rank's two slices, then one gather into v.  A CUDA
    tensor stays on the device with NCCL; gloo stages it through the host."""
    import torch
    import torch.distributed as dist

    b = np.asarray(bounds, np.int64)
    n = int(b[-1])
    width, idx = index if index is not None else _slice_index(b)
    t0, t1 = int(b[rank]), int(b[rank + 1])
    mine = torch.zeros(2 * width, dtype=v.dtype, device=v.device)
    mine[: t1 - t0] = v[t0:t1]
    mine[width:width + t1 - t0] = v[n + t0:n + t1]
    host = v.is_cuda and dist.get_backend(group) != "nccl"
    src = mine.cpu() if host else mine
    parts = [torch.empty_like(src) for _ in range(len(b) - 1)]
    dist.all_gather(parts, src, group=group)
    flat = torch.cat(parts).to(v.device)
    if not torch.is_tensor(idx):
        idx = torch.as_tensor(idx, device=v.device)
    v.copy_(flat[idx])


class _DevVec:
    """A raw device pointer of n doubles as a zero-copy torch tensor
    (__cuda_array_interface__)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


class DeviceExchange:
    """The tabi_set_exchange callback of one rank: completes the library's
    device vector on the library's stream (exchange_slices)."""

    def __init__(self, bounds, rank, group=None, device=None):
        import torch

        self.bounds = np.asarray(bounds, np.int64)
        self.rank = rank
        self.group = group
        self.device = torch.device(device if device is not None else "cuda")
        width, idx = _slice_index(self.bounds)
        self.index = (width, torch.as_tensor(idx, device=self.device))
        self.calls = 0

    def __call__(self, v_ptr, n2, t0, t1, stream):
        import torch

        assert n2 == 2 * int(self.bounds[-1])
        assert (t0, t1) == (int(self.bounds[self.rank]), int(self.bounds[self.rank + 1]))
        self.calls += 1
        with torch.cuda.stream(torch.cuda.ExternalStream(int(stream or 0), device=self.device)):
            v = torch.as_tensor(_DevVec(v_ptr, n2), device=self.device)
            exchange_slices(v, self.bounds, self.rank, self.group, self.index)


def sharded_solve(solver, b, bounds, rank, group=None, device=None):
    """The library's solve (tabi_solve: DGMRES, or GMRES-IR in mixed
    precision) across ranks: this rank's handle restricted to its shard, the
    exchange completing every operator and preconditioner result.  Every rank
    returns the same result, equal to the unsharded solve's."""
    solver.set_target_range(int(bounds[rank]), int(bounds[rank + 1]))
    ex = DeviceExchange(bounds, rank, group, device)
    solver.set_exchange(ex)
    try:
        res = solver.dgmres(b)
    except Exception:
        if getattr(solver, "exchange_error", None) is not None:
            raise solver.exchange_error
        raise
    finally:
        solver.set_exchange(None)
    res["exchanges"] = ex.calls
    return res
