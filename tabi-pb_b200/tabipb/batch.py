"""Batched solves of many molecules of uneven size (tabi_batch_run_dev) and the
leaf-size autotuner.

    mols = [make_molecule(natm, seed) for ...]          # device inputs
    table, _ = autotune(probe_mols, params)             # {size class: leaf size}
    stats, wall = run_batch(mols, params, ws=ws, nworkers=4, table=table)

The library runs the molecules on `nworkers` host threads, each with its own
handle and streams, so the latency-bound phases of one molecule overlap the
work of others; molecules are taken largest first.  The autotuner times the
whole solve of a probe molecule of each size class for every candidate leaf
size and keeps the fastest; the Taylor order and MAC are accuracy settings and
stay as given (the leaf size changes only how the work splits between near
field, far field and preconditioner, and the iteration count).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from ._lib import BATCH_STATS, MolDev, check

STAT_NAMES = ("iter", "err", "ierr", "soleng", "couleng", "near_pairs", "far", "nleaf",
              "wall_ms", "done_ms", "worker", "maxparnode")
# faces per size class boundary (classes: < 40k, < 120k, < 250k, >= 250k)
CLASS_EDGES = (40_000, 120_000, 250_000)


def size_class(nface):
    return int(np.searchsorted(CLASS_EDGES, nface, side="right"))


def make_molecule(natm, seed, density=10.0, device="cuda"):
    """A synthetic globule at the benchmark density and its surface, as device
    tensors (the inputs of tabi_run_dev)."""
    import torch

    from . import surface as S
    from .warmstart import globular_radius

    xyz, q, r = S.synthetic_molecule(natm, globular_radius(natm), min_sep=2.0, seed=seed)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=density, probe=1.4)
    fc, _ = S.face_filter(pos, fc)
    dev = torch.device(device)
    f = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    return dict(natm=natm, seed=seed, nspt=len(pos), nface=len(fc), nchr=natm,
                sptpos=f(pos), sptnrm=f(nrm),
                nvert=torch.from_numpy(np.ascontiguousarray(fc, dtype=np.int32)).to(dev),
                chrpos=f(xyz), atmchr=f(q))


def _moldev(m, maxparnode=0, order=0):
    p = lambda t: C.c_void_p(t.data_ptr())
    return MolDev(m["nspt"], p(m["sptpos"]), p(m["sptnrm"]), m["nface"], p(m["nvert"]),
                  m["nchr"], p(m["chrpos"]), p(m["atmchr"]), int(maxparnode), int(order))


def run_batch(mols, params, ws=None, nworkers=4, table=None):
    """Solves every molecule; returns an (nmol, 12) array of STAT_NAMES and the
    batch wall time in seconds.  table: {size class: leaf size} (autotune)."""
    L = _lib.load()
    arr = (MolDev * len(mols))()
    for k, m in enumerate(mols):
        leaf = table.get(size_class(m["nface"]), 0) if table else 0
        arr[k] = _moldev(m, maxparnode=leaf)
    st = np.zeros((len(mols), BATCH_STATS))
    t0 = time.perf_counter()
    check(None, L.tabi_batch_run_dev(C.byref(params), len(mols), arr,
                                     ws.h if ws is not None else None, int(nworkers),
                                     st.ctypes.data_as(C.POINTER(C.c_double))))
    return st, time.perf_counter() - t0


def autotune(probes, params, candidates=(200, 300, 400, 500, 700), repeats=2, log=None):
    """For each probe molecule (one per size class is enough), time the whole
    solve (one worker, so the molecule has the GPU to itself) for every
    candidate leaf size; returns {size class: fastest leaf size} and the
    timings {(class, leaf): ms}."""
    table, timings = {}, {}
    for m in probes:
        c = size_class(m["nface"])
        best = None
        for leaf in candidates:
            ts = []
            for _ in range(repeats):
                st, _ = run_batch([m], params, nworkers=1, table={c: leaf})
                ts.append(st[0, 8])
            t = min(ts)
            timings[(c, leaf)] = t
            if log:
                log(f"class {c} ({m['nface']} faces) leaf {leaf}: {t:.2f} ms, "
                    f"{int(st[0, 0])} iterations")
            if best is None or t < best[0]:
                best = (t, leaf)
        table[c] = best[1]
    return table, timings


def tune_workers(mols, params, table, candidates=(1, 2, 4), ws=None, repeats=2):
    """Times the batch call on `mols` for each worker count and returns the
    fastest count and the timings {workers: s}.  Concurrency pays when one
    molecule's launches leave the GPU idle (host round trips, short launch
    chains); when each solve already fills the GPU, extra workers only
    contend, so the count is measured, not assumed."""
    timings = {}
    for nw in candidates:
        ts = []
        for _ in range(repeats):
            _, t = run_batch(mols, params, ws=ws, nworkers=nw, table=table)
            ts.append(t)
        timings[nw] = min(ts)
    best = min(timings, key=timings.get)
    return best, timings
