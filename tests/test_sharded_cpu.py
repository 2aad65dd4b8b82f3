"""Target-sharded solve on two host ranks (gloo): each rank computes its
leaf-aligned shard of the operator and of the leaf-block preconditioner with
the CPU oracle, one all-gather completes every vector, and GMRES
(tabipb.sharded.dgmres) runs redundantly on both ranks.  The assembled
operator and preconditioner equal the unsharded oracle's bit for bit, the
ranks end with identical solutions, and the solve matches the oracle's own
DGMRES (same iteration count and residual history, solution to 1e-10)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path[:0] = [here, os.path.join(root, "tabi-pb_b200"), os.path.join(root, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    import oracle as O
    from conftest import BULK, EPS0, EPS1, molecule_case
    from tabipb import sharded as SH

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        c = molecule_case(60, 6.0, 2.0, seed=1)
        xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                       c["atmchr"], EPS0)
        T = O.Tree(xyz, tq, ar, b, 3, 200, 0.8)
        kap, eps = O.kappa(BULK, EPS1), EPS1 / EPS0
        ib, nr = T.leaves()  # creation order, 1-based starts
        starts = ib - 1
        bounds = SH.shard_bounds(starts, nr, world)
        t0, t1 = int(bounds[rank]), int(bounds[rank + 1])
        mine = [l for l in range(len(ib)) if starts[l] >= t0 and starts[l] + nr[l] <= t1]

        def local_matvec(x):
            return T.matvec_range(kap, eps, x, t0, t1)[0]

        def local_msolve(r):
            z = np.zeros_like(r)
            for l in mine:
                z += T.msolve(kap, eps, r, leaf0=l, leaf1=l + 1)
            return z

        op = SH.ShardedOperator(local_matvec, local_msolve, bounds, rank)
        bt = T.bvct
        x = np.random.default_rng(3).standard_normal(bt.size)
        y, z = op.matvec(x), op.msolve(x)
        res = SH.dgmres(op.matvec, op.msolve, bt, tol=1e-4)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), y=y, z=z, x=res["x"], iter=res["iter"],
                 err=res["err"], ierr=res["ierr"], hist=res["err_hist"], bounds=bounds,
                 nmine=len(mine))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_solve(tmp_path):
    import torch.multiprocessing as mp

    import oracle as O
    from conftest import BULK, EPS0, EPS1, molecule_case

    mp.start_processes(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"rank{k}.npz") for k in (0, 1))
    c = molecule_case(60, 6.0, 2.0, seed=1)
    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], EPS0)
    T = O.Tree(xyz, tq, ar, b, 3, 200, 0.8)
    kap, eps = O.kappa(BULK, EPS1), EPS1 / EPS0
    x = np.random.default_rng(3).standard_normal(2 * len(ar))
    # the shards split the targets and the leaves
    bnd = r0["bounds"]
    assert bnd[0] == 0 and bnd[-1] == len(ar) and 0 < bnd[1] < len(ar)
    assert int(r0["nmine"]) + int(r1["nmine"]) == len(T.leaves()[0])
    # assembled operator and preconditioner == unsharded, bit for bit
    np.testing.assert_array_equal(r0["y"], T.matvec(kap, eps, x))
    np.testing.assert_array_equal(r0["z"], T.msolve(kap, eps, x))
    np.testing.assert_array_equal(r0["y"], r1["y"])
    # both ranks end in the same state
    np.testing.assert_array_equal(r0["x"], r1["x"])
    assert int(r0["iter"]) == int(r1["iter"])
    # and the solve is the oracle's DGMRES
    ref = T.dgmres(kap, eps, T.bvct, iprcd=1, tol=1e-4)
    assert int(r0["ierr"]) == 0 == ref["ierr"]
    assert int(r0["iter"]) == ref["iter"], (int(r0["iter"]), ref["iter"])
    np.testing.assert_allclose(r0["hist"], ref["err_hist"][: len(r0["hist"])], rtol=1e-8)
    assert np.linalg.norm(r0["x"] - ref["x"]) <= 1e-10 * np.linalg.norm(ref["x"])


def test_shard_bounds_are_leaf_aligned_and_balanced():
    from tabipb.sharded import shard_bounds

    rng = np.random.default_rng(1)
    sizes = rng.integers(20, 500, 300)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    perm = rng.permutation(len(sizes))  # any leaf order
    for k in (1, 2, 3, 8):
        b = shard_bounds(starts[perm], sizes[perm], k)
        assert b[0] == 0 and b[-1] == sizes.sum() and np.all(np.diff(b) >= 0)
        ends = set((starts + sizes).tolist()) | {0}
        assert all(int(v) in ends for v in b)
        assert np.diff(b).max() <= sizes.sum() / k + sizes.max()


def _exchange_rank(rank, world, port, outdir, bounds):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path[:0] = [here, os.path.join(root, "tabi-pb_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist

    from tabipb import sharded as SH

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        b = np.asarray(bounds)
        n = int(b[-1])
        full = torch.arange(2 * n, dtype=torch.float64) * 0.5 + 1.0
        # this rank knows its own slices only; the rest is garbage
        v = torch.full((2 * n,), float("nan"), dtype=torch.float64)
        t0, t1 = int(b[rank]), int(b[rank + 1])
        v[t0:t1] = full[t0:t1]
        v[n + t0:n + t1] = full[n + t0:n + t1]
        SH.exchange_slices(v, b, rank)
        np.save(os.path.join(outdir, f"ex{rank}.npy"), v.numpy())
        np.save(os.path.join(outdir, "full.npy"), full.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bounds", [[0, 3, 7], [0, 5, 5, 9], [0, 1, 11, 12]])
def test_exchange_completes_every_rank(tmp_path, bounds):
    """exchange_slices (the all-gather of tabi_set_exchange's callback):
    uneven and empty shards, every rank ends with the whole vector."""
    import torch.multiprocessing as mp

    world = len(bounds) - 1
    mp.start_processes(_exchange_rank, args=(world, _free_port(), str(tmp_path), bounds),
                       nprocs=world, join=True, start_method="spawn")
    full = np.load(tmp_path / "full.npy")
    for r in range(world):
        np.testing.assert_array_equal(np.load(tmp_path / f"ex{r}.npy"), full)
