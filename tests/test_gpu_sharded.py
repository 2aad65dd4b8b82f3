"""Shards of the GPU operator (tabi_set_target_range): two handles restricted
to the two halves of the targets (leaf-aligned) assemble the full matvec and
preconditioner apply bit for bit -- each target's interactions are computed
and summed exactly as in the unsharded handle -- and GMRES across the shards
(tabipb.sharded.dgmres) matches the library's own solve.  Those shards run
one after the other in one process on the one GPU.  The library's own solve
across two processes (tabi_set_exchange with a gloo all-gather) runs as two
spawned processes on the one GPU that wait on each other on the host only;
the exchange itself is covered on the host by test_sharded_cpu.py."""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, molecule_case

pytestmark = pytest.mark.gpu


def _handles(case, nshards, **kw):
    import tabipb
    from tabipb.sharded import shard_bounds

    kap = tabipb.kappa(BULK, EPS1)
    hs = []
    for k in range(nshards + 1):  # the last one unrestricted
        s = tabipb.TabiSolver(kappa=kap, eps0=EPS0, eps1=EPS1, **kw)
        xyz, tq, ar, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                       case["chrpos"], case["atmchr"])
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b)
        hs.append(s)
    st, sz = hs[0].leaves()
    bounds = shard_bounds(st, sz, nshards)
    for k in range(nshards):
        hs[k].set_target_range(bounds[k], bounds[k + 1])
    return hs, bounds, bt


def _assemble(hs, bounds, fn, v):
    n = bounds[-1]
    out = np.empty_like(v)
    for k in range(len(bounds) - 1):
        t0, t1 = bounds[k], bounds[k + 1]
        part = getattr(hs[k], fn)(v)
        out[t0:t1] = part[t0:t1]
        out[n + t0:n + t1] = part[n + t0:n + t1]
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_shards_assemble_the_operator(gpu_lib, precision):
    case = molecule_case(200, 9.0, 4.0, seed=4)
    hs, bounds, bt = _handles(case, 3, maxparnode=300, precision=precision)
    try:
        full = hs[-1]
        x = np.random.default_rng(2).standard_normal(bt.size)
        np.testing.assert_array_equal(_assemble(hs, bounds, "matvec", x), full.matvec(x))
        np.testing.assert_array_equal(_assemble(hs, bounds, "msolve", x), full.msolve(x))
    finally:
        for h in hs:
            h.close()


def test_gmres_across_shards_matches_the_solve(gpu_lib):
    import tabipb
    from tabipb import sharded as SH

    case = molecule_case(200, 9.0, 4.0, seed=4)
    hs, bounds, bt = _handles(case, 2, maxparnode=300)
    try:
        full = hs[-1]
        res = SH.dgmres(lambda v: _assemble(hs, bounds, "matvec", v),
                        lambda v: _assemble(hs, bounds, "msolve", v), bt, tol=1e-4)
        ref = full.dgmres(bt)
        assert res["ierr"] == 0 == ref["ierr"]
        assert res["iter"] == ref["iter"], (res["iter"], ref["iter"])
        assert np.linalg.norm(res["x"] - ref["x"]) <= 1e-9 * np.linalg.norm(ref["x"])
        # a restricted handle computes one shard only: its own solve is refused
        with pytest.raises(tabipb.TabiError):
            hs[0].dgmres(bt)
    finally:
        for h in hs:
            h.close()


def test_target_range_must_be_leaf_aligned(gpu_lib):
    import tabipb

    case = molecule_case(60, 6.0, 2.0, seed=1)
    s = tabipb.TabiSolver(kappa=tabipb.kappa(BULK, EPS1), eps0=EPS0, eps1=EPS1, maxparnode=200)
    s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"], case["atmchr"])
    s.build_tree()
    st, sz = s.leaves()
    with pytest.raises(tabipb.TabiError):
        s.set_target_range(0, int(st[1]) + 1)
    s.set_target_range(0, int(st[1]))
    s.set_target_range(0, int(st[-1] + sz[-1]))  # the whole range lifts it
    s.close()


def _solve_rank(rank, world, port, outdir, precision):
    import os
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path[:0] = [here, os.path.join(root, "tabi-pb_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    import tabipb
    from tabipb import sharded as SH

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        case = molecule_case(200, 9.0, 4.0, seed=4)
        s = tabipb.TabiSolver(kappa=tabipb.kappa(BULK, EPS1), eps0=EPS0, eps1=EPS1,
                              maxparnode=300, precision=precision)
        _, _, _, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                   case["chrpos"], case["atmchr"])
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b)
        st, sz = s.leaves()
        bounds = SH.shard_bounds(st, sz, world)
        res = SH.sharded_solve(s, bt, bounds, rank, device="cuda:0")
        np.savez(os.path.join(outdir, f"solve{rank}.npz"), x=res["x"], iter=res["iter"],
                 err=res["err"], ierr=res["ierr"], hist=res["err_hist"], bounds=bounds,
                 exchanges=res["exchanges"])
        s.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", [0, 1])
def test_library_solve_across_two_processes(gpu_lib, tmp_path, precision):
    """Two processes on the one GPU, each a handle restricted to its shard,
    run the library's own solve (tabi_solve) with the exchange hook doing a
    gloo all-gather of every operator and preconditioner result: both ranks
    take the same steps and end with the unsharded solve's solution, bit for
    bit (the assembled vectors are the unsharded ones, see above).  The
    processes wait on each other on the host only (gloo), never on the GPU."""
    import socket

    import torch.multiprocessing as mp

    import tabipb

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    mp.start_processes(_solve_rank, args=(2, port, str(tmp_path), precision), nprocs=2,
                       join=True, start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"solve{k}.npz") for k in (0, 1))
    case = molecule_case(200, 9.0, 4.0, seed=4)
    s = tabipb.TabiSolver(kappa=tabipb.kappa(BULK, EPS1), eps0=EPS0, eps1=EPS1, maxparnode=300,
                          precision=precision)
    try:
        _, _, _, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                   case["chrpos"], case["atmchr"])
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b)
        ref = s.dgmres(bt)
    finally:
        s.close()
    b = r0["bounds"]
    assert 0 < b[1] < b[-1]
    assert int(r0["exchanges"]) > 2 * int(r0["iter"])
    for r in (r0, r1):
        assert int(r["ierr"]) == 0 == ref["ierr"]
        assert int(r["iter"]) == ref["iter"]
        np.testing.assert_array_equal(r["x"], ref["x"])
        np.testing.assert_array_equal(r["hist"], ref["err_hist"])
