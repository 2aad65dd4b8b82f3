"""Batched solves (tabi_batch_run_dev): every molecule's result equals the
single-molecule path (tabi_run_dev) bit for bit -- the workers only overlap
independent solves -- with per-molecule leaf sizes honoured, the warm start
usable inside the batch, and errors reported."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mols(gpu_lib):
    from tabipb import batch as B

    sizes = [150, 400, 90, 260, 600, 200]
    return [B.make_molecule(n, seed=50 + k, density=3.0) for k, n in enumerate(sizes)]


def _params(**kw):
    import tabipb

    return tabipb.default_params(**kw)


def _single(m, params, leaf=None, ws=None):
    import tabipb

    p = {f: getattr(params, f) for f, _ in params._fields_}
    if leaf:
        p["maxparnode"] = leaf
    with tabipb.TabiSolver(**p) as s:
        if ws is not None:
            s.set_warmstart(ws)
        return s.run_dev(m["nspt"], m["sptpos"].data_ptr(), m["sptnrm"].data_ptr(), m["nface"],
                         m["nvert"].data_ptr(), m["nchr"], m["chrpos"].data_ptr(),
                         m["atmchr"].data_ptr())


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_single_solves(mols, precision):
    from tabipb import batch as B

    prm = _params(precision=precision, maxparnode=300)
    table = {0: 200}
    st, wall = B.run_batch(mols, prm, nworkers=3, table=table)
    for k, m in enumerate(mols):
        leaf = table.get(B.size_class(m["nface"]), 0) or prm.maxparnode
        r = _single(m, prm, leaf=leaf)
        assert st[k, 11] == leaf
        assert st[k, 0] == r["iter"] and st[k, 2] == r["ierr"] == 0
        assert st[k, 3] == r["soleng"] and st[k, 4] == r["couleng"], (k, st[k, 3], r["soleng"])
        assert st[k, 7] == r["nleaf"]
    assert set(st[:, 10]) <= {0, 1, 2}
    assert np.all(st[:, 8] > 0) and np.all(st[:, 9] <= wall * 1e3 + 1)


def test_batch_with_warm_start(mols):
    from tabipb import batch as B
    from tabipb.warmstart import WarmStart

    ws = WarmStart(hidden=64, layers=2, seed=3)
    prm = _params(precision=1, tol=1e-6)
    st, _ = B.run_batch(mols[:3], prm, ws=ws, nworkers=2)
    for k, m in enumerate(mols[:3]):
        r = _single(m, prm, ws=ws)
        assert st[k, 0] == r["iter"] and st[k, 3] == r["soleng"]


def test_batch_reports_errors(mols):
    import tabipb
    from tabipb import batch as B
    from tabipb._lib import MolDev

    L = tabipb.load()
    bad = (MolDev * 2)()
    bad[0] = B._moldev(mols[0])
    bad[1] = B._moldev(mols[1])
    bad[1].nface = 0
    st = np.zeros((2, 12))
    rc = L.tabi_batch_run_dev(C.byref(_params()), 2, bad, None, 2,
                              st.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == -1
    assert b"positive" in L.tabi_last_error(None)


def test_autotune_picks_a_candidate(mols):
    from tabipb import batch as B

    table, timings = B.autotune([mols[4]], _params(), candidates=(150, 300), repeats=1)
    c = B.size_class(mols[4]["nface"])
    assert table[c] in (150, 300)
    assert timings[(c, table[c])] == min(timings[(c, 150)], timings[(c, 300)])


def test_worker_tuner_picks_the_fastest_count(mols):
    from tabipb import batch as B

    prm = _params(precision=1, maxparnode=300)
    nw, timings = B.tune_workers(mols, prm, None, candidates=(1, 2), repeats=1)
    assert set(timings) == {1, 2} and nw in (1, 2)
    assert timings[nw] == min(timings.values())
    # the chosen count changes nothing but the overlap
    a, _ = B.run_batch(mols, prm, nworkers=1)
    b, _ = B.run_batch(mols, prm, nworkers=nw)
    assert np.array_equal(a[:, 3], b[:, 3]) and np.array_equal(a[:, 0], b[:, 0])
