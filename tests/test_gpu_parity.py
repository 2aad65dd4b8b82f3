"""GPU path (libtabi_gpu.so through the C ABI) against the CPU oracle.

Parity bars: tree node sets identical; matvec relative L2 <= 1e-10 (the bar
of the reference path is 1e-6, the two sides differ only in rounding);
preconditioner apply relative L2 <= 1e-10; GMRES iteration count equal and
solvation energy relative difference <= 1e-8 (bar 1e-4).
"""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, born_case, molecule_case

pytestmark = pytest.mark.gpu

MATVEC_TOL = 1e-10
ENERGY_TOL = 1e-8


def _setup(case, order=3, maxparnode=500, theta=0.8, iprcd=1, flags=0):
    import oracle as O
    import tabipb

    kap = O.kappa(BULK, EPS1)
    s = tabipb.TabiSolver(order=order, maxparnode=maxparnode, theta=theta, kappa=kap,
                          eps0=EPS0, eps1=EPS1, iprcd=iprcd, flags=flags)
    xyz, tq, ar, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                   case["chrpos"], case["atmchr"])
    oxyz, otq, oar, ob = O.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                       case["chrpos"], case["atmchr"], EPS0)
    T = O.Tree(oxyz, otq, oar, ob, order, maxparnode, theta)
    s.build_tree()
    return s, T, kap, (xyz, tq, ar, b), (oxyz, otq, oar, ob)


def _to_tree(v, orderarr, n):
    o = orderarr - 1
    return np.concatenate([v[:n][o], v[n:][o]])


def _from_tree(v, orderarr, n):
    o = orderarr - 1
    out = np.empty_like(v)
    out[o] = v[:n]
    out[n + o] = v[n:]
    return out


CASES = {
    "born_l3_L100": (lambda: born_case(3), dict(maxparnode=100)),
    "born_l4_L500": (lambda: born_case(4), dict(maxparnode=500)),
    "mol60_L200": (lambda: molecule_case(60, 6.0, 2.0, seed=1), dict(maxparnode=200)),
    "mol60_p5_L150": (lambda: molecule_case(60, 6.0, 2.0, seed=2), dict(maxparnode=150, order=5,
                                                                         theta=0.7)),
    # the large configuration's order and MAC, and the highest generated order
    "mol60_p6_L100": (lambda: molecule_case(60, 6.0, 2.0, seed=4), dict(maxparnode=100, order=6,
                                                                         theta=0.7)),
    "born_l3_p8_L100": (lambda: born_case(3), dict(maxparnode=100, order=8, theta=0.6)),
    # MSOLVEprec (main.f90:532-542): diagonal scaling instead of the leaf blocks
    "mol60_L200_iprcd0": (lambda: molecule_case(60, 6.0, 2.0, seed=1), dict(maxparnode=200,
                                                                             iprcd=0)),
    # two of its 75 leaf blocks need row interchanges (DGETRF2 swaps 4 rows):
    # they fail the no-interchange check and are factored with pivoting
    "mol60_d3_L100": (lambda: molecule_case(60, 6.0, 3.0, seed=3), dict(maxparnode=100)),
    # every leaf with partial pivoting (TABI_FLAG_PIVOTED_LU)
    "mol60_L200_pivoted": (lambda: molecule_case(60, 6.0, 2.0, seed=1), dict(maxparnode=200,
                                                                              flags=1)),
}

# leaf blocks that need partial pivoting, per case (the others take the
# certified unpivoted factorisation)
PIVOTED = {"mol60_d3_L100": 2, "mol60_L200_pivoted": 54}


@pytest.fixture(scope="module", params=list(CASES))
def setup(request, gpu_lib):
    mk, kw = CASES[request.param]
    case = mk()
    s, T, kap, g, o = _setup(case, **kw)
    T.iprcd = kw.get("iprcd", 1)
    yield request.param, case, s, T, kap, g, o
    s.close()


def test_form_matrix(setup):
    name, case, s, T, kap, g, o = setup
    xyz, tq, ar, b = g
    oxyz, otq, oar, ob = o
    # centroids are built without contraction: bit-identical (the tree depends on them)
    assert np.array_equal(xyz, O_orig(case)[0])
    np.testing.assert_allclose(tq, O_orig(case)[1], rtol=0, atol=1e-15)
    np.testing.assert_allclose(ar, O_orig(case)[2], rtol=1e-15, atol=0)
    rel = np.linalg.norm(b - O_orig(case)[3]) / np.linalg.norm(O_orig(case)[3])
    assert rel < 1e-12, rel


_orig_cache = {}


def O_orig(case):
    import oracle as O

    key = id(case)
    if key not in _orig_cache:
        _orig_cache[key] = O.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                         case["chrpos"], case["atmchr"], EPS0)
    return _orig_cache[key]


def test_tree_nodes(setup):
    name, case, s, T, kap, g, o = setup
    gn = s.tree_nodes()
    on = T.nodes()
    assert s.nleaf == T.nleaf
    assert len(gn["ibeg"]) == len(on["ibeg"])
    assert np.array_equal(gn["ibeg"], on["ibeg"])
    assert np.array_equal(gn["numpar"], on["iend"] - on["ibeg"] + 1)
    assert np.array_equal(gn["level"], on["level"])
    assert np.array_equal(gn["nchild"], on["nchild"])
    big = gn["numpar"] >= 2  # 1-face nodes keep the split box in the reference; never used
    assert np.array_equal(gn["geo"][big], on["geo"][big])
    # same face sets per node (the order inside a node may differ: the
    # reference's PARTITION is not stable)
    go, oo = s.orderarr, T.orderarr
    for ib, npar in zip(gn["ibeg"], gn["numpar"]):
        a = np.sort(go[ib - 1: ib - 1 + npar])
        b = np.sort(oo[ib - 1: ib - 1 + npar])
        assert np.array_equal(a, b)


def test_matvec(setup):
    name, case, s, T, kap, g, o = setup
    n = s.nface
    rng = np.random.default_rng(7)
    x = rng.normal(size=2 * n)
    yg = _from_tree(s.matvec(_to_tree(x, s.orderarr, n)), s.orderarr, n)
    yo, cnt = T.matvec(kap, EPS1 / EPS0, _to_tree(x, T.orderarr, n), nthreads=8,
                       return_counts=True)
    yo = _from_tree(yo, T.orderarr, n)
    rel = np.linalg.norm(yg - yo) / np.linalg.norm(yo)
    assert rel < MATVEC_TOL, rel
    near, far = s.counts()
    assert near == cnt[0] and far == cnt[1]


def test_matvec_zero_shortcut(setup):
    name, case, s, T, kap, g, o = setup
    x = np.zeros(2 * s.nface)
    x[3] = 1e-12  # sum|x| < 1e-10: MATVECmain returns y = x
    assert np.array_equal(s.matvec(x), x)


def test_pivoted_leaves(setup):
    name, case, s, T, kap, g, o = setup
    if T.iprcd != 1:
        return
    assert s.pivoted_leaves() == PIVOTED.get(name, 0)


def test_msolve(setup):
    name, case, s, T, kap, g, o = setup
    n = s.nface
    rng = np.random.default_rng(11)
    r = rng.normal(size=2 * n)
    zg = _from_tree(s.msolve(_to_tree(r, s.orderarr, n)), s.orderarr, n)
    zo = _from_tree(T.msolve(kap, EPS1 / EPS0, _to_tree(r, T.orderarr, n), iprcd=T.iprcd,
                             nthreads=8), T.orderarr, n)
    rel = np.linalg.norm(zg - zo) / np.linalg.norm(zo)
    assert rel < MATVEC_TOL, rel


def test_solve_and_energy(setup):
    name, case, s, T, kap, g, o = setup
    n = s.nface
    _, _, _, b = g
    bt = _to_tree(b, s.orderarr, n)
    res = s.dgmres(bt)
    ores = T.dgmres(kap, EPS1 / EPS0, T.bvct, iprcd=T.iprcd, tol=1e-4, nthreads=8)
    assert res["ierr"] == ores["ierr"] == 0
    assert res["iter"] == ores["iter"]
    np.testing.assert_allclose(res["err_hist"], ores["err_hist"], rtol=1e-8)
    xg = _from_tree(res["x"], s.orderarr, n)
    xo = _from_tree(ores["x"], T.orderarr, n)
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-9
    se, ce = s.energy(case["chrpos"], case["atmchr"], res["x"])
    ose, oce = T.energy(case["chrpos"], case["atmchr"], kap, EPS1 / EPS0, EPS0, ores["x"],
                        nthreads=8)
    assert abs(se - ose) <= ENERGY_TOL * abs(ose)
    assert abs(ce - oce) <= 1e-12 * max(abs(oce), 1e-30)


def test_output_potential(setup):
    """main.f90:226-326: vertex potentials and the scaled face values, GPU vs
    oracle (same solution vector, un-permuted by orderarr)."""
    import oracle as O

    name, case, s, T, kap, g, o = setup
    xyz, tq, ar, b = g
    n = len(ar)
    rng = np.random.default_rng(4)
    x_tree = rng.standard_normal(2 * n)
    xo_gpu, vert_gpu = s.output_potential(case["sptpos"], case["nvert"], x_tree)
    x_orig = _from_tree(x_tree, s.orderarr, n)
    vert_ref, xs_ref = O.output_potential(case["sptpos"], case["nvert"], xyz, x_orig)
    np.testing.assert_array_equal(xo_gpu, xs_ref)
    used = np.isfinite(vert_ref[:, 0])
    np.testing.assert_array_equal(np.isfinite(vert_gpu[:, 0]), used)
    np.testing.assert_allclose(vert_gpu[used], vert_ref[used], rtol=1e-14, atol=0)


def test_direct_sum_targets(setup):
    """tabi_direct_targets (FP64 direct sum, the accuracy reference of the
    treecode) against the oracle's direct sum, at sampled targets."""
    import oracle as O

    name, case, s, T, kap, g, o = setup
    xyz, tq, ar, b = g
    n = len(ar)
    rng = np.random.default_rng(6)
    x_tree = rng.standard_normal(2 * n)
    tg = np.sort(rng.choice(n, min(n, 300), replace=False)).astype(np.int32)
    y1, y2 = s.direct_targets(tg, x_tree)
    # the oracle on the same (tree) face order
    txyz, ttq, tar, _ = s.permute(xyz, tq, ar, b)
    yd = O.matvec_direct(txyz, ttq, tar, kap, EPS1 / EPS0, x_tree)
    np.testing.assert_allclose(y1, yd[tg], rtol=1e-12, atol=1e-12 * np.abs(yd).max())
    np.testing.assert_allclose(y2, yd[n + tg], rtol=1e-12, atol=1e-12 * np.abs(yd).max())
