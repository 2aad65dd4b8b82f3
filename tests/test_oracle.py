"""The CPU oracle (oracle/tabi_oracle.c) against known answers.

The reference has no tests and no stored outputs, and no Fortran compiler is
available, so the oracle cannot be compared with the reference binary; it is
pinned instead to (a) the analytic Kirkwood/Born solvation energy, (b) an
FP64 O(N^2) direct sum, (c) LAPACK (numpy) for the restated DGETRF/DGETRS, and
(d) the committed golden fixtures of tests/golden (its own earlier output).
"""
import os

import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, born_case

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def born_exact(a=2.0, q=1.0):
    kap = O.kappa(BULK, EPS1)
    return 0.5 * 332.0716 * q * q / a * (1.0 / (EPS1 * (1.0 + kap * a)) - 1.0 / EPS0)


def solve_born(level, L):
    c = born_case(level)
    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], EPS0)
    T = O.Tree(xyz, tq, ar, b, 3, L, 0.8)
    kap = O.kappa(BULK, EPS1)
    res = T.dgmres(kap, EPS1 / EPS0, T.bvct, iprcd=1, tol=1e-4, nthreads=4)
    se, ce = T.energy(c["chrpos"], c["atmchr"], kap, EPS1 / EPS0, EPS0, res["x"], nthreads=4)
    return T, res, se


def test_kappa_real4_literal():
    # main.f90:62: 8.430325455 is a REAL*4 literal
    assert O.kappa(0.15, 80.0) == pytest.approx(0.12572533685666004, rel=0, abs=1e-17)
    assert abs(O.kappa(0.15, 80.0) - np.sqrt(8.430325455 * 0.15 / 80.0)) > 1e-10


def test_born_analytic():
    exact = born_exact()
    assert exact == pytest.approx(-82.18868, abs=1e-4)
    prev = None
    for level, L in ((2, 100), (3, 100)):
        _, res, se = solve_born(level, L)
        assert res["ierr"] == 0
        err = abs(se - exact) / abs(exact)
        # centroid collocation: error shrinks with refinement (~3.3% at 320, ~1.8% at 1280)
        assert err < (0.05 if level == 2 else 0.025), (level, se, exact)
        if prev is not None:
            assert err < prev
        prev = err


def test_tree_vs_direct():
    c = born_case(3)
    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], EPS0)
    T = O.Tree(xyz, tq, ar, b, 3, 100, 0.8)
    kap = O.kappa(BULK, EPS1)
    x = np.random.default_rng(0).normal(size=2 * T.n)
    yt = T.matvec(kap, EPS1, x, nthreads=4)
    yd = O.matvec_direct(T.xyz, T.tq, T.area, kap, EPS1, x, nthreads=4)
    rel = np.linalg.norm(yt - yd) / np.linalg.norm(yd)
    assert 1e-6 < rel < 1e-2  # treecode approximation error at order 3, theta 0.8
    # a MAC that accepts nothing gives the direct sum up to rounding
    T2 = O.Tree(xyz, tq, ar, b, 3, 100, 1e-9)
    y2 = T2.matvec(kap, EPS1, x, nthreads=4)
    # tree order differs from original order only by the permutation
    y2o = np.empty_like(y2)
    n = T2.n
    y2o[T2.orderarr - 1] = y2[:n]
    y2o[n + T2.orderarr - 1] = y2[n:]
    ydo = O.matvec_direct(xyz, tq, ar, kap, EPS1,
                          np.concatenate([x[:n], x[n:]]), nthreads=4)
    xo = np.empty_like(x)
    xo[T2.orderarr - 1] = x[:n]
    xo[n + T2.orderarr - 1] = x[n:]
    ydo = O.matvec_direct(xyz, tq, ar, kap, EPS1, xo, nthreads=4)
    assert np.linalg.norm(y2o - ydo) / np.linalg.norm(ydo) < 1e-13


def test_tree_partition_invariants():
    c = born_case(4)
    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], EPS0)
    T = O.Tree(xyz, tq, ar, b, 3, 500, 0.8)
    nd = T.nodes()
    assert sorted(T.orderarr) == list(range(1, T.n + 1))
    num = nd["iend"] - nd["ibeg"] + 1
    assert num[0] == T.n
    leaves = nd["nchild"] == 0
    assert num[leaves].sum() == T.n and leaves.sum() == T.nleaf
    assert (num[leaves] <= 500).all() and (num[~leaves] > 500).all()
    # every face lies in its leaf's box (radius = half diagonal)
    pts = T.xyz
    for ib, ie, g, nc in zip(nd["ibeg"], nd["iend"], nd["geo"], nd["nchild"]):
        d = np.linalg.norm(pts[ib - 1: ie] - g[:3], axis=1)
        assert (d <= g[3] * (1 + 1e-12)).all()


def test_dgetrf_dgetrs_vs_lapack():
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 17, 64):
        a = rng.normal(size=(n, n)) + np.eye(n) * 0.1
        lu, piv, info = O.dgetrf(a)
        assert info == 0
        b = rng.normal(size=n)
        x = O.dgetrs(lu, piv, n, b)
        np.testing.assert_allclose(a @ x, b, rtol=1e-10, atol=1e-10)
        import scipy.linalg as sl

        lu2, piv2 = sl.lu_factor(a)
        assert np.array_equal(piv + 0, piv2 + 1)  # same partial-pivot choices
    # exact zero column: info reported, no crash
    a = np.eye(3)
    a[:, 1] = 0.0
    _, _, info = O.dgetrf(a)
    assert info == 2


def test_surface_area_filter():
    c = born_case(2)
    nv = c["nvert"].copy()
    # duplicate face (same centroid within the 10-face window) and a degenerate face
    extra = np.array([nv[5], [1, 1, 2]], dtype=np.int32)
    nv2 = np.concatenate([nv[:6], extra, nv[6:]])
    kept, s_area = O.surface_area(c["sptpos"], nv2)
    assert len(kept) == len(nv)
    assert np.array_equal(kept, nv)


def test_golden_born():
    g = np.load(os.path.join(GOLDEN, "born_l3.npz"))
    T, res, se = solve_born(3, 100)
    assert res["iter"] == int(g["iter"])
    np.testing.assert_allclose(res["x"], g["x"], rtol=1e-10, atol=1e-14)
    assert se == pytest.approx(float(g["soleng"]), rel=1e-12)
    np.testing.assert_array_equal(T.orderarr, g["orderarr"])


def test_gmres_settings_fail_modes():
    c = born_case(2)
    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], EPS0)
    T = O.Tree(xyz, tq, ar, b, 3, 100, 0.8)
    kap = O.kappa(BULK, EPS1)
    # a one-cycle budget at an unreachable tolerance ends with IERR = 1
    res = T.dgmres(kap, EPS1, T.bvct, tol=1e-30, maxl=2, nrmax=-1, nthreads=2)
    assert res["ierr"] in (1, 2)
    assert res["iter"] <= 2
