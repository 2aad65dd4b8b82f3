"""Mixed precision (TABI_PREC_MIXED): FP32 treecode operator, FP64 refinement.

Bars: the FP32 operator agrees with the FP64 one to relative L2 <= 2e-5, far below the treecode's own truncation error at these
settings; the refined solve meets tol on the FP64 residual, which this test
recomputes with an FP64 handle; the solvation energy agrees with the FP64 solve
to <= 1e-4 relative (the bar of the mixed path), and with tol 1e-6 to <= 1e-6.
"""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, born_case, molecule_case

pytestmark = pytest.mark.gpu

OPERATOR_TOL = 2e-5


def _pair(case, tol=1e-4, **kw):
    import tabipb

    kap = tabipb.kappa(BULK, EPS1)
    out = []
    for prec in (tabipb.PREC_FP64, tabipb.PREC_MIXED):
        s = tabipb.TabiSolver(kappa=kap, eps0=EPS0, eps1=EPS1, tol=tol, precision=prec, **kw)
        xyz, tq, ar, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                       case["chrpos"], case["atmchr"])
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b)
        out.append((s, bt))
    return out


def _close(pairs):
    for s, _ in pairs:
        s.close()


def _fp64_measure(s64, b, x):
    """|M^-1 (b - A x)| / |M^-1 b| with the FP64 operator (DGMRES ITOL = 2)."""
    r = b - s64.matvec(x)
    return np.linalg.norm(s64.msolve(r)) / np.linalg.norm(s64.msolve(b))


CASES = {
    "mol60_L200": (lambda: molecule_case(60, 6.0, 2.0, seed=1), dict(maxparnode=200)),
    "mol400_L500": (lambda: molecule_case(400, 11.0, 6.0, seed=3), dict(maxparnode=500)),
    "mol200_p6_L300": (lambda: molecule_case(200, 9.0, 4.0, seed=4),
                       dict(maxparnode=300, order=6, theta=0.7)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_operator_close_to_fp64(name, gpu_lib):
    mk, kw = CASES[name]
    case = mk()
    pairs = _pair(case, **kw)
    try:
        (s64, bt), (s32, _) = pairs
        assert np.array_equal(s64.orderarr, s32.orderarr)
        rng = np.random.default_rng(11)
        for trial in range(2):
            x = rng.standard_normal(bt.size) if trial else bt.copy()
            y64 = s64.matvec(x)
            y32 = s32.matvec(x)
            rel = np.linalg.norm(y32 - y64) / np.linalg.norm(y64)
            assert rel <= OPERATOR_TOL, (name, trial, rel)
            # interaction part alone (y - pre * x), the part the FP32 arithmetic touches
            eps = EPS1 / EPS0
            n = bt.size // 2
            pre = np.concatenate([np.full(n, 0.5 * (1 + eps)), np.full(n, 0.5 * (1 + 1 / eps))])
            i64, i32 = pre * x - y64, pre * x - y32
            reli = np.linalg.norm(i32 - i64) / np.linalg.norm(i64)
            assert reli <= 10 * OPERATOR_TOL, (name, trial, reli)
    finally:
        _close(pairs)


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_solve_meets_tol_on_fp64_residual(name, gpu_lib):
    mk, kw = CASES[name]
    case = mk()
    pairs = _pair(case, **kw)
    try:
        (s64, bt), (s32, _) = pairs
        r64 = s64.dgmres(bt)
        r32 = s32.dgmres(bt)
        assert r64["ierr"] == 0 and r32["ierr"] == 0, (r64["ierr"], r32["ierr"])
        assert r32["err"] <= 1e-4
        meas = _fp64_measure(s64, bt, r32["x"])
        assert meas <= 1e-4 * (1 + 1e-9), meas
        assert abs(meas - r32["err"]) <= 1e-6 * max(meas, 1e-12) + 1e-12, (meas, r32["err"])
        e64, _ = s64.energy(case["chrpos"], case["atmchr"], r64["x"])
        e32, _ = s32.energy(case["chrpos"], case["atmchr"], r32["x"])
        assert abs(e32 - e64) <= 1e-4 * abs(e64), (e32, e64)
        # the refinement adds few iterations over the FP64 path
        assert r32["iter"] <= r64["iter"] + 4, (r32["iter"], r64["iter"])
    finally:
        _close(pairs)


def test_mixed_refines_to_1e6(gpu_lib):
    case = molecule_case(200, 9.0, 4.0, seed=4)
    pairs = _pair(case, tol=1e-6, maxparnode=300)
    try:
        (s64, bt), (s32, _) = pairs
        r64 = s64.dgmres(bt)
        r32 = s32.dgmres(bt)
        assert r64["ierr"] == 0 and r32["ierr"] == 0
        meas = _fp64_measure(s64, bt, r32["x"])
        assert meas <= 1e-6 * (1 + 1e-9), meas
        e64, _ = s64.energy(case["chrpos"], case["atmchr"], r64["x"])
        e32, _ = s32.energy(case["chrpos"], case["atmchr"], r32["x"])
        assert abs(e32 - e64) <= 1e-6 * abs(e64), (e32, e64)
        h = r32["err_hist"]
        assert h.size == r32["iter"] and np.all(np.isfinite(h))
    finally:
        _close(pairs)


def test_mixed_born_ion_kirkwood(gpu_lib):
    """Born ion: the mixed solve lands where the FP64 one does, near Kirkwood."""
    case = born_case(4)
    pairs = _pair(case, maxparnode=500)
    try:
        (s64, bt), (s32, _) = pairs
        r64, r32 = s64.dgmres(bt), s32.dgmres(bt)
        e64, _ = s64.energy(case["chrpos"], case["atmchr"], r64["x"])
        e32, _ = s32.energy(case["chrpos"], case["atmchr"], r32["x"])
        assert abs(e32 - e64) <= 1e-4 * abs(e64)
        kap = s64.params.kappa
        a = 2.0
        kirk = 0.5 * 332.0716 * (1.0 / (EPS1 * (1 + kap * a)) - 1.0 / EPS0) / a
        assert abs(e32 - kirk) <= 0.015 * abs(kirk), (e32, kirk)
    finally:
        _close(pairs)


def test_mixed_precision_rejects_unknown_mode(gpu_lib):
    import tabipb

    with pytest.raises(tabipb.TabiError):
        tabipb.TabiSolver(precision=7)
