"""Failure paths of the device solve, all made on the host side (no GPU
fault, no hang): non-finite right-hand sides and initial guesses, the GMRES
iteration cap, and a leaf block that cannot be factored.

The reference has no error handling on these paths: DGMRES iterates on NaNs
until its iteration limit, and LEAFMATVECpara ignores DGETRF's info
(treecode3d_pb.f:1530).  The library refuses non-finite inputs with
TABI_ERR_ARG, returns DGMRES's own IERR for the iteration cap
(dgmres_dep.f:819-851), and reports a leaf block with a zero or non-finite
pivot as TABI_ERR_SINGULAR; after each error the handle still gives the
fresh handle's results.
"""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, born_case

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_SINGULAR = -1, -5


def _solver(**kw):
    import oracle as O
    import tabipb

    prm = dict(order=3, maxparnode=100, theta=0.8, kappa=O.kappa(BULK, EPS1), eps0=EPS0,
               eps1=EPS1)
    prm.update(kw)
    return tabipb.TabiSolver(**prm)


def _code(fn, *a, **kw):
    from tabipb._lib import TabiError

    with pytest.raises(TabiError) as e:
        fn(*a, **kw)
    return e.value.code, str(e.value)


def _loaded(s, case):
    xyz, tq, ar, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                   case["chrpos"], case["atmchr"])
    s.build_tree()
    return s.permute(bvct=b)[3]


@pytest.mark.parametrize("precision", [0, 1])
def test_nonfinite_rhs_and_initial_guess(gpu_lib, precision):
    case = born_case(3)
    with _solver(precision=precision) as s:
        bt = _loaded(s, case)
        ref = s.dgmres(bt)
        bad = bt.copy()
        bad[7] = np.nan
        code, msg = _code(s.dgmres, bad)
        assert code == ERR_ARG and "not finite" in msg
        bad[7] = np.inf
        assert _code(s.dgmres, bad)[0] == ERR_ARG
        x0 = np.zeros_like(bt)
        x0[3] = np.nan
        code, msg = _code(s.dgmres, bt, x0=x0)
        assert code == ERR_ARG and "x0" in msg
        # the handle is unchanged by the refused calls
        again = s.dgmres(bt)
        assert again["iter"] == ref["iter"] and np.array_equal(again["x"], ref["x"])


def test_iteration_cap_matches_oracle(gpu_lib):
    """MAXL 2 and NRMAX -1 (no restart) at a tolerance two Krylov steps cannot
    meet: DGMRES stops with IERR 1 (dgmres_dep.f:819-827); iterations and
    error estimates equal the oracle's."""
    import oracle as O

    case = born_case(3)
    kap = O.kappa(BULK, EPS1)
    with _solver(maxl=2, nrmax=-1, tol=1e-10) as s:
        bt = _loaded(s, case)
        res = s.dgmres(bt)
    xyz, tq, ar, b = O.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                   case["chrpos"], case["atmchr"], EPS0)
    T = O.Tree(xyz, tq, ar, b, 3, 100, 0.8)
    ores = T.dgmres(kap, EPS1 / EPS0, T.bvct, iprcd=1, tol=1e-10, maxl=2, nrmax=-1, nthreads=8)
    assert res["ierr"] == ores["ierr"] == 1
    assert res["iter"] == ores["iter"] == 2
    np.testing.assert_allclose(res["err_hist"], ores["err_hist"], rtol=1e-8)
    assert res["err"] > 1e-10
    # restarts allowed: the same settings then converge
    with _solver(maxl=2, nrmax=10, tol=1e-4) as s:
        bt = _loaded(s, case)
        assert s.dgmres(bt)["ierr"] == 0


def test_coincident_faces_make_a_leaf_block_singular(gpu_lib):
    """Two faces with the same centroid make the leaf block's kernel values
    non-finite (rho = 0): tabi_build_tree reports TABI_ERR_SINGULAR instead of
    factoring NaNs, and the handle takes a valid surface afterwards."""
    import oracle as O

    case = born_case(2)
    xyz, tq, ar, b = O.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                   case["chrpos"], case["atmchr"], EPS0)
    dup = lambda a: np.concatenate([a, a[5:6]])
    with _solver() as s:
        s.set_surface(dup(xyz), dup(tq), dup(ar))
        code, msg = _code(s.build_tree)
        assert code == ERR_SINGULAR and "non-finite" in msg
        # no tree is left behind: operators refuse to run
        assert _code(s.matvec, np.ones(2 * s.nface))[0] == -4
        s.set_surface(xyz, tq, ar)
        s.build_tree()
        x = np.random.default_rng(2).normal(size=2 * s.nface)
        y = s.matvec(x)
    with _solver() as s:
        s.set_surface(xyz, tq, ar)
        s.build_tree()
        assert np.array_equal(y, s.matvec(x))
