"""Error reporting through the C ABI.  Calls out of order, empty surfaces,
face lists that name vertices outside 1..nspt and vectors of the wrong length
come back as a negative TABI_ERR_* code with a message (the reference would
STOP or run on with garbage), and the handle stays usable: a correct sequence
afterwards gives the same result as on a fresh handle."""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, born_case

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_STATE = -1, -4


def _solver():
    import oracle as O
    import tabipb

    return tabipb.TabiSolver(order=3, maxparnode=100, theta=0.8, kappa=O.kappa(BULK, EPS1),
                             eps0=EPS0, eps1=EPS1)


def _code(fn, *a):
    from tabipb._lib import TabiError

    with pytest.raises(TabiError) as e:
        fn(*a)
    assert str(e.value)  # a message comes with the code
    return e.value.code


def _matvec_of(case, x=None):
    with _solver() as s:
        s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                      case["atmchr"])
        s.build_tree()
        if x is None:
            x = np.random.default_rng(3).normal(size=2 * s.nface)
        return s.matvec(x), x


def test_calls_out_of_order(gpu_lib):
    with _solver() as s:
        assert _code(s.build_tree) == ERR_STATE                    # no surface yet
        assert _code(s.matvec, np.ones(8)) == ERR_STATE             # no tree yet
        assert _code(s.msolve, np.ones(8)) == ERR_STATE
        case = born_case(2)
        s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                      case["atmchr"])
        assert _code(s.matvec, np.ones(2 * s.nface)) == ERR_STATE   # surface, no tree
        s.build_tree()
        assert _code(s.build_tree) == ERR_STATE                    # tree already built


def test_bad_surfaces_and_vectors(gpu_lib):
    case = born_case(2)
    with _solver() as s:
        nv = case["nvert"].copy()
        nv[0, 0] = 0                                                # indices are 1-based
        assert _code(s.form_matrix, case["sptpos"], case["sptnrm"], nv, case["chrpos"],
                     case["atmchr"]) == ERR_ARG
        nv = case["nvert"].copy()
        nv[-1, 2] = len(case["sptpos"]) + 1                         # past the last vertex
        assert _code(s.form_matrix, case["sptpos"], case["sptnrm"], nv, case["chrpos"],
                     case["atmchr"]) == ERR_ARG
        empty = np.zeros((0, 3), np.int32)                          # no faces
        assert _code(s.form_matrix, case["sptpos"], case["sptnrm"], empty, case["chrpos"],
                     case["atmchr"]) == ERR_ARG
        # the same handle then runs a correct sequence
        s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                      case["atmchr"])
        s.build_tree()
        n = s.nface
        assert _code(s.matvec, np.ones(2 * n + 2)) == ERR_ARG       # wrong length
        assert _code(s.msolve, np.ones(2 * n - 2)) == ERR_ARG
        assert _code(s.direct_targets, np.array([n]), np.ones(2 * n)) == ERR_ARG
        x = np.random.default_rng(3).normal(size=2 * n)
        y = s.matvec(x)
    # equal to a fresh handle's result on the same input
    y_fresh, _ = _matvec_of(case, x)
    assert np.all(np.isfinite(y))
    assert np.array_equal(y, y_fresh)


def test_caller_buffers(gpu_lib):
    """form_matrix and dgmres write into caller-owned arrays (page-locked ones,
    for instance) with results identical to the allocating calls; arrays of
    the wrong shape are refused before the library is called."""
    case = born_case(2)
    with _solver() as s:
        a = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                          case["atmchr"])
        n = s.nface
        out = (np.empty((n, 3)), np.empty((n, 3)), np.empty(n), np.empty(2 * n))
        b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                          case["atmchr"], out=out)
        assert all(np.array_equal(u, v) for u, v in zip(a, b))
        assert all(u is v for u, v in zip(b, out))
        with pytest.raises(ValueError):
            s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                          case["atmchr"], out=(out[0], out[1], out[2], np.empty(n)))
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b[3])
        r1 = s.dgmres(bt)
        x = np.full(2 * n, 7.0)
        r2 = s.dgmres(bt, out=x)
        assert r2["x"] is x and np.array_equal(r1["x"], x) and r1["iter"] == r2["iter"]
