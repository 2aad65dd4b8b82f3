"""The leaf-block LU's paths on single large blocks: the certified
unpivoted factorisation (the default), and, with TABI_FLAG_PIVOTED_LU, the
pivoted kernels' three panel paths, chosen by the rows a panel has left
(block order m = 2 x leaf faces): the register-resident panel for up to 1,024
rows, the shared-memory panel above that (blocks up to 1,536), and the
global-memory LU for larger blocks.  Each case is one leaf, so one
preconditioner apply (LEAFMATVECpara, treecode3d_pb.f:1393-1542: DGETRF +
DGETRS of the whole block) is checked against the oracle's."""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, born_case, molecule_case

pytestmark = pytest.mark.gpu

TOL = 1e-10

CASES = {
    # 666 faces in one leaf: m = 1332, shared-memory panels first, then the
    # register panels of 512 x 2, 512 x 1 and 256 x 1 rows
    "one_leaf_m1332": (lambda: molecule_case(10, 3.0, 2.0, seed=3), 700, 1332),
    # 1,280 faces in one leaf: m = 2560, global-memory LU
    "one_leaf_m2560": (lambda: born_case(3), 1280, 2560),
}


@pytest.mark.parametrize("flags", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_msolve_one_large_block(name, flags, gpu_lib):
    import oracle as O
    import tabipb

    mk, leaf, m = CASES[name]
    case = mk()
    kap = O.kappa(BULK, EPS1)
    with tabipb.TabiSolver(order=3, maxparnode=leaf, theta=0.8, kappa=kap, eps0=EPS0,
                           eps1=EPS1, iprcd=1, flags=flags) as s:
        s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"], case["chrpos"],
                      case["atmchr"])
        s.build_tree()
        _, sizes = s.leaves()
        assert sizes.size == 1 and 2 * int(sizes[0]) == m
        assert s.pivoted_leaves() == flags
        oxyz, otq, oar, ob = O.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                           case["chrpos"], case["atmchr"], EPS0)
        T = O.Tree(oxyz, otq, oar, ob, 3, leaf, 0.8)
        n = s.nface
        r = np.random.default_rng(5).normal(size=2 * n)
        # both solvers in original face order
        og, oo = s.orderarr - 1, T.orderarr - 1
        rg = np.concatenate([r[:n][og], r[n:][og]])
        ro = np.concatenate([r[:n][oo], r[n:][oo]])
        zg_t = s.msolve(rg)
        zo_t = T.msolve(kap, EPS1 / EPS0, ro, nthreads=8)
        zg = np.empty(2 * n)
        zo = np.empty(2 * n)
        zg[og], zg[n + og] = zg_t[:n], zg_t[n:]
        zo[oo], zo[n + oo] = zo_t[:n], zo_t[n:]
        rel = np.linalg.norm(zg - zo) / np.linalg.norm(zo)
        assert rel < TOL, rel
        # twice in a row: the factors are kept, the apply is repeatable
        assert np.array_equal(s.msolve(rg), zg_t)
