"""GPU vs oracle at the benchmark's own sizes and on the reference's own
inputs (the oracle on all host threads).

* The benchmark molecule (2,000 atoms, 92,848 faces; order 3, MAC 0.8, leaf
  500, tol 1e-4): the whole solve -- node table and face sets, a full-size
  matvec and preconditioner apply, GMRES iterations and error history, the
  solution and the energies.
* The large configuration (20,000 atoms, 434,048 faces; order 6, MAC 0.7,
  leaf 400): the FP64 treecode matvec at 4,096 targets in 8 blocks spread
  over the tree order, against the oracle's target loop on the same input
  vector, and the FP32 (mixed-precision) operator at the same targets.
* src/test_proteins/1a63.pqr and 4mn3.pqr with the reference's own
  usrdata.in settings (den 5, order 3, leaf 100, MAC 0.8), through the host
  driver tabipb: iterations and energies equal the oracle's on the same
  surface (main.f90:136-159).
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

NT = os.cpu_count() or 1
BUILD = os.path.join(ROOT, "tabi-pb_b200", "_build")


def _to_tree(v, orderarr, n):
    o = orderarr - 1
    return np.concatenate([v[:n][o], v[n:][o]])


def _from_tree(v, orderarr, n):
    o = orderarr - 1
    out = np.empty_like(v)
    out[o] = v[:n]
    out[n + o] = v[n:]
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_benchmark_molecule_solve(gpu_lib):
    import oracle as O
    import tabipb
    from tabipb import workloads

    w = workloads.WORKLOADS["globular"]
    inp = workloads.make_inputs("globular")
    kap = O.kappa(w["bulk"], w["eps1"])
    eps = w["eps1"] / w["eps0"]
    rng = np.random.default_rng(21)
    with tabipb.TabiSolver(order=w["order"], maxparnode=w["maxparnode"], theta=w["theta"],
                           kappa=kap, eps0=w["eps0"], eps1=w["eps1"], tol=w["tol"]) as s:
        xyz, tq, ar, b = s.form_matrix(inp["sptpos"], inp["sptnrm"], inp["nvert"],
                                       inp["chrpos"], inp["atmchr"])
        s.build_tree()
        n = s.nface
        assert n == 92848
        gn = s.tree_nodes()
        go = s.orderarr.copy()
        x = rng.normal(size=2 * n)
        yg = _from_tree(s.matvec(_to_tree(x, go, n)), go, n)
        zg = _from_tree(s.msolve(_to_tree(x, go, n)), go, n)
        near, far = s.counts()
        res = s.dgmres(s.permute(bvct=b)[3])
        se, ce = s.energy(inp["chrpos"], inp["atmchr"], res["x"])
        xg = _from_tree(res["x"], go, n)

    oxyz, otq, oar, ob = O.form_matrix(inp["sptpos"], inp["sptnrm"], inp["nvert"],
                                       inp["chrpos"], inp["atmchr"], w["eps0"], nthreads=NT)
    assert np.array_equal(xyz, oxyz)
    assert _rel(b, ob) < 1e-12
    T = O.Tree(oxyz, otq, oar, ob, w["order"], w["maxparnode"], w["theta"])
    on = T.nodes()
    assert s.nleaf == T.nleaf == 551
    assert np.array_equal(gn["ibeg"], on["ibeg"])
    assert np.array_equal(gn["numpar"], on["iend"] - on["ibeg"] + 1)
    assert np.array_equal(gn["level"], on["level"])
    assert np.array_equal(gn["nchild"], on["nchild"])
    big = gn["numpar"] >= 2
    assert np.array_equal(gn["geo"][big], on["geo"][big])
    for ib, npar in zip(gn["ibeg"], gn["numpar"]):
        assert np.array_equal(np.sort(go[ib - 1: ib - 1 + npar]),
                              np.sort(T.orderarr[ib - 1: ib - 1 + npar]))
    yo, cnt = T.matvec(kap, eps, _to_tree(x, T.orderarr, n), nthreads=NT, return_counts=True)
    assert _rel(yg, _from_tree(yo, T.orderarr, n)) < 1e-10
    assert (near, far) == (int(cnt[0]), int(cnt[1]))
    zo = T.msolve(kap, eps, _to_tree(x, T.orderarr, n), nthreads=NT)
    assert _rel(zg, _from_tree(zo, T.orderarr, n)) < 1e-10
    ores = T.dgmres(kap, eps, T.bvct, iprcd=1, tol=w["tol"], nthreads=NT)
    assert res["ierr"] == ores["ierr"] == 0
    assert res["iter"] == ores["iter"]
    np.testing.assert_allclose(res["err_hist"], ores["err_hist"], rtol=1e-8)
    assert _rel(xg, _from_tree(ores["x"], T.orderarr, n)) < 1e-9
    ose, oce = T.energy(inp["chrpos"], inp["atmchr"], kap, eps, w["eps0"], ores["x"],
                        nthreads=NT)
    assert abs(se - ose) <= 1e-8 * abs(ose), (se, ose)
    assert abs(ce - oce) <= 1e-12 * abs(oce)


def test_large_configuration_matvec_at_sampled_targets(gpu_lib):
    import oracle as O
    import tabipb
    from tabipb import workloads

    w = workloads.WORKLOADS["large"]
    inp = workloads.make_inputs("large")
    kap = O.kappa(w["bulk"], w["eps1"])
    eps = w["eps1"] / w["eps0"]
    prm = dict(order=w["order"], maxparnode=w["maxparnode"], theta=w["theta"], kappa=kap,
               eps0=w["eps0"], eps1=w["eps1"])
    atoms = (np.zeros((1, 3)), np.zeros(1))  # the operator does not depend on the charges
    x = np.random.default_rng(5).normal(size=2 * len(inp["nvert"]))
    ys = {}
    for prec in (tabipb.PREC_FP64, tabipb.PREC_MIXED):
        with tabipb.TabiSolver(precision=prec, **prm) as s:
            xyz, tq, ar, _ = s.form_matrix(inp["sptpos"], inp["sptnrm"], inp["nvert"], *atoms)
            s.build_tree()
            n = s.nface
            ys[prec] = _from_tree(s.matvec(_to_tree(x, s.orderarr, n)), s.orderarr, n)
    assert n == 434048
    T = O.Tree(xyz, tq, ar, None, w["order"], w["maxparnode"], w["theta"])
    T.matvec_prepare(_to_tree(x, T.orderarr, n))
    rows = []
    yo = np.zeros(2 * n)
    for s0 in np.linspace(0, n - 512, 8).astype(int):
        y, _ = T.matvec_targets(kap, eps, int(s0), int(s0) + 512, nthreads=NT)
        t = np.arange(s0, s0 + 512)
        f = T.orderarr[t] - 1           # original face of each oracle tree slot
        yo[f], yo[n + f] = y[t], y[n + t]
        rows.append(f)
    f = np.concatenate(rows)
    pick = lambda v: np.concatenate([v[f], v[n + f]])
    assert _rel(pick(ys[tabipb.PREC_FP64]), pick(yo)) < 1e-10
    assert _rel(pick(ys[tabipb.PREC_MIXED]), pick(yo)) < 2e-5


def _run_driver(tmp_path, name, atoms):
    from tabipb import surface as S

    (tmp_path / "test_proteins").mkdir()
    pqr = tmp_path / "test_proteins" / f"{name}.pqr"
    S.write_pqr(str(pqr), atoms[:, :3], atoms[:, 3], atoms[:, 4])
    # the reference's own usrdata.in (src/usrdata.in) for this molecule
    (tmp_path / "usrdata.in").write_text(
        f"fname {name}\nden 5\nepsp 1\nepsw 80\nbulk_strength 0.15\norder 3\n"
        "maxparnode 100\nmac 0.8\niprcd 1\nisurf_type 1\n")
    out = subprocess.run([os.path.join(BUILD, "tabipb")], cwd=tmp_path, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0, out.stdout + out.stderr
    m = re.search(r"err=\s*(\S+)\s+ierr=\s*(-?\d+)\s+iter=\s*(\d+)", out.stdout)
    se = float(re.search(r"Solvation energy=:\s*(\S+)", out.stdout).group(1))
    return dict(err=float(m.group(1)), ierr=int(m.group(2)), iter=int(m.group(3)), soleng=se,
                pqr=str(pqr))


@pytest.mark.parametrize("name", ["4mn3", "1a63"])
def test_reference_proteins_through_the_driver(gpu_lib, tmp_path, name):
    import oracle as O
    from tabipb import surface as S

    atoms = np.load(os.path.join(ROOT, "tests", "golden", "proteins.npz"))[name]
    drv = _run_driver(tmp_path, name, atoms)
    # the same surface (the generator is deterministic) and atoms for the oracle
    xyz, q, r = S.read_pqr(drv["pqr"])
    S.write_xyzr(str(tmp_path / "o.xyzr"), xyz, r)
    subprocess.run([os.path.join(BUILD, "tabi_msms"), "-if", str(tmp_path / "o.xyzr"), "-prob",
                    "1.4", "-de", "5", "-of", str(tmp_path / "o")], check=True,
                   capture_output=True)
    pos, nrm, fc = S.read_msms(str(tmp_path / "o"))
    fc, _ = O.surface_area(pos, fc)
    kap = O.kappa(0.15, 80.0)
    oxyz, otq, oar, ob = O.form_matrix(pos, nrm, fc, xyz, q, 1.0, nthreads=NT)
    T = O.Tree(oxyz, otq, oar, ob, 3, 100, 0.8)
    ores = T.dgmres(kap, 80.0, T.bvct, iprcd=1, tol=1e-4, nthreads=NT)
    ose, _ = T.energy(xyz, q, kap, 80.0, 1.0, ores["x"], nthreads=NT)
    assert drv["ierr"] == ores["ierr"] == 0
    assert drv["iter"] == ores["iter"]
    assert abs(drv["err"] - ores["err"]) <= 1e-6 * ores["err"]
    assert abs(drv["soleng"] - ose) <= 1e-8 * abs(ose), (drv["soleng"], ose)
