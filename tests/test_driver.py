"""The host driver tabipb (mirror of the reference's program TABIPB,
main.f90:11-222): usrdata.in + test_proteins/<fname>.pqr in, surface from
tabi_msms with MSMS's flags, solve through the C ABI, surface_potential.dat
out.  Its energy must equal the library's on the same surface."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "tabi-pb_b200", "_build")


def test_driver_matches_library(gpu_lib, tmp_path):
    import tabipb
    from tabipb import surface as S

    xyz, q, r = S.synthetic_molecule(40, 5.0, min_sep=2.0, seed=7)
    (tmp_path / "test_proteins").mkdir()
    S.write_pqr(str(tmp_path / "test_proteins" / "mol.pqr"), xyz, q, r)
    (tmp_path / "usrdata.in").write_text(
        "fname mol\nden 2\nepsp 1\nepsw 80\nbulk_strength 0.15\norder 3\nmaxparnode 100\n"
        "mac 0.8\niprcd 1\nisurf_type 1\n")
    out = subprocess.run([os.path.join(BUILD, "tabipb")], cwd=tmp_path, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    se = float(re.search(r"Solvation energy=:\s*(\S+)", out.stdout).group(1))
    dat = (tmp_path / "surface_potential.dat").read_text().split("\n")
    nspt, nface = map(int, dat[0].split())
    assert len(dat) >= 1 + nspt + nface
    # same surface through the library API (PQR values are REAL*4, as the driver reads them)
    xyz32, q32, r32 = S.read_pqr(str(tmp_path / "test_proteins" / "mol.pqr"))
    S.write_xyzr(str(tmp_path / "m.xyzr"), xyz32, r32)
    subprocess.run([os.path.join(BUILD, "tabi_msms"), "-if", str(tmp_path / "m.xyzr"), "-prob",
                    "1.4", "-de", "2", "-of", str(tmp_path / "m")], check=True,
                   capture_output=True)
    pos, nrm, fc = S.read_msms(str(tmp_path / "m"))
    import oracle as O

    fc, _ = O.surface_area(pos, fc)
    res = tabipb.solve_molecule(pos, nrm, fc, xyz32, q32, order=3, maxparnode=100, theta=0.8,
                                kappa=tabipb.kappa(0.15, 80.0), eps0=1.0, eps1=80.0)
    assert res["ierr"] == 0
    assert abs(se - res["soleng"]) <= 1e-9 * abs(res["soleng"]), (se, res["soleng"])
    # vertex potentials of surface_potential.dat (main.f90:307-312), against
    # the oracle's output_potential of the same solution
    xyz_o, _, _, _ = O.form_matrix(pos, nrm, fc, xyz32, q32, 1.0)
    vert_ref, _ = O.output_potential(pos, fc, xyz_o, res["x_orig"])
    vert_dat = np.array([[float(t) for t in line.split()[7:9]] for line in dat[1:1 + nspt]])
    ok = np.isfinite(vert_ref[:, 0])
    np.testing.assert_allclose(vert_dat[ok], vert_ref[ok], rtol=1e-7, atol=2e-10)
