"""Input generators: icosphere (Born), synthetic molecules, the MSMS-format
surface generator and its file format (readin.f90:204-246)."""
import os

import numpy as np

from conftest import EPS0, molecule_case


def test_icosphere_counts():
    from tabipb import surface as S

    pos, nrm, fc = S.icosphere(4, 2.0)
    assert pos.shape == (2562, 3) and fc.shape == (5120, 3)
    assert fc.min() == 1 and fc.max() == 2562
    np.testing.assert_allclose(np.linalg.norm(pos, axis=1), 2.0, rtol=1e-14)
    np.testing.assert_allclose(pos / 2.0, nrm, atol=1e-15)


def test_msms_roundtrip(tmp_path):
    from tabipb import surface as S

    pos, nrm, fc = S.icosphere(2, 2.0)
    prefix = str(tmp_path / "ico")
    S.write_msms(prefix, pos, nrm, fc)
    p2, n2, f2 = S.read_msms(prefix)
    assert np.array_equal(f2, fc)
    np.testing.assert_allclose(p2, np.round(pos, 3), atol=1e-12)


def test_synthetic_molecule():
    from tabipb import surface as S

    xyz, q, r = S.synthetic_molecule(200, 9.0, min_sep=2.0, seed=3)
    assert xyz.shape == (200, 3)
    assert (np.linalg.norm(xyz, axis=1) <= 9.0).all()
    d = np.linalg.norm(xyz[:, None] - xyz[None], axis=2) + np.eye(200) * 10
    assert d.min() >= 2.0
    assert abs(q.sum() - round(q.sum())) < 1e-9
    assert (r >= 1.5).all() and (r <= 2.0).all()
    x2, q2, r2 = S.synthetic_molecule(200, 9.0, min_sep=2.0, seed=3)
    assert np.array_equal(xyz, x2) and np.array_equal(q, q2)


def test_gaussian_surface_closed_and_outward():
    from tabipb import surface as S

    xyz = np.zeros((1, 3))
    pos, nrm, fc, h = S.gaussian_surface(xyz, np.array([2.0]), density=4.0, quantize=False)
    # a single blob is a sphere of radius 2 (rho = 1 where |x| = r)
    rr = np.linalg.norm(pos, axis=1)
    np.testing.assert_allclose(rr, 2.0, rtol=2e-3)
    np.testing.assert_allclose((nrm * pos).sum(1) / rr, 1.0, atol=1e-6)  # outward
    # closed: every edge shared by exactly two faces
    e = np.sort(np.concatenate([fc[:, [0, 1]], fc[:, [1, 2]], fc[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert (cnt == 2).all()
    # density close to the request
    area = 4 * np.pi * 4.0
    assert 0.6 < len(pos) / area / 4.0 < 1.6


def test_pqr_reader(tmp_path):
    from tabipb import surface as S

    p = str(tmp_path / "m.pqr")
    with open(p, "w") as f:
        f.write("REMARK x\nATOM      1  N   GLY     1      -1.065   5.170  -7.209  0.2943  1.5500\n")
        f.write("ATOM      2  CA  GLY     1       0.100   0.200   0.300 -0.0100  1.7000\nEND\n")
    xyz, q, r = S.read_pqr(p)
    assert xyz.shape == (2, 3)
    assert q[0] == np.float32(0.2943) and r[1] == np.float32(1.7)


def test_molecule_case_pipeline():
    c = molecule_case(30, 5.0, 1.0, seed=4)
    import oracle as O

    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], EPS0)
    assert (ar > 0).all()
    np.testing.assert_allclose(np.linalg.norm(tq, axis=1), 1.0, atol=1e-12)


def test_face_filter_matches_oracle():
    """tabipb.surface.face_filter (the product's readin.f90:264-333) keeps the
    same faces as the oracle's restatement, duplicates and slivers included."""
    import oracle as O
    from tabipb import surface as S

    xyz, q, r = S.synthetic_molecule(120, 7.0, min_sep=2.0, seed=9)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=4.0, probe=1.4)
    base, _ = S.face_filter(pos, fc)
    # plant a repeat of face 5 right after it (caught: within the 10 faces
    # before it), one at the end (not caught: the reference looks back 10
    # faces only) and a zero-area sliver
    fc = np.concatenate([fc[:6], fc[5:6], fc[6:], fc[5:6],
                         np.array([[fc[7, 0], fc[7, 0], fc[7, 1]]])])
    a, sa = O.surface_area(pos, fc)
    b, sb = S.face_filter(pos, fc)
    assert np.array_equal(a, b)
    assert len(b) == len(base) + 1
    assert abs(sa - sb) <= 1e-12 * sa
