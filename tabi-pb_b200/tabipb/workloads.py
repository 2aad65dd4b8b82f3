"""Named synthetic workloads of the benchmark and the scale tests.

Seeded stand-ins for molecules (no dataset is involved): atoms uniform in a
sphere with a 2.0 A minimum separation (3 A is geometrically infeasible at
these densities: 2,000 atoms in 18 A is a packing fraction of 1.16), radii
U(1.5, 2.0) A, charges N(0, 0.4) e shifted to an integer net charge; surface
from the project's MSMS-format generator, then the reference's face filter
(readin.f90:264-333); eps 1/80, 0.15 M.

* ``globular`` -- 2,000 atoms in 18 A, 10 vertices/A^2 (92,848 faces); order
  3, MAC 0.8, leaf 500, GMRES tol 1e-4, FP64: the benchmark molecule.
* ``medium``   -- 600 atoms in 12 A with the same settings (profiler captures).
* ``large``    -- 20,000 atoms in 40 A, 10 vertices/A^2 (434,048 faces);
  order 6, MAC 0.7, leaf 400, tol 1e-6 (the large mixed-precision solve).
"""
from __future__ import annotations

import numpy as np

WORKLOADS = {
    "globular": dict(natm=2000, radius=18.0, min_sep=2.0, density=10.0, probe=1.4, seed=0,
                     order=3, theta=0.8, maxparnode=500, tol=1e-4, eps0=1.0, eps1=80.0,
                     bulk=0.15, name="globular-2000-atoms-18A-10vA2-p3-mac0.8-leaf500-fp64"),
    "medium": dict(natm=600, radius=12.0, min_sep=2.0, density=10.0, probe=1.4, seed=0,
                   order=3, theta=0.8, maxparnode=500, tol=1e-4, eps0=1.0, eps1=80.0,
                   bulk=0.15, name="globular-600-atoms-12A-10vA2-p3-mac0.8-leaf500-fp64"),
    "large": dict(natm=20000, radius=40.0, min_sep=2.0, density=10.0, probe=1.4, seed=0,
                  order=6, theta=0.7, maxparnode=400, tol=1e-6, eps0=1.0, eps1=80.0, bulk=0.15,
                  name="large-20000-atoms-40A-10vA2-p6-mac0.7-leaf400-mixed-tol1e-6"),
}


def make_inputs(name: str = "globular") -> dict:
    """Host arrays of one workload: sptpos, sptnrm (nspt, 3), nvert (nface, 3)
    1-based and face-filtered, chrpos (natm, 3), atmchr (natm,), grid step."""
    from . import surface as S

    w = WORKLOADS[name]
    xyz, q, r = S.synthetic_molecule(w["natm"], w["radius"], min_sep=w["min_sep"],
                                     seed=w["seed"])
    pos, nrm, fc, h = S.gaussian_surface(xyz, r, density=w["density"], probe=w["probe"])
    fc, _ = S.face_filter(pos, fc)
    return dict(sptpos=np.ascontiguousarray(pos), sptnrm=np.ascontiguousarray(nrm),
                nvert=np.ascontiguousarray(fc, dtype=np.int32),
                chrpos=np.ascontiguousarray(xyz), atmchr=np.ascontiguousarray(q), grid=h)
