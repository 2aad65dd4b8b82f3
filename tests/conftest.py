"""Shared test setup: import paths, the gpu marker, common fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "tabi-pb_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libtabi_gpu.so")


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    """Built libtabi_gpu.so; GPU tests fail (not skip) when it is missing."""
    import build_lib as _b  # tabi-pb_b200/build_lib.py

    _b.build()
    import tabipb

    return tabipb.load()


# ---- standard inputs
EPS0, EPS1, BULK = 1.0, 80.0, 0.15


def born_case(level=4, radius=2.0):
    from tabipb import surface as S

    pos, nrm, fc = S.icosphere(level, radius)
    return dict(sptpos=pos, sptnrm=nrm, nvert=fc, chrpos=np.zeros((1, 3)),
                atmchr=np.array([1.0]), atmrad=np.array([radius]))


def molecule_case(natm=60, radius=6.0, density=2.0, seed=1):
    from tabipb import surface as S

    xyz, q, r = S.synthetic_molecule(natm, radius, min_sep=2.0, seed=seed)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=density, probe=1.4)
    import oracle as O

    fc2, _ = O.surface_area(pos, fc)
    return dict(sptpos=pos, sptnrm=nrm, nvert=fc2, chrpos=xyz, atmchr=q, atmrad=r)
