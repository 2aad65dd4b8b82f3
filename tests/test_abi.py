"""C ABI checks that need no GPU: the library builds for sm_100a, loads, and
exports every function include/tabi_gpu.h declares; calls fail cleanly (an
error code, no crash) when no GPU is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "tabi_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tabi_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_abi():
    names = declared_functions()
    for must in ("tabi_create", "tabi_matvec", "tabi_msolve", "tabi_solve", "tabi_energy",
                 "tabi_build_tree", "tabi_form_matrix"):
        assert must in names


def test_library_exports_every_symbol(gpu_lib):
    for name in declared_functions():
        assert hasattr(gpu_lib, name), name
    import tabipb._lib as L

    assert sorted(L.SYMBOLS) == declared_functions()


def test_library_is_sm100a(gpu_lib):
    # the in-tree build passes only sm_100a to nvcc
    import build_lib

    assert "arch=compute_100a,code=sm_100a" in " ".join(build_lib.ARCH)
    assert os.path.exists(build_lib.LIB)


def test_kappa_and_defaults(gpu_lib):
    import tabipb

    assert tabipb.kappa(0.15, 80.0) == 0.12572533685666004
    p = tabipb.default_params()
    assert (p.order, p.maxparnode, p.theta, p.iprcd, p.maxl, p.nrmax) == (3, 500, 0.8, 1, 10, 10)
    assert p.tol == 1e-4


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_cleanly(gpu_lib):
    import tabipb

    with pytest.raises(tabipb.TabiError) as ei:
        tabipb.TabiSolver()
    assert ei.value.code == -2


def test_bad_params_rejected(gpu_lib):
    import tabipb

    for kw in (dict(theta=1.0), dict(order=0), dict(order=9), dict(maxparnode=0),
               dict(eps0=0.0)):
        with pytest.raises(tabipb.TabiError) as ei:
            tabipb.TabiSolver(**kw)
        assert ei.value.code in (-1, -6) or (ei.value.code == -2 and not has_gpu())
