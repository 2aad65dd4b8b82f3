"""tabi_energy_noalloc: the energy entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc (device memory owned by
another allocator, or a pipeline that cannot take cudaFree's device-wide
synchronisation).  Its scratch is a static device array shared by all calls,
so this test calls it twice in a row, through the C ABI, and checks both
results against the allocating entry point (tabi_energy) on the same solution.
The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1, molecule_case

pytestmark = pytest.mark.gpu


def test_energy_noalloc_matches_tabi_energy(gpu_lib):
    import torch

    import tabipb

    case = molecule_case(60, 6.0, 2.0, seed=5)
    kap = tabipb.kappa(BULK, EPS1)
    with tabipb.TabiSolver(order=3, maxparnode=200, theta=0.8, kappa=kap, eps0=EPS0,
                           eps1=EPS1) as s:
        xyz, tq, ar, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                       case["chrpos"], case["atmchr"])
        s.build_tree()
        txyz, ttq, tar, bt = s.permute(xyz, tq, ar, b)
        res = s.dgmres(bt)
        assert res["ierr"] == 0
        se_ref, ce_ref = s.energy(case["chrpos"], case["atmchr"], res["x"])

    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    d_xyz, d_q, d_ar, d_x = t(txyz), t(ttq), t(tar), t(res["x"])
    d_cp, d_qa = t(case["chrpos"]), t(case["atmchr"])
    L = gpu_lib
    for call in range(2):  # the shared scratch keeps the previous call's contents
        out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        rc = L.tabi_energy_noalloc(len(tar), d_xyz.data_ptr(), d_q.data_ptr(), d_ar.data_ptr(),
                                   d_x.data_ptr(), len(case["atmchr"]), d_cp.data_ptr(),
                                   d_qa.data_ptr(), kap, EPS0, EPS1, out.data_ptr(),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, L.tabi_last_error(None)
        torch.cuda.synchronize()
        se, ce = out.cpu().tolist()
        assert abs(se - se_ref) <= 1e-10 * abs(se_ref), (call, se, se_ref)
        assert abs(ce - ce_ref) <= 1e-10 * abs(ce_ref), (call, ce, ce_ref)


def test_energy_noalloc_rejects_oversize(gpu_lib):
    import torch

    dev = torch.device("cuda", 0)
    z = torch.zeros(16, dtype=torch.float64, device=dev)
    rc = gpu_lib.tabi_energy_noalloc(1, z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(),
                                     600000, z.data_ptr(), z.data_ptr(), 0.1, 1.0, 80.0,
                                     z.data_ptr(), None)
    assert rc == -6  # TABI_ERR_LIMIT, checked before any launch
    assert b"524288" in gpu_lib.tabi_last_error(None)


def test_energy_noalloc_many_atoms_one_row(gpu_lib):
    """5,003 atoms (not a multiple of the 8 atoms per block, so the last block
    is partial) over a small surface: 626 atom blocks fill the GPU, the grid
    keeps a single row of face chunks, and the per-atom partial sums then
    need no second row.  Two calls in a row against tabi_energy on the same
    surface, atoms and vector."""
    import torch

    import tabipb

    case = molecule_case(60, 6.0, 2.0, seed=5)
    rng = np.random.default_rng(17)
    natm = 5003
    u = rng.normal(size=(natm, 3))
    cp = u / np.linalg.norm(u, axis=1, keepdims=True) * (3.0 * rng.random((natm, 1)) ** (1 / 3))
    qa = rng.normal(0.0, 0.4, natm)
    kap = tabipb.kappa(BULK, EPS1)
    with tabipb.TabiSolver(order=3, maxparnode=200, theta=0.8, kappa=kap, eps0=EPS0,
                           eps1=EPS1) as s:
        xyz, tq, ar, b = s.form_matrix(case["sptpos"], case["sptnrm"], case["nvert"],
                                       case["chrpos"], case["atmchr"])
        s.build_tree()
        txyz, ttq, tar, _ = s.permute(xyz, tq, ar, b)
        x = rng.normal(size=2 * len(tar))
        se_ref, ce_ref = s.energy(cp, qa, x)

    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    d_xyz, d_q, d_ar, d_x, d_cp, d_qa = t(txyz), t(ttq), t(tar), t(x), t(cp), t(qa)
    for call in range(2):
        out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
        rc = gpu_lib.tabi_energy_noalloc(len(tar), d_xyz.data_ptr(), d_q.data_ptr(),
                                         d_ar.data_ptr(), d_x.data_ptr(), natm, d_cp.data_ptr(),
                                         d_qa.data_ptr(), kap, EPS0, EPS1, out.data_ptr(),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, gpu_lib.tabi_last_error(None)
        torch.cuda.synchronize()
        se, ce = out.cpu().tolist()
        assert abs(se - se_ref) <= 1e-10 * abs(se_ref), (call, se, se_ref)
        assert abs(ce - ce_ref) <= 1e-10 * abs(ce_ref), (call, ce, ce_ref)
