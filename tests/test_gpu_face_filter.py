"""readin.f90:264-333 surface_area on the device (tabi_face_filter_dev)
against the oracle's restatement: the same kept faces in the same order, the
same total area up to summation order, on raw generator surfaces (whose
welded vertices leave a few slivers and repeats for the filter to find) and
on a surface with planted repeats and zero-area faces."""
import numpy as np
import pytest

from conftest import BULK, EPS0, EPS1

pytestmark = pytest.mark.gpu


def _filter_gpu(pos, fc):
    import torch

    import tabipb

    dev = torch.device("cuda", 0)
    sp = torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float64)).to(dev)
    nv = torch.from_numpy(np.ascontiguousarray(fc, dtype=np.int32)).to(dev)
    out = torch.full_like(nv, -7)
    with tabipb.TabiSolver(kappa=tabipb.kappa(BULK, EPS1), eps0=EPS0, eps1=EPS1) as s:
        nk, area = s.face_filter_dev(len(pos), sp.data_ptr(), len(fc), nv.data_ptr(),
                                     out.data_ptr())
    torch.cuda.synchronize()
    return out[:nk].cpu().numpy(), area


@pytest.mark.parametrize("natm,seed,density", [(60, 1, 2.0), (300, 4, 6.0), (1500, 7, 10.0)])
def test_face_filter_matches_oracle(gpu_lib, natm, seed, density):
    import oracle as O
    from tabipb import surface as S
    from tabipb.warmstart import globular_radius

    xyz, q, r = S.synthetic_molecule(natm, globular_radius(natm), min_sep=2.0, seed=seed)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=density, probe=1.4)
    kept, area = _filter_gpu(pos, fc)
    okept, oarea = O.surface_area(pos, fc)
    assert np.array_equal(kept, okept)
    assert abs(area - oarea) <= 1e-12 * oarea


def test_face_filter_planted_repeats_and_slivers(gpu_lib):
    import oracle as O
    from tabipb import surface as S

    pos, nrm, fc = S.icosphere(3, 2.0)
    fc = fc.copy()
    rng = np.random.default_rng(3)
    # repeats 1..10 faces later (dropped) and 11 faces later (kept), and
    # faces with a repeated vertex (zero area)
    planted = []
    for k in rng.choice(len(fc) - 20, 40, replace=False):
        lag = int(rng.integers(1, 12))
        planted.append((k + lag, fc[k].copy()))
    for i, f in planted:
        fc[i] = f
    for i in rng.choice(len(fc), 25, replace=False):
        fc[i, 2] = fc[i, 1]
    kept, area = _filter_gpu(pos, fc)
    okept, oarea = O.surface_area(pos, fc)
    assert len(okept) < len(fc) - 40
    assert np.array_equal(kept, okept)
    assert abs(area - oarea) <= 1e-12 * oarea


def test_face_filter_rejects_bad_vertex_index(gpu_lib):
    import torch

    import tabipb
    from tabipb import surface as S
    from tabipb._lib import TabiError

    pos, nrm, fc = S.icosphere(2, 2.0)
    fc = fc.copy()
    fc[17, 1] = len(pos) + 1
    dev = torch.device("cuda", 0)
    sp = torch.from_numpy(np.ascontiguousarray(pos)).to(dev)
    nv = torch.from_numpy(np.ascontiguousarray(fc, dtype=np.int32)).to(dev)
    out = torch.empty_like(nv)
    with tabipb.TabiSolver() as s:
        with pytest.raises(TabiError) as e:
            s.face_filter_dev(len(pos), sp.data_ptr(), len(fc), nv.data_ptr(), out.data_ptr())
    assert e.value.code == -1
