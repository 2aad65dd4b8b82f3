"""The CPU reference of the warm-start network: its backward pass against
finite differences of its forward pass (exact weights), and its invariance
under a rigid motion of the molecule.  The GPU kernels are checked against
this reference in test_gpu_warmstart.py."""
import numpy as np

from conftest import molecule_case


def _mol():
    import oracle as O

    c = molecule_case(30, 5.0, 1.0, seed=7)
    xyz, tq, ar, b = O.form_matrix(c["sptpos"], c["sptnrm"], c["nvert"], c["chrpos"],
                                   c["atmchr"], 1.0)
    return xyz.reshape(-1, 3), tq.reshape(-1, 3), ar, b


def test_backward_matches_finite_differences():
    import warmstart_ref as W

    pos, nrm, area, b = _mol()
    n = len(area)
    sel = np.arange(0, n, max(1, n // 300))[:300]
    pos, nrm, area = pos[sel], nrm[sel], area[sel]
    b = np.concatenate([b[:n][sel], b[n:][sel]])
    H, L, R, K = 8, 2, 4, 6
    nbr = W.knn(pos, K)
    theta = W.init_params(H, L, R, seed=3).astype(np.float64) * 0.7
    rng = np.random.default_rng(5)
    target = rng.standard_normal(2 * len(area)) * np.std(b)
    z = b + 0.1 * rng.standard_normal(b.size) * np.std(b)
    _, loss, cache = W.forward(theta, H, L, R, pos, nrm, area, b, nbr, target, round_bf16=False,
                               z=z)
    g = W.backward(cache, H, L, R, nbr)
    idx = rng.choice(theta.size, 60, replace=False)
    h = 1e-6
    for k in idx:
        tp = theta.copy()
        tp[k] += h
        tm = theta.copy()
        tm[k] -= h
        lp = W.forward(tp, H, L, R, pos, nrm, area, b, nbr, target, round_bf16=False, z=z)[1]
        lm = W.forward(tm, H, L, R, pos, nrm, area, b, nbr, target, round_bf16=False, z=z)[1]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (k, fd, g[k])


def test_prediction_invariant_under_rigid_motion():
    import warmstart_ref as W

    pos, nrm, area, b = _mol()
    H, L, R, K = 8, 2, 4, 8
    theta = W.init_params(H, L, R, seed=1)
    x0 = W.forward(theta, H, L, R, pos, nrm, area, b, W.knn(pos, K))[0]
    q, _ = np.linalg.qr(np.random.default_rng(2).standard_normal((3, 3)))
    pos2 = pos @ q.T + np.array([3.0, -1.0, 7.5])
    nrm2 = nrm @ q.T
    x1 = W.forward(theta, H, L, R, pos2, nrm2, area, b, W.knn(pos2, K))[0]
    np.testing.assert_allclose(x1, x0, rtol=1e-9, atol=1e-12)


def test_param_count_of_the_shipped_shape():
    import warmstart_ref as W

    assert W.nparams(160, 3, 8) == 238722
