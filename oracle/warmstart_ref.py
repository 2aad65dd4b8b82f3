"""CPU reference of the learned warm-start network (numpy, FP64 arithmetic).

TEST INFRASTRUCTURE ONLY: tests use it to check the CUDA forward pass, loss and
gradients of libtabi_gpu.so's warm-start network (tabi_ws_* in
include/tabi_gpu.h); nothing in the product imports it.  The reference solver
has no learned component: this restates the network the CUDA kernels
implement, term for term, so the two can be compared.

Network ("panel network"), for one molecule of N panels (centroid r_i, unit
normal n_i, area A_i, right-hand side b = [b1; b2] of main.f90:592-606, and
z = [z1; z2] = M^-1 b, the leaf-block preconditioner's solution, which solves
the boundary integral equations exactly within each leaf; without z, z = [0; b2]):

  neighbours  nbr(i, :) = the K nearest other panels by centroid distance,
              ascending, ties by index
  scales      s = sqrt(mean b1^2), Abar = mean A, dbar_i = mean_k |r_j - r_i|
  node input  f_i (10): b1_i/s, b2_i/s, log(A_i/Abar), log(Abar),
              mean_k n_i.(r_j - r_i) dbar_i / |r_j - r_i|^2, mean_k n_i.n_j,
              log(dbar_i), mean_k (b1_j - b1_i)/s, asinh(z1_i/s), asinh((z2_i - b2_i)/s)
  edge input  e_ij (R + 3): exp(-((|r_ij|/dbar_i - mu_m)/sigma)^2) for
              mu_m = 2.5 m/(R-1), sigma = 2.5/(R-1); n_i.n_j; n_i.r_ij/|r_ij|;
              n_j.r_ij/|r_ij|   (r_ij = r_j - r_i)
  layers      h = silu(f W0 + b0)
              repeat L times:  u = h Wa
                               a_i = 1/K sum_k silu(e_ij Wf + bf) * u_j
                               z = h Wb1 + a Wb2 + bb ;  h = h + silu(z)
  output      o = h Wo + bo ;  x1 = z1 + s o_0 ,  x2 = z2 + s o_1
  loss        1/N sum_i (o_i0 - (x1_i - z1_i)/s)^2 + (o_i1 - (x2_i - z2_i)/s)^2

Every input is invariant under rotations and translations of the molecule,
so the predicted potentials are too; scaling all charges scales s, b and the
prediction alike.  Weight matrices are used rounded to bfloat16 (round to
nearest even); biases stay FP32.
"""
from __future__ import annotations

import numpy as np

NODE_F = 10


def edge_dim(R):
    return R + 3


def param_shapes(H, L, R):
    """Flat parameter layout, in order: (name, shape)."""
    E = edge_dim(R)
    out = [("W0", (NODE_F, H)), ("b0", (H,))]
    for l in range(L):
        out += [(f"Wa{l}", (H, H)), (f"Wf{l}", (E, H)), (f"bf{l}", (H,)), (f"Wb1{l}", (H, H)),
                (f"Wb2{l}", (H, H)), (f"bb{l}", (H,))]
    out += [("Wo", (H, 2)), ("bo", (2,))]
    return out


def nparams(H, L, R):
    return sum(int(np.prod(s)) for _, s in param_shapes(H, L, R))


def unpack(theta, H, L, R):
    p, o = {}, 0
    for name, shp in param_shapes(H, L, R):
        k = int(np.prod(shp))
        p[name] = theta[o:o + k].reshape(shp)
        o += k
    return p


def pack(grads, H, L, R):
    return np.concatenate([grads[name].ravel() for name, _ in param_shapes(H, L, R)])


def bf16_round(w):
    """float32 -> bfloat16 (round to nearest, ties to even) -> float64."""
    a = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    a = ((a + 0x7FFF + lsb) >> 16) << 16
    return a.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(x):
    return x / (1.0 + np.exp(-x))


def dsilu(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def knn(pos, K):
    """K nearest other panels (brute force; ties by index)."""
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    n = len(pos)
    out = np.empty((n, K), np.int64)
    for i0 in range(0, n, 512):
        blk = pos[i0:i0 + 512]
        d2 = ((blk[:, None, :] - pos[None, :, :]) ** 2).sum(-1)
        d2[np.arange(len(blk)), np.arange(i0, i0 + len(blk))] = np.inf
        idx = np.argsort(d2, axis=1, kind="stable")[:, :K]  # stable: ties by index
        out[i0:i0 + 512] = idx
    return out


def baseline(b, z):
    n = len(b) // 2
    return np.concatenate([np.zeros(n), b[n:]]) if z is None else np.asarray(z, np.float64)


def features(pos, nrm, area, b, nbr, R, z=None):
    n = len(area)
    b1, b2 = b[:n], b[n:]
    z = baseline(b, z)
    s = np.sqrt(np.mean(b1 * b1))
    if s == 0.0:
        s = 1.0
    abar = area.mean()
    rij = pos[nbr] - pos[:, None, :]                    # N x K x 3
    d = np.sqrt((rij * rij).sum(-1))                    # N x K
    dbar = d.mean(1)
    ni = nrm[:, None, :]
    nj = nrm[nbr]
    f = np.zeros((n, NODE_F))
    f[:, 0] = b1 / s
    f[:, 1] = b2 / s
    f[:, 2] = np.log(area / abar)
    f[:, 3] = np.log(abar)
    f[:, 4] = ((ni * rij).sum(-1) * dbar[:, None] / (d * d)).mean(1)
    f[:, 5] = (ni * nj).sum(-1).mean(1)
    f[:, 6] = np.log(dbar)
    f[:, 7] = ((b1[nbr] - b1[:, None]) / s).mean(1)
    f[:, 8] = np.arcsinh(z[:n] / s)
    f[:, 9] = np.arcsinh((z[n:] - b2) / s)
    mu = 2.5 * np.arange(R) / (R - 1)
    sig = 2.5 / (R - 1)
    rho = d / dbar[:, None]
    e = np.zeros((n, nbr.shape[1], edge_dim(R)))
    e[..., :R] = np.exp(-(((rho[..., None] - mu) / sig) ** 2))
    e[..., R] = (ni * nj).sum(-1)
    e[..., R + 1] = (ni * rij).sum(-1) / d
    e[..., R + 2] = (nj * rij).sum(-1) / d
    return f, e, s


def forward(theta, H, L, R, pos, nrm, area, b, nbr, target=None, round_bf16=True, z=None):
    """Returns (x_pred, loss or None, cache).  round_bf16=False keeps the
    weights exact (for finite-difference checks of backward())."""
    th = np.asarray(theta, np.float32 if round_bf16 else np.float64)
    p = {k: (bf16_round(v) if (round_bf16 and k.startswith("W")) else v.astype(np.float64))
         for k, v in unpack(th, H, L, R).items()}
    n = len(area)
    K = nbr.shape[1]
    f, e, s = features(pos, nrm, area, b, nbr, R, z)
    zb = baseline(b, z)
    pre0 = f @ p["W0"] + p["b0"]
    h = silu(pre0)
    cache = dict(f=f, e=e, s=s, pre0=pre0, hs=[h], us=[], pres=[], as_=[], zs=[], p=p)
    for l in range(L):
        u = h @ p[f"Wa{l}"]
        pre = e @ p[f"Wf{l}"] + p[f"bf{l}"]            # N x K x H
        a = (silu(pre) * u[nbr]).sum(1) / K
        zl = h @ p[f"Wb1{l}"] + a @ p[f"Wb2{l}"] + p[f"bb{l}"]
        h = h + silu(zl)
        cache["us"].append(u)
        cache["pres"].append(pre)
        cache["as_"].append(a)
        cache["zs"].append(zl)
        cache["hs"].append(h)
    o = h @ p["Wo"] + p["bo"]
    cache["o"] = o
    x = np.concatenate([zb[:n] + s * o[:, 0], zb[n:] + s * o[:, 1]])
    loss = None
    if target is not None:
        t0 = (target[:n] - zb[:n]) / s
        t1 = (target[n:] - zb[n:]) / s
        loss = np.mean((o[:, 0] - t0) ** 2 + (o[:, 1] - t1) ** 2)
        cache["t"] = np.stack([t0, t1], 1)
    return x, loss, cache


def backward(cache, H, L, R, nbr):
    """Gradient of the loss with respect to the flat parameters."""
    p = cache["p"]
    o, t = cache["o"], cache["t"]
    n = len(o)
    K = nbr.shape[1]
    g = {}
    do = 2.0 * (o - t) / n
    h = cache["hs"][L]
    g["Wo"] = h.T @ do
    g["bo"] = do.sum(0)
    dh = do @ p["Wo"].T
    e = cache["e"]
    for l in reversed(range(L)):
        hin = cache["hs"][l]
        z, a, u, pre = cache["zs"][l], cache["as_"][l], cache["us"][l], cache["pres"][l]
        dz = dh * dsilu(z)
        g[f"Wb1{l}"] = hin.T @ dz
        g[f"Wb2{l}"] = a.T @ dz
        g[f"bb{l}"] = dz.sum(0)
        dhin = dh + dz @ p[f"Wb1{l}"].T
        da = dz @ p[f"Wb2{l}"].T
        gate = silu(pre)                                  # N x K x H
        du = np.zeros_like(u)
        np.add.at(du, nbr, gate * da[:, None, :] / K)
        dpre = u[nbr] * da[:, None, :] / K * dsilu(pre)
        g[f"Wf{l}"] = np.einsum("ike,ikh->eh", e, dpre)
        g[f"bf{l}"] = dpre.sum((0, 1))
        g[f"Wa{l}"] = hin.T @ du
        dhin = dhin + du @ p[f"Wa{l}"].T
        dh = dhin
    dpre0 = dh * dsilu(cache["pre0"])
    g["W0"] = cache["f"].T @ dpre0
    g["b0"] = dpre0.sum(0)
    return pack(g, H, L, R)


def init_params(H, L, R, seed=0):
    """Scaled normal weights (all matrices, the output layer included, so that
    every gradient is non-zero), zero biases; for checks of the CUDA side."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shp in param_shapes(H, L, R):
        if name.startswith("W"):
            fan_in = shp[0]
            parts.append(rng.standard_normal(shp) / np.sqrt(fan_in))
        else:
            parts.append(np.zeros(shp))
    return np.concatenate([q.ravel() for q in parts]).astype(np.float32)
