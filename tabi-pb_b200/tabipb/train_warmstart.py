"""Trains the warm-start network on solutions of this solver and evaluates it.

    python -m tabipb.train_warmstart --train 500 --test 50 --epochs 20 \\
        --out tabi-pb_b200/weights/warmstart_h160_l3.npz

Training molecules: synthetic globules (the benchmark generator at the
benchmark's atom density and 10 vertices/A^2 surfaces) with atom counts
log-uniform in [--min-atoms, --max-atoms], seeds 10000 + k; held-out
molecules: --test-atoms atoms, seeds 90000 + k.  Each is solved from zero to
--tol (mixed precision); the network is trained on those solutions and then
evaluated by the GMRES iterations and solve time to --tol from its prediction
against from zero, on the held-out set.  Surfaces are generated by a pool of
host processes (started before the GPU is touched).
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np


def _surface(args):
    natm, seed, density = args
    from tabipb import surface as S
    from tabipb.warmstart import globular_radius

    xyz, q, r = S.synthetic_molecule(natm, globular_radius(natm), min_sep=2.0, seed=seed)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=density, probe=1.4)
    fc, _ = S.face_filter(pos, fc)
    return dict(natm=natm, seed=seed, sptpos=pos, sptnrm=nrm, nvert=fc, chrpos=xyz, atmchr=q)


def solve_sample(h, tol, device="cuda"):
    """Solves one molecule from zero; returns the tree-ordered device sample."""
    import torch

    from tabipb import PREC_MIXED
    from tabipb.solver import TabiSolver, kappa

    prm = dict(order=3, maxparnode=500, theta=0.8, kappa=kappa(0.15, 80.0), eps0=1.0, eps1=80.0,
               tol=tol, precision=PREC_MIXED)
    with TabiSolver(**prm) as s:
        txyz, ttq, tar, b = s.form_matrix(h["sptpos"], h["sptnrm"], h["nvert"], h["chrpos"],
                                          h["atmchr"])
        s.build_tree()
        txyz, ttq, tar, bt = s.permute(txyz, ttq, tar, b)
        zt = s.msolve(bt)
        res = s.dgmres(bt)
    dev = torch.device(device)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).ravel()).to(dev)
    return dict(n=len(tar), natm=h["natm"], seed=h["seed"], xyz=t(txyz), tq=t(ttq), area=t(tar),
                b=t(bt), z=t(zt), x=t(res["x"]), iters=res["iter"], ierr=res["ierr"],
                host={k: h[k] for k in ("sptpos", "sptnrm", "nvert", "chrpos", "atmchr")},
                prm=prm)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=500)
    ap.add_argument("--test", type=int, default=50)
    ap.add_argument("--min-atoms", type=int, default=500)
    ap.add_argument("--max-atoms", type=int, default=5000)
    ap.add_argument("--test-atoms", type=int, default=3000)
    ap.add_argument("--density", type=float, default=10.0)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=5e-5)
    ap.add_argument("--hidden", type=int, default=160)
    ap.add_argument("--layers", type=int, default=3)
    ap.add_argument("--procs", type=int, default=min(16, os.cpu_count() or 1))
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None, help="JSON summary path")
    a = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)

    rng = np.random.default_rng(2024)
    sizes = np.exp(rng.uniform(np.log(a.min_atoms), np.log(a.max_atoms), a.train)).astype(int)
    jobs = [(int(n), 10000 + k, a.density) for k, n in enumerate(sizes)]
    jobs += [(a.test_atoms, 90000 + k, a.density) for k in range(a.test)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(a.procs) as pool:
        hosts = pool.map(_surface, jobs, chunksize=1)
    t_surf = time.perf_counter() - t0
    log(f"{len(hosts)} surfaces in {t_surf:.1f} s ({a.procs} processes)")

    import torch

    from tabipb.warmstart import WarmStart, evaluate, train

    t0 = time.perf_counter()
    samples = [solve_sample(h, a.tol) for h in hosts]
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - t0
    tr, te = samples[:a.train], samples[a.train:]
    log(f"solved {len(samples)} molecules in {t_solve:.1f} s; faces "
        f"{min(s['n'] for s in samples)}..{max(s['n'] for s in samples)}")
    ws = WarmStart(a.hidden, a.layers, seed=0)
    t0 = time.perf_counter()
    hist = train(ws, tr, epochs=a.epochs, lr=a.lr, lr_final=a.lr_final, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    ev = evaluate(ws, te, tol=a.tol)
    it0 = float(np.mean([e["iters_zero"] for e in ev]))
    itw = float(np.mean([e["iters_ws"] for e in ev]))
    s0 = float(np.mean([e["solve_s_zero"] for e in ev]))
    sw = float(np.mean([e["solve_s_ws"] + e["predict_s"] for e in ev]))
    rep = dict(train_molecules=a.train, test_molecules=a.test, atoms=[a.min_atoms, a.max_atoms],
               test_atoms=a.test_atoms, density=a.density, tol=a.tol, epochs=a.epochs,
               hidden=a.hidden, layers=a.layers, nparams=ws.nparams,
               loss_first_epoch=hist[0], loss_last_epoch=hist[-1],
               surface_s=t_surf, solve_s=t_solve, train_s=t_train,
               test_iters_from_zero=it0, test_iters_from_network=itw,
               test_iters_from_baseline=float(np.mean([e["iters_baseline"] for e in ev])),
               test_solve_s_from_zero=s0, test_solve_s_from_network_incl_predict=sw,
               test_x0_rel_err_mean=float(np.mean([e["x0_rel_err"] for e in ev])),
               all_converged=all(e["ierr"] == (0, 0) for e in ev))
    log(json.dumps(rep))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)
    if a.out:
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        ws.save(a.out, train_molecules=a.train, epochs=a.epochs, density=a.density,
                min_atoms=a.min_atoms, max_atoms=a.max_atoms, tol=a.tol)
    return rep


if __name__ == "__main__":
    main()
