#!/usr/bin/env python3
"""TABI-PB solve throughput on B200 -- prints one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

Workload (one "step" = one complete TABI-PB solve of one molecule):
  synthetic globular molecule, 2,000 atoms uniform in an 18 A sphere (minimum
  separation 2.0 A: 3 A is geometrically infeasible at that density), radii
  U(1.5, 2.0) A, charges N(0, 0.4) e shifted to an integer net charge, seed 0;
  surface from the project's MSMS-format generator at 10 vertices/A^2
  (92,848 faces after the reference's face filter); eps 1/80, 0.15 M; Taylor
  order 3, MAC 0.8, leaf 500; GMRES tol 1e-4 (MAXL 10, NRMAX 10); FP64.
  The step runs form_matrix -> tree -> interaction lists -> leaf-block LU ->
  GMRES -> solvation energy on device-resident inputs (tabi_run_dev).

`value` is solves/s over all ranks (device time, CUDA events, max over
ranks); `e2e` runs the same solve through the host-array C ABI
(tabi_form_matrix ... tabi_energy) with the host<->device copies inside the
timed region.  Multi-GPU runs are independent replicas (one molecule per
rank, weak scaling).  `--impl reference` times complete solves of the same
molecule by the CPU restatement of the reference (oracle/, all host threads).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "tabi-pb_b200"), os.path.join(ROOT, "oracle")]

from tabipb.workloads import WORKLOADS  # noqa: E402

WORKLOAD = WORKLOADS["globular"]
WORKLOAD_NAME = WORKLOAD["name"]
METRIC = "solves/s (TABI-PB solve at <=1e-4 dG error; plain FP64)"
# trained warm-start network (tabipb.train_warmstart)
WEIGHTS = os.path.join(ROOT, "tabi-pb_b200", "weights", "warmstart_h160_l3.npz")
OPS_NEAR_PAIR = 64  # algorithmic ops per near-field pair (reference formulas)


def far_ops(p):
    from math import comb

    return 2 * (47 * comb(p + 3, 3) + 12 * comb(p + 6, 3))


def make_inputs():
    from tabipb import workloads

    return workloads.make_inputs(next(k for k, v in WORKLOADS.items() if v is WORKLOAD))


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # sampling has begun once the first line is in; samples taken
            # before the timed region are dropped
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:
                time.sleep(0.01)
            self.lines.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=smax,
                    reasons=sorted(reasons), samples=len(sm))


# ---------------------------------------------------------------- oracle sample
def oracle_estimate(inp, iters, nthreads, target_sample=32768, leaf_sample=48,
                    atom_sample=200, face_frac=0.5):
    """Times the CPU restatement of the reference on a bounded sample of one
    solve and extrapolates: form_matrix RHS on a face subset, full tree build,
    one matvec (moments + a spread sample of targets), one preconditioner
    apply (a few leaves, scaled by sum (2n)^3 -- the reference re-factors
    every leaf on every apply), energy on an atom subset.
    Solve = form + tree + iters*matvec + (iters+2)*msolve + energy."""
    import oracle as O

    w = WORKLOAD
    kap = O.kappa(w["bulk"], w["eps1"])
    eps = w["eps1"] / w["eps0"]
    nface = len(inp["nvert"])
    natm = len(inp["atmchr"])
    t = {}
    # form_matrix: geometry for all faces; RHS sum on a face subset
    xyz, tq, ar, _ = O.form_matrix(inp["sptpos"], inp["sptnrm"], inp["nvert"], np.zeros((0, 3)),
                                   np.zeros(0), w["eps0"])
    sub = inp["nvert"][:: max(1, int(round(1.0 / face_frac)))]
    t0 = time.perf_counter()
    O.form_matrix(inp["sptpos"], inp["sptnrm"], sub, inp["chrpos"], inp["atmchr"], w["eps0"])
    t["form"] = (time.perf_counter() - t0) * nface / len(sub)
    t0 = time.perf_counter()
    T = O.Tree(xyz, tq, ar, None, w["order"], w["maxparnode"], w["theta"])
    t["tree"] = time.perf_counter() - t0
    x = np.random.default_rng(0).normal(size=2 * nface)
    t0 = time.perf_counter()
    T.matvec_prepare(x)
    t_prep = time.perf_counter() - t0
    nb = 16
    per = max(1, target_sample // nb)
    starts = np.linspace(0, nface - per, nb).astype(int)
    t0 = time.perf_counter()
    for s0 in starts:
        T.matvec_targets(kap, eps, s0, s0 + per, nthreads=nthreads)
    t_s = time.perf_counter() - t0
    t["matvec"] = t_prep + t_s * nface / (nb * per)
    ib, nr = T.leaves()
    order = np.argsort(nr)
    pick = order[np.linspace(0, len(order) - 1, min(leaf_sample, len(order))).astype(int)]
    r = np.random.default_rng(1).normal(size=2 * nface)
    t0 = time.perf_counter()
    if leaf_sample >= len(nr):
        pick = order
        T.msolve(kap, eps, r, iprcd=1, nthreads=nthreads)
    else:
        for lf in pick:
            T.msolve(kap, eps, r, iprcd=1, leaf0=int(lf), leaf1=int(lf) + 1, nthreads=nthreads)
    t_l = time.perf_counter() - t0
    cube = (2.0 * nr.astype(float)) ** 3
    t["msolve"] = t_l * cube.sum() / cube[pick].sum()
    asub = np.arange(0, natm, max(1, natm // atom_sample))
    t0 = time.perf_counter()
    O.energy_surface(T.xyz, T.tq, T.area, inp["chrpos"][asub], inp["atmchr"][asub], kap, eps,
                     w["eps0"], np.random.default_rng(2).normal(size=2 * nface),
                     nthreads=nthreads)
    t["energy"] = (time.perf_counter() - t0) * natm / len(asub)
    solve = t["form"] + t["tree"] + iters * t["matvec"] + (iters + 2) * t["msolve"] + t["energy"]
    sample = (f"form_matrix RHS on {len(sub)} of {nface} faces; full tree; one matvec = "
              f"moments + {nb * per} of {nface} targets (16 spread blocks); one "
              f"preconditioner apply = {len(pick)} of {len(nr)} leaves scaled by sum (2n)^3; "
              f"energy on {len(asub)} of {natm} atoms; solve = form + tree + {iters} matvecs + "
              f"{iters + 2} applies + energy")
    return 1.0 / solve, t, sample


# ---------------------------------------------------------------- GPU arm
def gpu_arm(args):
    import torch
    import torch.distributed as dist

    import tabipb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    w = WORKLOAD
    inp = make_inputs()
    dev = torch.device("cuda", local)
    d = {k: torch.from_numpy(inp[k]).to(dev) for k in ("sptpos", "sptnrm", "nvert", "chrpos",
                                                       "atmchr")}
    nspt, nface, natm = len(inp["sptpos"]), len(inp["nvert"]), len(inp["atmchr"])
    kap = tabipb.kappa(w["bulk"], w["eps1"])
    flags = tabipb.FLAG_PIVOTED_LU if args.pivoted_lu else 0
    solver = tabipb.TabiSolver(order=w["order"], maxparnode=w["maxparnode"], theta=w["theta"],
                               kappa=kap, eps0=w["eps0"], eps1=w["eps1"], tol=w["tol"],
                               flags=flags)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def step():
        return solver.run_dev(nspt, d["sptpos"].data_ptr(), d["sptnrm"].data_ptr(), nface,
                              d["nvert"].data_ptr(), natm, d["chrpos"].data_ptr(),
                              d["atmchr"].data_ptr(), None, sp)

    fp64_peak = tabipb.probe_fp64_peak(300.0)
    fp32_peak = tabipb.probe_fp32_peak(300.0)
    for _ in range(args.warmup):
        res = step()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    solver.profile(True)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = step()
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in times)
    prof = solver.profile_read()
    solver.profile(False)
    # the leaf blocks' orders m = 2 x leaf size: the factorisation's work
    # (2/3 m^3 flops per block, DGETRF's leading term) and the factor bytes
    # one apply streams (m^2 doubles per block, plus its 32 x 32 inverse
    # diagonal blocks)
    leaf_m = 2 * solver.leaves()[1].astype(np.float64)
    lu_flop = float((2.0 / 3.0 * leaf_m ** 3).sum())
    apply_bytes = float(8 * (leaf_m ** 2).sum() + 8 * (np.ceil(leaf_m / 32) * 2 * 32 * 32).sum())
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())

    # ---- the same solve with the mixed-precision operator (FP32 treecode,
    # FP64 refinement): same workload, tol, flush and timing
    def timed_leg(solver):
        """The timed loop of the main leg, on another solver configuration."""
        def st():
            return solver.run_dev(nspt, d["sptpos"].data_ptr(), d["sptnrm"].data_ptr(), nface,
                                  d["nvert"].data_ptr(), natm, d["chrpos"].data_ptr(),
                                  d["atmchr"].data_ptr(), None, sp)

        for _ in range(args.warmup):
            r = st()
        torch.cuda.synchronize()
        solver.profile(True)
        tt = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = st()
            e1.record(stream)
            tt.append((e0, e1))
        torch.cuda.synchronize()
        lms = sum(a.elapsed_time(b) for a, b in tt)
        lprof = solver.profile_read()
        solver.profile(False)
        lms_t = torch.tensor([lms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(lms_t, op=dist.ReduceOp.MAX)
        lms = float(lms_t.item())
        return {"value": world * args.steps / (lms / 1e3), "unit": "solves/s",
                "ms_per_step": lms / args.steps, "gmres_iterations": r["iter"],
                "fp64_residual_measure": r["err"], "ierr": r["ierr"],
                "soleng_kcal_mol": r["soleng"],
                "dG_rel_diff_vs_fp64": abs(r["soleng"] - res["soleng"]) / abs(res["soleng"]),
                "phase_ms_per_step": {k: v[0] / args.steps for k, v in lprof.items()
                                      if k != "all"},
                "gpu_launches": int(lprof["all"][1])}

    # ---- the same solve with the mixed-precision operator (FP32 treecode,
    # FP64 refinement), and with the learned warm start on top
    mixed = learned = None
    if not args.no_mixed:
        msolver = tabipb.TabiSolver(order=w["order"], maxparnode=w["maxparnode"],
                                    theta=w["theta"], kappa=kap, eps0=w["eps0"], eps1=w["eps1"],
                                    tol=w["tol"], precision=tabipb.PREC_MIXED)
        mixed = timed_leg(msolver)
        # the FP32 treecode operator alone: its roofline against the FFMA peak
        # and its interaction rate (the same interaction counts as FP64)
        xm = torch.randn(2 * nface, dtype=torch.float64, device=dev)
        ym = torch.empty_like(xm)
        for _ in range(3):
            msolver.matvec_dev(xm.data_ptr(), ym.data_ptr(), 2 * nface, sp)
        ev = []
        for _ in range(10):
            a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            msolver.matvec_dev(xm.data_ptr(), ym.data_ptr(), 2 * nface, sp)
            b_.record(stream)
            ev.append((a, b_))
        torch.cuda.synchronize()
        mv32_s = sum(a.elapsed_time(b_) for a, b_ in ev) / len(ev) / 1e3
        ops32 = res["near_pairs"] * OPS_NEAR_PAIR + res["far"] * far_ops(w["order"])
        mixed["roofline"] = {"kernel": "FP32 treecode matvec: near_kernel_f32 || "
                                       "far_kernel<p, float> (+ moments, reduce)",
                             "bound": "fp32", "achieved": ops32 / mv32_s / 1e12,
                             "peak": fp32_peak / 1e12, "unit": "TFLOP/s",
                             "frac": ops32 / mv32_s / fp32_peak,
                             "peak_source": "FFMA loop probe (tabi_probe_fp32_peak), this GPU",
                             "avg_launch_ms": mv32_s * 1e3}
        mixed["matvec_interactions_per_s"] = (res["near_pairs"] + res["far"]) / mv32_s
        if os.path.exists(WEIGHTS):
            from tabipb.warmstart import WarmStart

            ws = WarmStart.load(WEIGHTS)
            msolver.set_warmstart(ws)
            learned = timed_leg(msolver)
            learned["weights"] = os.path.relpath(WEIGHTS, ROOT)
            msolver.set_warmstart(None)
            ws.close()
        else:
            learned = {"unavailable": "no trained weights at " + os.path.relpath(WEIGHTS, ROOT)}
        msolver.close()

    # ---- end to end through the host-array C ABI: one handle (one molecule
    # at a time, buffers reused), host arrays in and out every step
    e2e_steps = args.steps
    h2d = 0
    d2h = 0
    e2e_solver = tabipb.TabiSolver(order=w["order"], maxparnode=w["maxparnode"],
                                   theta=w["theta"], kappa=kap, eps0=w["eps0"], eps1=w["eps1"],
                                   tol=w["tol"])

    # the step's inputs and outputs in page-locked host memory (as a caller
    # streaming molecules would hold them); the tensors keep the buffers alive
    pinned_t = {k: torch.from_numpy(np.ascontiguousarray(inp[k], dtype=dt)).pin_memory()
                for k, dt in (("sptpos", np.float64), ("sptnrm", np.float64),
                              ("nvert", np.int32), ("chrpos", np.float64),
                              ("atmchr", np.float64))}
    pin = {k: t.numpy() for k, t in pinned_t.items()}
    # and the arrays the step reads back
    nf = len(inp["nvert"])
    for k, shape in (("xyz", (nf, 3)), ("tq", (nf, 3)), ("ar", (nf,)), ("b", (2 * nf,)),
                     ("bt", (2 * nf,)), ("x", (2 * nf,))):
        pinned_t[k] = torch.empty(shape, dtype=torch.float64).pin_memory()
        pin[k] = pinned_t[k].numpy()

    def e2e_once():
        nonlocal h2d, d2h
        s = e2e_solver
        xyz, tq, ar, b = s.form_matrix(pin["sptpos"], pin["sptnrm"], pin["nvert"],
                                       pin["chrpos"], pin["atmchr"],
                                       out=(pin["xyz"], pin["tq"], pin["ar"], pin["b"]))
        s.build_tree()
        _, _, _, bt = s.permute(bvct=b)
        pin["bt"][:] = bt
        bt = pin["bt"]
        r = s.dgmres(bt, out=pin["x"])
        se, ce = s.energy(pin["chrpos"], pin["atmchr"], r["x"])
        h2d = (pin["sptpos"].nbytes + pin["sptnrm"].nbytes + pin["nvert"].nbytes
               + pin["chrpos"].nbytes + pin["atmchr"].nbytes + 2 * bt.nbytes
               + pin["chrpos"].nbytes + pin["atmchr"].nbytes + r["x"].nbytes)
        d2h = (xyz.nbytes + tq.nbytes + ar.nbytes + b.nbytes + 4 * nface + r["x"].nbytes + 16)
        return se

    e2e_once()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        se_e2e = e2e_once()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_t.item())
    e2e_solver.close()

    batched = batched_leg(args, dev, rank) if args.batch > 0 else None
    large = large_leg(args, dev) if (args.large and rank == 0) else None

    out = None
    if rank == 0:
        near_ms, near_n = prof["near"]
        far_ms, far_n = prof["far"]
        mv_ms, mv_n = prof["matvec"]
        n_mv = max(mv_n, 1)
        near_pairs, far_int = res["near_pairs"], res["far"]
        mv_avg_s = mv_ms / n_mv / 1e3
        ops_mv = near_pairs * OPS_NEAR_PAIR + far_int * far_ops(WORKLOAD["order"])
        achieved = ops_mv / mv_avg_s / 1e12
        peak = fp64_peak / 1e12
        value = world * args.steps / (ms_max / 1e3)
        out = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "faces": nface, "vertices": nspt,
                       "atoms": natm, "order": w["order"], "theta": w["theta"],
                       "maxparnode": w["maxparnode"], "tol": w["tol"],
                       "gmres_iterations": res["iter"], "leaves": res["nleaf"],
                       "soleng_kcal_mol": res["soleng"],
                       "parallelism": f"replicas x{world}",
                       "l2": "256 MB buffer written between timed steps"},
            "matvec_interactions_per_s": (near_pairs + far_int) / mv_avg_s,
            "interactions_per_matvec": {"near_pairs": near_pairs, "far": far_int},
            "phase_ms_per_step": {k: v[0] / args.steps for k, v in prof.items() if k != "all"},
            "roofline": {"kernel": "treecode matvec: near_kernel || far_kernel<p> "
                                   "(+ moments, reduce), fork to join",
                         "bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                         "peak_source": "DFMA loop probe (tabi_probe_fp64_peak), this GPU",
                         "ops_per_launch": ops_mv, "avg_launch_ms": mv_avg_s * 1e3,
                         "ops_per_unit": {"near_pair": OPS_NEAR_PAIR,
                                          "far_interaction": far_ops(WORKLOAD["order"])},
                         "near_kernel_avg_ms": near_ms / max(near_n, 1),
                         "far_kernel_avg_ms": far_ms / max(far_n, 1)},
            "lu": lu_entry(prof, lu_flop, fp64_peak),
            "apply": apply_entry(prof, apply_bytes),
            "e2e": {"value": world / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(prof["all"][1]),
            "clocks": clk,
        }
        if mixed is not None:
            out["mixed"] = mixed
            out["mixed_learned"] = learned
        if batched is not None:
            out["batched"] = batched
        if large is not None:
            out["large_mixed"] = large
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, parts, sample = oracle_estimate(inp, res["iter"], nthreads=1)
        out["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": 1, "kind": "port",
                               "sample": sample,
                               "phase_s": {k: round(x, 4) for k, x in parts.items()}}
    if out is not None:
        print(json.dumps(out), flush=True)
    solver.close()


# ---------------------------------------------------------------- large mixed leg
LARGE = WORKLOADS["large"]


def large_leg(args, dev):
    """The large mixed-precision configuration: 20,000 atoms in 40 A (same
    generator, 10 vertices/A^2), order 6, MAC 0.7, leaf 400, FP32 treecode with
    FP64 refinement to 1e-6 (FP64 residual measure).  Reported: solves/s (one
    timed solve after one warm-up), iterations, and the operator's error
    against the FP64 direct sum (tabi_direct_targets) at 10,000 sampled
    targets, for the FP32 and the FP64 treecode."""
    import torch

    import tabipb
    from tabipb import workloads

    w = LARGE
    inp = workloads.make_inputs("large")
    pos, nrm, fc, xyz, q = (inp["sptpos"], inp["sptnrm"], inp["nvert"], inp["chrpos"],
                            inp["atmchr"])
    nspt, nface, natm = len(pos), len(fc), len(q)
    f = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d = dict(sptpos=f(pos), sptnrm=f(nrm), nvert=f(np.asarray(fc, np.int32)), chrpos=f(xyz),
             atmchr=f(q))
    kap = tabipb.kappa(w["bulk"], w["eps1"])
    prm = dict(order=w["order"], maxparnode=w["maxparnode"], theta=w["theta"], kappa=kap,
               eps0=w["eps0"], eps1=w["eps1"], tol=w["tol"])
    s32 = tabipb.TabiSolver(precision=tabipb.PREC_MIXED, **prm)
    x = torch.zeros(2 * nface, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def run():
        return s32.run_dev(nspt, d["sptpos"].data_ptr(), d["sptnrm"].data_ptr(), nface,
                           d["nvert"].data_ptr(), natm, d["chrpos"].data_ptr(),
                           d["atmchr"].data_ptr(), x.data_ptr(), stream.cuda_stream)

    run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = run()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    xt = x.cpu().numpy()
    rng = np.random.default_rng(11)
    tg = np.sort(rng.choice(nface, min(10000, nface), replace=False)).astype(np.int32)
    yd1, yd2 = s32.direct_targets(tg, xt)
    y32 = s32.matvec(xt)
    s64 = tabipb.TabiSolver(**prm)
    s64.form_matrix(pos, nrm, fc, xyz, q)
    s64.build_tree()
    y64 = s64.matvec(xt)
    s64.close()
    s32.close()
    yd = np.concatenate([yd1, yd2])
    pick = lambda y: np.concatenate([y[tg], y[nface + tg]])
    rel = lambda y: float(np.linalg.norm(pick(y) - yd) / np.linalg.norm(yd))
    return {"value": 1e3 / ms, "unit": "solves/s", "ms_per_solve": ms, "workload": w["name"],
            "faces": nface, "atoms": natm, "gmres_iterations": res["iter"],
            "fp64_residual_measure": res["err"], "ierr": res["ierr"],
            "soleng_kcal_mol": res["soleng"], "near_pairs_per_matvec": res["near_pairs"],
            "far_per_matvec": res["far"],
            "operator_rel_error_vs_fp64_direct_sum": {"targets": int(tg.size),
                                                      "fp32_treecode": rel(y32),
                                                      "fp64_treecode": rel(y64)},
            "note": "the generator at 10 vertices/A^2 gives this face count for 20,000 atoms "
                    "in 40 A"}


# ---------------------------------------------------------------- batched leg
def _batch_surface(job):
    natm, seed, density = job
    from tabipb import surface as S
    from tabipb.warmstart import globular_radius

    xyz, q, r = S.synthetic_molecule(natm, globular_radius(natm), min_sep=2.0, seed=seed)
    pos, nrm, fc, _ = S.gaussian_surface(xyz, r, density=density, probe=1.4)
    fc, _ = S.face_filter(pos, fc)
    return natm, seed, pos, nrm, fc, xyz, q


def hbm_peak_gbs():
    """The measured copy bandwidth of this pool's B200s (the driver-written
    peaks file at the repository root), else the earlier pool measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (6.65 TB/s, earlier pool measurement)"


def lu_entry(prof, lu_flop, fp64_peak):
    """The leaf-block factorisation's FP64 rate: its work over the span from
    its first launch to the join of both LU streams (library event timer)."""
    ms, n = prof.get("lu", (0.0, 0))
    if n <= 0 or ms <= 0:
        return None
    t = ms / n
    return {"flop_per_factorisation": lu_flop, "ms": t, "tflops": lu_flop / t / 1e9,
            "frac_of_fp64_peak": lu_flop / t / 1e9 / (fp64_peak / 1e12),
            "timing": "CUDA events around the factorisation (both streams), mean over the timed steps"}


def apply_entry(prof, apply_bytes):
    """The preconditioner apply's streaming rate against the HBM peak: the
    factor bytes over one apply's span (fork to join)."""
    ms, n = prof.get("apply", (0.0, 0))
    if n <= 0 or ms <= 0:
        return None
    peak, src = hbm_peak_gbs()
    t = ms / n
    return {"bytes_per_apply": apply_bytes, "us": t * 1e3, "gbs": apply_bytes / t / 1e6,
            "frac_of_hbm": apply_bytes / t / 1e6 / peak, "hbm_peak_gbs": peak,
            "peak_source": src, "applies_per_step": n / max(prof.get("lu", (0, 1))[1], 1)}


def batched_leg(args, dev, rank):
    """Many molecules of uneven size in one tabi_batch_run_dev call: atom counts
    log-uniform in 300..8000 (seeded; rank r uses seeds r*1000 + k), the
    benchmark's atom density and surface density, mixed precision, tol 1e-4,
    leaf size per size class from the autotuner, the trained warm start when
    its weights exist, and the worker count (1, 2 or --batch-workers) that
    ran the first quarter of the batch fastest.  The whole batch is timed on
    one worker (the same molecules back to back) and on that count, best of 3
    each; the leg reports the faster (`workers`, with the tuner's pick in
    `tuned_workers`), both values and the per-molecule wall-time
    percentiles."""
    import multiprocessing as mp

    import torch

    import tabipb
    from tabipb import batch as B

    rng = np.random.default_rng(7 + rank)
    sizes = np.exp(rng.uniform(np.log(300), np.log(8000), args.batch)).astype(int)
    jobs = [(int(n), rank * 1000 + k, 10.0) for k, n in enumerate(sizes)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        hosts = pool.map(_batch_surface, jobs, chunksize=1)
    t_gen = time.perf_counter() - t0
    f = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    mols = [dict(natm=n, seed=sd, nspt=len(pos), nface=len(fc), nchr=n, sptpos=f(pos),
                 sptnrm=f(nrm), nvert=torch.from_numpy(np.ascontiguousarray(fc, np.int32)).to(dev),
                 chrpos=f(xyz), atmchr=f(q)) for n, sd, pos, nrm, fc, xyz, q in hosts]
    w = WORKLOAD
    prm = tabipb.default_params(order=w["order"], theta=w["theta"], maxparnode=w["maxparnode"],
                                kappa=tabipb.kappa(w["bulk"], w["eps1"]), eps0=w["eps0"],
                                eps1=w["eps1"], tol=w["tol"], precision=tabipb.PREC_MIXED)
    # autotune the leaf size on one probe molecule per size class present
    probes = {}
    for m in mols:
        probes.setdefault(B.size_class(m["nface"]), m)
    table, timings = B.autotune(list(probes.values()), prm, candidates=(300, 500, 700),
                                repeats=1)
    ws = None
    if os.path.exists(WEIGHTS):
        from tabipb.warmstart import WarmStart

        ws = WarmStart.load(WEIGHTS)
    B.run_batch(mols[:2], prm, ws=ws, nworkers=2, table=table)  # warm-up
    # worker count: measured on the first quarter of the batch (at least 8)
    cands = tuple(sorted({1, 2, args.batch_workers}))
    nw, wt = B.tune_workers(mols[: max(8, len(mols) // 4)], prm, table, candidates=cands, ws=ws,
                            repeats=2)

    def best_of(n, nworkers):  # the batch call's wall time varies run to run
        runs = [B.run_batch(mols, prm, ws=ws, nworkers=nworkers, table=table) for _ in range(n)]
        return min(runs, key=lambda r: r[1])

    seq, t_seq = best_of(3, 1)
    par, t_par = best_of(3, nw) if nw != 1 else (seq, t_seq)
    tuned_workers = nw
    if t_par > t_seq:  # the subset's choice did not carry over: one worker ran faster
        nw, par, t_par = 1, seq, t_seq
    ok = bool(np.all(par[:, 2] == 0)) and bool(np.array_equal(seq[:, 3], par[:, 3]))
    # each molecule's solvation energy against its own plain solve (FP64,
    # leaf 500, no warm start, the same tol): the error of the accelerated
    # configuration (FP32 treecode + refinement, tuned leaf size, warm start)
    prm64 = tabipb.default_params(order=w["order"], theta=w["theta"],
                                  maxparnode=w["maxparnode"],
                                  kappa=tabipb.kappa(w["bulk"], w["eps1"]), eps0=w["eps0"],
                                  eps1=w["eps1"], tol=w["tol"], precision=tabipb.PREC_FP64)
    ref64, _ = B.run_batch(mols, prm64, ws=None, nworkers=nw, table=None)
    dg_err = np.abs(par[:, 3] - ref64[:, 3]) / np.abs(ref64[:, 3])
    return {"value": len(mols) / t_par, "unit": "molecules/s", "molecules": len(mols),
            "workers": nw, "tuned_workers": tuned_workers,
            "worker_tuning_s": {str(k): round(v, 4) for k, v in wt.items()},
            "sequential_value": len(mols) / t_seq,
            "speedup_vs_sequential": t_seq / t_par,
            "faces_min_max": [int(min(m["nface"] for m in mols)),
                              int(max(m["nface"] for m in mols))],
            "atoms": "log-uniform 300..8000, seeded", "precision": "mixed", "tol": w["tol"],
            "warm_start": ws is not None,
            "leaf_table": {str(k): v for k, v in table.items()},
            "per_molecule_ms_p50": float(np.percentile(par[:, 8], 50)),
            "per_molecule_ms_p99": float(np.percentile(par[:, 8], 99)),
            "all_converged_and_equal_to_sequential": ok,
            "dG_rel_err_vs_plain_fp64_leaf500": {"max": float(dg_err.max()),
                                                 "p99": float(np.percentile(dg_err, 99)),
                                                 "median": float(np.median(dg_err))},
            "timing": "host wall clock around the whole batch call (inputs on the device), "
                      "best of 3 calls",
            "surface_generation_s": t_gen}


# ---------------------------------------------------------------- reference arm
def oracle_solve(inp, nthreads):
    """One complete solve by the CPU restatement of the reference (oracle/):
    form_matrix -> tree -> DGMRES (the leaf blocks re-factored on every
    preconditioner apply, as LEAFMATVECpara does) -> energy, on nthreads host
    threads.  Returns (seconds per phase, result)."""
    import oracle as O

    w = WORKLOAD
    kap = O.kappa(w["bulk"], w["eps1"])
    eps = w["eps1"] / w["eps0"]
    t0 = time.perf_counter()
    xyz, tq, ar, b = O.form_matrix(inp["sptpos"], inp["sptnrm"], inp["nvert"], inp["chrpos"],
                                   inp["atmchr"], w["eps0"], nthreads=nthreads)
    t1 = time.perf_counter()
    T = O.Tree(xyz, tq, ar, b, w["order"], w["maxparnode"], w["theta"])
    t2 = time.perf_counter()
    r = T.dgmres(kap, eps, T.bvct, iprcd=1, tol=w["tol"], nthreads=nthreads)
    t3 = time.perf_counter()
    se, ce = T.energy(inp["chrpos"], inp["atmchr"], kap, eps, w["eps0"], r["x"],
                      nthreads=nthreads)
    t4 = time.perf_counter()
    t = dict(form=t1 - t0, tree=t2 - t1, dgmres=t3 - t2, energy=t4 - t3)
    return t, dict(iter=r["iter"], ierr=r["ierr"], err=r["err"], soleng=se, couleng=ce,
                   n_matvec=r["n_matvec"], n_msolve=r["n_msolve"])


def reference_arm(args):
    """The reference's CPU path on the host cores: every timed step is one
    complete solve of the benchmark molecule by the oracle (the C restatement
    of the reference; the Fortran cannot be built here) on all host threads.
    The untimed warm-up steps run a bounded sample of the same code paths."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    inp = make_inputs()
    for _ in range(args.warmup):
        oracle_estimate(inp, 6, nthreads, target_sample=2048, leaf_sample=4, atom_sample=16,
                        face_frac=0.05)
    t0 = time.perf_counter()
    steps = []
    for _ in range(args.steps):
        ts = time.perf_counter()
        parts, res = oracle_solve(inp, nthreads)
        steps.append(time.perf_counter() - ts)
    wall = time.perf_counter() - t0
    value = args.steps / sum(steps)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(steps) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "faces": len(inp["nvert"]),
                   "atoms": len(inp["atmchr"]), "gmres_iterations": res["iter"],
                   "soleng_kcal_mol": res["soleng"]},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads,
                         "kind": "port",
                         "sample": "complete solves (form_matrix, tree, DGMRES with the leaf "
                                   "blocks re-factored on every apply as the reference does, "
                                   "energy) of the benchmark molecule, every timed step; "
                                   f"{nthreads} host threads",
                         "phase_s": {k: round(x, 4) for k, x in parts.items()},
                         "matvecs": res["n_matvec"], "applies": res["n_msolve"]},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "timed_wall_s": wall,
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("gpu", "reference"), default="gpu")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision leg (FP32 treecode + FP64 refinement)")
    ap.add_argument("--batch", type=int, default=256,
                    help="molecules in the batched leg (0 skips it)")
    ap.add_argument("--batch-workers", type=int, default=4)
    ap.add_argument("--no-large", dest="large", action="store_false",
                    help="skip the large mixed-precision leg (20,000 atoms, order 6, tol 1e-6)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="globular")
    ap.add_argument("--pivoted-lu", action="store_true",
                    help="factor every leaf block with partial pivoting (TABI_FLAG_PIVOTED_LU) "
                         "in the main leg, instead of the certified unpivoted factorisation")
    args = ap.parse_args()
    global WORKLOAD, WORKLOAD_NAME
    WORKLOAD = WORKLOADS[args.workload]
    WORKLOAD_NAME = WORKLOAD["name"]
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
