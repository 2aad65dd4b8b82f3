"""Live kernel timeline of one complete solve (tabi_run_dev) on a named
workload, recorded by CUPTI through torch.profiler: every kernel and copy with
its start, end and stream, as they ran (concurrent streams overlap; nothing
is serialised, unlike a profiler's replay).

    python -m tabipb.trace [--workload globular] [--json out.json]

prints the solve's span and the union of busy intervals, the kernels by
total time, the span and busy time of each stream that ran leaf-LU kernels,
and the longest idle gaps of the GPU with the operations around them.
"""
from __future__ import annotations

import argparse
import collections
import json


def _name(raw: str) -> str:
    nm = raw.replace("(anonymous namespace)::", "").replace("tabi::", "")
    nm = nm.replace("void ", "")
    return nm.split("(")[0]


def trace_solve(workload: str = "globular", warmup: int = 3):
    """[(start_us, end_us, name, stream)] of one solve, sorted by start."""
    import numpy as np
    import torch
    from torch.profiler import ProfilerActivity, profile

    from . import TabiSolver, default_params, kappa
    from .workloads import WORKLOADS, make_inputs

    w = WORKLOADS[workload]
    inp = make_inputs(workload)
    prm = default_params(order=w["order"], theta=w["theta"], maxparnode=w["maxparnode"],
                         kappa=kappa(w["bulk"], w["eps1"]), eps0=w["eps0"], eps1=w["eps1"],
                         tol=w["tol"])
    dev = torch.device("cuda:0")
    d = {k: torch.from_numpy(np.ascontiguousarray(inp[k])).to(dev)
         for k in ("sptpos", "sptnrm", "nvert", "chrpos", "atmchr")}
    stream = torch.cuda.Stream()
    with TabiSolver(prm) as s:
        def run():
            return s.run_dev(d["sptpos"].shape[0], d["sptpos"].data_ptr(),
                             d["sptnrm"].data_ptr(), d["nvert"].shape[0], d["nvert"].data_ptr(),
                             d["chrpos"].shape[0], d["chrpos"].data_ptr(),
                             d["atmchr"].data_ptr(), stream=stream.cuda_stream)

        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as p:
            res = run()
            torch.cuda.synchronize()
    rows = [(e.time_range.start, e.time_range.end, _name(e.name),
             getattr(e, "device_resource_id", -1))
            for e in p.events() if e.device_type == torch.autograd.DeviceType.CUDA]
    rows.sort()
    t0 = rows[0][0]
    return [(a - t0, b - t0, n, sid) for a, b, n, sid in rows], res


def summarize(rows, top: int = 25, gaps: int = 12) -> str:
    out = []
    span = rows[-1][1] - rows[0][0]
    busy, cur_s, cur_e = 0.0, rows[0][0], rows[0][1]
    for a, b, _, _ in rows[1:]:
        if a > cur_e:
            busy += cur_e - cur_s
            cur_s, cur_e = a, b
        else:
            cur_e = max(cur_e, b)
    busy += cur_e - cur_s
    out.append(f"operations {len(rows)}  span {span:.1f} us  busy (union) {busy:.1f} us")
    agg = collections.defaultdict(lambda: [0, 0.0])
    for a, b, n, _ in rows:
        agg[n][0] += 1
        agg[n][1] += b - a
    out.append(f"{'kernel / copy':<44} {'count':>5} {'total us':>10} {'us each':>9}")
    for n, (c, t) in sorted(agg.items(), key=lambda x: -x[1][1])[:top]:
        out.append(f"{n[:44]:<44} {c:>5} {t:>10.1f} {t / c:>9.1f}")
    lu = [r for r in rows if r[2].startswith("lu_")]
    for sid in sorted({r[3] for r in lu}):
        xs = [r for r in lu if r[3] == sid]
        out.append(f"LU stream {sid}: {len(xs)} launches, {xs[0][0]:.0f}-"
                   f"{max(r[1] for r in xs):.0f} us, kernel time {sum(r[1] - r[0] for r in xs):.0f} us")
    idle, cur, prev = [], rows[0][1], rows[0][2]
    for a, b, n, _ in rows[1:]:
        if a > cur + 2.0:
            idle.append((a - cur, cur, prev, n))
        if b > cur:
            cur, prev = b, n
    idle.sort(reverse=True)
    out.append(f"idle gaps > 2 us: {len(idle)}, {sum(g[0] for g in idle):.0f} us in total")
    for g, t, p, n in idle[:gaps]:
        out.append(f"  {g:7.1f} us at {t:8.1f}  after {p[:30]:<30} before {n[:30]}")
    return "\n".join(out)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="globular")
    ap.add_argument("--json", default=None, help="write the rows here")
    a = ap.parse_args(argv)
    rows, res = trace_solve(a.workload)
    print(f"workload {a.workload}: {res['iter']} GMRES iterations")
    print(summarize(rows))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rows, f)


if __name__ == "__main__":
    main()
