"""Serving benchmark: a seeded, uneven batch of solve requests through the
continuous-batching server (serving.Server), against solving the same cases
one at a time on the same GPU (serving.serial_baseline).

    python -m openludwig_b200.serve_bench [--n 24] [--seed 1234] [--storage f16]
        [--rate 0] [--check-every 200] [--window 1000] [--tol 1e-3]
        [--max-steps 4000] [--budget-gb 120] [--no-serial]

Cases come from workloads.batch_mix (sphere / cube / NACA0012 wing, finest
body size 16-48 cells, 1-3 levels, Re 1e3-1e6, angles of attack and
sideslip) and are prepared with the device voxelisation and Bouzidi q-map.
Preparation is timed apart: a request's latency runs from its arrival to its
retirement.  --rate 0 submits every request at t = 0; a positive rate draws
Poisson arrivals (requests per second).  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import serving as SV
from . import workloads as W
from .native import Context, prepare_case


def prepare_batch(n: int, seed: int, device: int = 0) -> tuple[list, float]:
    t0 = time.perf_counter()
    cases = []
    for i, m in enumerate(W.batch_mix(n, seed=seed)):
        cfg, mesh = W.mix_case_config(m)
        cfg.ramp_steps = 0
        cases.append(prepare_case(cfg, mesh, f"{m.kind}{m.size_cells}_L{m.levels}_{i}",
                                  device=device))
    return cases, time.perf_counter() - t0


def _summary(r: dict) -> dict:
    return {k: r[k] for k in ("n", "wall_s", "solves_per_hour") if k in r} | {
        k: r[k] for k in ("p50_s", "p99_s", "converged", "busy_s") if k in r}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=24)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--storage", default="f16", choices=["f16", "f32"])
    ap.add_argument("--rate", type=float, default=0.0)
    ap.add_argument("--check-every", type=int, default=200)
    ap.add_argument("--window", type=int, default=1000)
    ap.add_argument("--tol", type=float, default=1e-3)
    ap.add_argument("--max-steps", type=int, default=4000)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-serial", action="store_true")
    a = ap.parse_args()

    cases, prep_s = prepare_batch(a.n, a.seed, a.device)
    arrivals = (SV.poisson_arrivals(a.n, a.rate, seed=a.seed) if a.rate > 0
                else np.zeros(a.n))
    reqs = [SV.Request(i, float(arrivals[i]), c) for i, c in enumerate(cases)]
    budget = int(a.budget_gb * (1 << 30))
    rule = dict(check_every=a.check_every, window=a.window, tol=a.tol, max_steps=a.max_steps)
    ctx = Context(device=a.device, budget_bytes=budget, storage=a.storage)
    served = SV.Server(ctx, **rule).run(reqs)
    ctx.close()
    line = {"metric": "solves_per_hour", "storage": a.storage, "n": a.n, "seed": a.seed,
            "rate_per_s": a.rate, "rule": rule, "prep_s": prep_s,
            "cell_updates_per_step": [c.cell_updates_per_step for c in cases],
            "served": _summary(served),
            "steps": [r.steps for r in sorted(served["results"], key=lambda r: r.rid)]}
    if not a.no_serial:
        serial = SV.serial_baseline(cases, storage=a.storage, budget_bytes=budget, **rule)
        line["serial"] = _summary(serial)
        if a.rate == 0:
            # every request queued at t = 0: request k completes after cases 0..k
            done = np.cumsum([r.finish_s for r in serial["results"]])
            line["serial"]["p50_s"] = float(np.percentile(done, 50))
            line["serial"]["p99_s"] = float(np.percentile(done, 99))
        line["served_over_serial"] = served["solves_per_hour"] / serial["solves_per_hour"]
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
