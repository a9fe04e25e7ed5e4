"""Serving benchmark: a seeded, uneven batch of solve requests through the
continuous-batching server (serving.Server over the library's ol_serve_*
layer), against solving the same cases one at a time on the same GPU through
the plain FP32 drop-in path (serving.serial_baseline).

    python -m openludwig_b200.serve_bench [--n 24] [--seed 1234] [--storage f16]
        [--rate 0] [--large-frac 0] [--check-every 200] [--window 2000]
        [--tol 1e-3] [--max-steps 10000] [--budget-gb 160] [--no-serial]

Cases come from workloads.batch_mix (sphere / cube / NACA0012 wing, finest
body size 16-48 cells, 1-3 levels, Re 1e3-1e6, angles of attack and
sideslip; --large-frac adds that share of 64-cell, 3-level cases).  Each
request is prepared when it arrives (host domain build with the device
voxelisation and Bouzidi q-map), so its latency runs from arrival through
preparation, queueing and solving to retirement.  --rate 0 submits every
request at t = 0; a positive rate draws Poisson arrivals (requests per
second).  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import serving as SV
from . import workloads as W
from .native import Context, prepare_case


def case_makers(n: int, seed: int, device: int = 0, large_frac: float = 0.0) -> list:
    """Preparation functions of the seeded batch (called when a request arrives)."""
    out = []
    for i, m in enumerate(W.batch_mix(n, seed=seed, large_frac=large_frac)):
        def make(m=m, i=i):
            cfg, mesh = W.mix_case_config(m)
            cfg.ramp_steps = 0
            return prepare_case(cfg, mesh, f"{m.kind}{m.size_cells}_L{m.levels}_{i}", device=device)
        out.append(make)
    return out


def summary(r: dict) -> dict:
    return {k: v for k, v in r.items() if k != "results"}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=24)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--storage", default="f16", choices=["f16", "f32"])
    ap.add_argument("--rate", type=float, default=0.0)
    ap.add_argument("--large-frac", type=float, default=0.0)
    ap.add_argument("--check-every", type=int, default=200)
    ap.add_argument("--window", type=int, default=2000)
    ap.add_argument("--tol", type=float, default=1e-3)
    ap.add_argument("--max-steps", type=int, default=10000)
    ap.add_argument("--budget-gb", type=float, default=160.0)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-serial", action="store_true")
    a = ap.parse_args()

    makers = case_makers(a.n, a.seed, a.device, a.large_frac)
    arrivals = (SV.poisson_arrivals(a.n, a.rate, seed=a.seed) if a.rate > 0
                else np.zeros(a.n))
    reqs = [SV.Request(i, float(arrivals[i]), mk) for i, mk in enumerate(makers)]
    rule = dict(check_every=a.check_every, window=a.window, tol=a.tol, max_steps=a.max_steps)
    ctx = Context(device=a.device, budget_bytes=int(a.budget_gb * (1 << 30)), storage=a.storage)
    served = SV.Server(ctx, **rule).run(reqs)
    ctx.close()
    line = {"metric": "solves_per_hour", "storage": a.storage, "n": a.n, "seed": a.seed,
            "rate_per_s": a.rate, "large_frac": a.large_frac, "rule": rule,
            "served": summary(served),
            "steps": [r.steps for r in sorted(served["results"], key=lambda r: r.rid)]}
    if not a.no_serial:
        serial = SV.serial_baseline(makers, arrivals, **rule)
        line["serial_f32_dropin"] = summary(serial)
        line["served_over_serial"] = served["solves_per_hour"] / serial["solves_per_hour"]
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
