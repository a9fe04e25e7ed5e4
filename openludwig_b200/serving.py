"""Continuous-batching solve service over the native context.

Requests (prepared cases) arrive over time; the loop admits them as soon as
their HBM footprint fits the budget, advances every resident case together
(one graph replay per coarse step), checks each case's drag coefficient every
`check_every` of its own steps, and retires a case when
|Cd(t) - Cd(t - window)| < tol, or at `max_steps`.  Requests that arrive
while others run join the next chunk: work of cases at different ages
overlaps on the device.  Latency = retirement time - arrival time; the clock
is wall time measured around the device work (host domain preprocessing is
done before a request is submitted and is not part of its latency).
"""
from __future__ import annotations

import dataclasses as dc
import time

import numpy as np

from .native import Context, PreparedCase


@dc.dataclass
class Request:
    rid: int
    arrival_s: float
    case: PreparedCase


@dc.dataclass
class Result:
    rid: int
    arrival_s: float
    admit_s: float
    finish_s: float
    steps: int
    cd: float
    converged: bool
    status: int
    cd_history: list

    @property
    def latency_s(self) -> float:
        return self.finish_s - self.arrival_s


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


class Server:
    def __init__(self, ctx: Context, check_every: int = 200, window: int = 2000,
                 tol: float = 1e-3, max_steps: int = 20000, min_steps: int | None = None):
        if window % check_every:
            raise ValueError("window must be a multiple of check_every")
        self.ctx = ctx
        self.check_every = check_every
        self.window = window
        self.tol = tol
        self.max_steps = max_steps
        self.min_steps = window if min_steps is None else min_steps

    def _converged(self, hist: list) -> bool:
        lag = self.window // self.check_every
        if len(hist) <= lag:
            return False
        return abs(hist[-1] - hist[-1 - lag]) < self.tol

    def run(self, requests: list[Request], clock=time.perf_counter) -> dict:
        ctx = self.ctx
        pending = sorted(requests, key=lambda r: r.arrival_s)
        queue: list[Request] = []
        resident: dict[int, dict] = {}
        results: list[Result] = []
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        budget = ctx.stats()["budget"]
        i = 0
        busy_s = 0.0
        while i < len(pending) or queue or resident:
            while i < len(pending) and pending[i].arrival_s <= now():
                queue.append(pending[i])
                i += 1
            if not resident and not queue and i < len(pending):
                # idle: wait for the next arrival
                time.sleep(max(0.0, min(0.05, pending[i].arrival_s - now())))
                continue
            # admit in arrival order while the footprint fits
            while queue:
                r = queue[0]
                need = ctx.footprint(r.case)
                if ctx.stats()["used"] + need > budget:
                    if not resident:
                        raise RuntimeError(f"request {r.rid} needs {need} B, above the budget")
                    break
                cid = ctx.add_case(r.case)
                resident[cid] = {"req": r, "admit": now(), "cd": []}
                queue.pop(0)
            if not resident:
                continue
            s0 = clock()
            ctx.step(self.check_every)
            ctx.sync()
            busy_s += clock() - s0
            done = []
            for cid, st in resident.items():
                steps, status = ctx.info(cid)
                cd = ctx.forces(cid).Cd
                st["cd"].append(cd)
                conv = steps >= self.min_steps and self._converged(st["cd"])
                if conv or status & 1 or steps >= self.max_steps or not np.isfinite(cd):
                    done.append((cid, steps, status, conv))
            for cid, steps, status, conv in done:
                st = resident.pop(cid)
                ctx.remove_case(cid)
                r = st["req"]
                results.append(Result(r.rid, r.arrival_s, st["admit"], now(), steps,
                                      st["cd"][-1], conv, status, st["cd"]))
        wall = now()
        lat = np.array([r.latency_s for r in results]) if results else np.zeros(1)
        return {
            "n": len(results),
            "converged": int(sum(r.converged for r in results)),
            "wall_s": wall,
            "busy_s": busy_s,
            "solves_per_hour": len(results) / wall * 3600.0 if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)),
            "results": results,
        }


def serial_baseline(cases: list[PreparedCase], storage: str = "f32", budget_bytes: int = 8 << 30,
                    check_every: int = 200, window: int = 2000, tol: float = 1e-3,
                    max_steps: int = 20000, clock=time.perf_counter) -> dict:
    """One case at a time on the same GPU (the plain form the service is
    compared with): same convergence rule, no overlap between cases."""
    out = []
    t0 = clock()
    for k, case in enumerate(cases):
        ctx = Context(budget_bytes=budget_bytes, storage=storage)
        srv = Server(ctx, check_every, window, tol, max_steps)
        r = srv.run([Request(k, 0.0, case)], clock=clock)
        out.append(r["results"][0])
        ctx.close()
    wall = clock() - t0
    return {"n": len(out), "wall_s": wall, "solves_per_hour": len(out) / wall * 3600.0,
            "results": out}
