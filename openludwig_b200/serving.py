"""Continuous-batching solve service: the Python driver of the library's
serving layer (ol_server_* / ol_serve_*, csrc/serve.cu).

Requests arrive over time.  A request carries either a prepared case or a
function that prepares it (host domain build with the device voxelisation
and Bouzidi q-map); lazy requests are prepared when they arrive, on a pool
of host threads, so their latency counts the preparation.  Prepared cases
are submitted to the library with their arrival time; the library admits
them in arrival order as soon as their HBM footprint fits the context's
budget, advances every resident case together (one graph replay per coarse
step), checks each case's drag coefficient every `check_every` of its own
steps, and retires a case when |Cd(t) - Cd(t - window)| < tol (after
min_steps), on its watchdog flag, at max_steps or on a non-finite Cd.
Requests that arrive while others run join the next chunk: work of cases
at different ages overlaps on the device.

Latency = retirement time - arrival time, on the library's steady clock.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import dataclasses as dc
import time
from typing import Callable, Union

import numpy as np

from . import _native as N
from .native import COEFF_NAMES, Context, PreparedCase, build_case_desc, coeff_ref

CaseSource = Union[PreparedCase, Callable[[], PreparedCase]]


@dc.dataclass
class Request:
    rid: int
    arrival_s: float
    case: CaseSource


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
    coefficients: dict = dc.field(default_factory=dict)
    prep_s: float = 0.0

    @property
    def latency_s(self) -> float:
        return self.finish_s - self.arrival_s


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


def _summary(results: list, wall: float, busy: float = 0.0) -> dict:
    lat = np.array([r.latency_s for r in results]) if results else np.zeros(1)
    prep = np.array([r.prep_s for r in results]) if results else np.zeros(1)
    return {
        "n": len(results),
        "converged": int(sum(r.converged for r in results)),
        "wall_s": wall,
        "busy_s": busy,
        "solves_per_hour": len(results) / wall * 3600.0 if wall > 0 else 0.0,
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
        "prep_p50_s": float(np.percentile(prep, 50)),
        "results": results,
    }


class Server:
    def __init__(self, ctx: Context, check_every: int = 200, window: int = 2000,
                 tol: float = 1e-3, max_steps: int = 20000, min_steps: int | None = None,
                 prep_workers: int = 4):
        if window % check_every:
            raise ValueError("window must be a multiple of check_every")
        self.ctx = ctx
        self.rule = N.ServeRule(check_every=check_every, window=window, tol=tol,
                                max_steps=max_steps,
                                min_steps=window if min_steps is None else min_steps)
        self.prep_workers = max(1, prep_workers)

    def run(self, requests: list[Request]) -> dict:
        h = C.c_void_p()
        N.call("ol_server_create", C.byref(h), self.ctx._h, C.byref(self.rule))
        pool = cf.ThreadPoolExecutor(self.prep_workers)
        try:
            return self._loop(h, requests, pool)
        finally:
            pool.shutdown(wait=True)
            N.call("ol_server_destroy", h)

    def _loop(self, h, requests, pool) -> dict:
        clock = C.c_double()

        def now() -> float:
            N.call("ol_server_clock", h, C.byref(clock))
            return clock.value

        pending = sorted(requests, key=lambda r: r.arrival_s)
        by_rid: dict[int, tuple] = {}    # library rid -> (request, case, desc keep-alive, prep_s)
        preparing: list[tuple] = []       # (request, future or None, start)
        results: list[Result] = []
        out = (N.ServeResult * 64)()
        n_res, n_queued, n_out = C.c_int32(), C.c_int32(), C.c_int32()
        hist = (C.c_double * 4096)()
        busy = 0.0
        i = 0
        while True:
            t = now()
            while i < len(pending) and pending[i].arrival_s <= t:
                r = pending[i]
                i += 1
                if isinstance(r.case, PreparedCase):
                    preparing.append((r, None, t))
                else:
                    preparing.append((r, pool.submit(r.case), t))
            still = []
            for r, fut, start in preparing:
                if fut is not None and not fut.done():
                    still.append((r, fut, start))
                    continue
                case = r.case if fut is None else fut.result()
                prep_s = 0.0 if fut is None else now() - start
                cd, keep = build_case_desc(case, self.ctx.f16_scale)
                ref = coeff_ref(case)
                rid = C.c_int32()
                N.call("ol_serve_submit", h, C.byref(cd), C.byref(ref), r.arrival_s, C.byref(rid))
                by_rid[rid.value] = (r, case, (cd, keep, ref), prep_s)
            preparing = still
            s0 = time.perf_counter()
            N.call("ol_serve_advance", h, C.byref(n_res), C.byref(n_queued))
            if n_res.value:
                busy += time.perf_counter() - s0
            while True:
                N.call("ol_serve_poll", h, out, len(out), C.byref(n_out))
                for k in range(n_out.value):
                    o = out[k]
                    r, case, _, prep_s = by_rid.pop(o.rid)
                    nh = C.c_int32()
                    N.call("ol_serve_history", h, o.rid, hist, len(hist), C.byref(nh))
                    coeff = dict(zip(COEFF_NAMES, o.coeff[:]))
                    results.append(Result(r.rid, o.arrival_s, o.admit_s, o.finish_s, o.steps,
                                          coeff["Cd"], bool(o.converged), o.status,
                                          list(hist[:min(nh.value, len(hist))]), coeff, prep_s))
                if n_out.value < len(out):
                    break
            if i >= len(pending) and not preparing and not by_rid:
                break
            if n_res.value == 0:
                # nothing on the device: wait for an arrival or a preparation
                nxt = pending[i].arrival_s - now() if i < len(pending) else 0.005
                time.sleep(min(0.05, max(0.0005, nxt)))
        return _summary(results, now(), busy)


def serial_baseline(cases: list, arrivals=None, check_every: int = 200, window: int = 2000,
                    tol: float = 1e-3, max_steps: int = 20000, min_steps: int | None = None,
                    device=None) -> dict:
    """The plain form the service is compared with: one case at a time on the
    same GPU through the FP32 drop-in path (solver.Simulation: one
    ol_stream_collide / Bouzidi call per level sub-step), the same
    convergence rule, no overlap between cases.  `cases` are prepared cases
    or preparation functions (prepared in turn, and counted).  Arrivals: the
    serial queue starts each case when it has arrived and the previous one
    has finished; latency = finish - arrival."""
    import torch

    from .solver import Simulation
    dev = device or torch.device("cuda", torch.cuda.current_device())
    min_steps = window if min_steps is None else min_steps
    lag = window // check_every
    arrivals = np.zeros(len(cases)) if arrivals is None else np.asarray(arrivals, float)
    order = np.argsort(arrivals, kind="stable")
    results = []
    t_free = 0.0
    for k in order:
        item = cases[k]
        t0 = time.perf_counter()
        case = item if isinstance(item, PreparedCase) else item()
        prep_s = time.perf_counter() - t0
        sim = Simulation(case.cfg, case.mesh, case.params, case.levels, dev)
        cds, steps, conv = [], 0, False
        while steps < max_steps:
            sim.run(check_every, diag_freq=check_every)
            steps += check_every
            fr, _ = sim.forces()
            cds.append(fr.Cd)
            conv = steps >= min_steps and len(cds) > lag and abs(cds[-1] - cds[-1 - lag]) < tol
            if conv or not np.isfinite(fr.Cd):
                break
        torch.cuda.synchronize()
        took = time.perf_counter() - t0
        start = max(t_free, float(arrivals[k]))
        t_free = start + took
        results.append(Result(int(k), float(arrivals[k]), start, t_free, steps, cds[-1], conv,
                              0, cds, {}, prep_s))
        del sim
    return _summary(results, t_free, sum(r.finish_s - r.admit_s for r in results))
