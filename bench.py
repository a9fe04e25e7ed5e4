#!/usr/bin/env python
"""Benchmark of the LBM time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cube_3lvl|sphere_1lvl] [--storage f32|f16]

Workload (default): the three-level refined cube -- coarsest 160x80x80,
side 16/32/64 cells on levels 1..3, alpha = 10 deg, Re = 1e5, cumulant + WALE
(C_w = 0.5) + log-law wall model, Bouzidi walls on the finest level.  Synthetic
inputs: the geometry is generated; the state starts from the reference's
f = w_k.  A step is one coarse time step: the full recursive 2:1 sequence
(level 1 once, level 2 twice, level 3 four times), i.e.
sum_l cells_l * 2^(l-1) cell updates.

Reported:
  value       MLUPS (true cell updates / s, whole job) with the state resident
              in HBM; each coarse step replayed from a CUDA graph
  e2e         the same metric through the reference-facing C ABI, one
              ol_stream_collide / ol_bouzidi_apply_links call per level sub-step
              from the host driver, with the per-step diagnostic (FP64 flow
              statistics) read back to pinned host memory every step
  roofline    HBM roofline of the dominant kernel (finest-level stream-collide)
              from CUDA events around repeated launches of it
  mlups_reference_formula  the reference's own figure (main.jl:232): active
              cells of all levels once per coarse step / time, beside the
              sub-step-weighted value
  batched     the block pool on config 4 (48 seeded uneven cases in one pool):
              FP16-shifted and FP32 MLUPS, HBM roofline fraction at 108 / 216
              bytes per update (the drag error of FP16 storage against the
              FP64 oracle is asserted by tests/test_gpu_oracle64.py)
  served      continuous batching on a sample of the config-5 stream (the
              config-4 mix plus 10 % large cases, Poisson arrivals at 80 % of
              the measured capacity, 2000-step window, 160 GB budget), with
              case preparation inside each request's latency, against the same
              requests solved one at a time on the plain FP32 drop-in path
  cpu_baseline the CPU oracle (restatement of the reference's algorithm) on the
              host cores, over a bounded number of coarse steps
Multi-GPU: one independent replica per rank (the reference has no multi-GPU
path; cases shard by case), scaling "weak", value = sum over ranks / max time.
`--gpus N` without torchrun starts the N ranks itself (torch.distributed.run
on 127.0.0.1).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG = {"f32": 216.0, "f16": 108.0}  # algorithmic bytes per cell update (2 Q sizeof)


def peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle-reason samples taken DURING the timed region.

    NVML is polled from a thread every 10 ms (a read-only query), so that even
    a timed region of a few tens of milliseconds gets samples; `nvidia-smi
    -lms 200` is the fallback when NVML cannot be opened.  With `out_dir`
    the samples are also written to <out_dir>/clocks_rank<i>.csv."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, device=None, out_dir=None):
        self.index = index
        self.out_dir = out_dir
        self.device = device
        self.proc = None
        self.thread = None
        self.samples = []          # (sm_mhz, max_mhz, reason names)
        self.path = os.path.join(out_dir or tempfile.gettempdir(),
                                 f"clocks_rank{index}.csv" if out_dir else
                                 f"ol_clocks_{os.getpid()}_rank{index}.csv")

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        if self.device is not None:
            try:
                import torch
                uuid = str(torch.cuda.get_device_properties(self.device).uuid)
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(
                    uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h):
        bits = [(nv.nvmlClocksEventReasonHwSlowdown, "hw_slowdown"),
                (nv.nvmlClocksEventReasonHwThermalSlowdown, "hw_thermal_slowdown"),
                (nv.nvmlClocksEventReasonSwThermalSlowdown, "sw_thermal_slowdown"),
                (nv.nvmlClocksEventReasonSwPowerCap, "sw_power_cap")]
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_flag.is_set():
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((float(sm), float(mx), [n for b, n in bits if r & b]))
            self.stop_flag.wait(0.01)

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            import threading
            nv, h = self._nvml_handle()
            self.stop_flag = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            if self.out_dir:
                with open(self.path, "w") as fh:
                    fh.write("sm_mhz,max_sm_mhz,reasons\n")
                    for sm, mx, rs in self.samples:
                        fh.write(f"{sm:.0f},{mx:.0f},{'|'.join(rs)}\n")
            sm = [x[0] for x in self.samples]
            mx = [x[1] for x in self.samples]
            reasons = set(n for x in self.samples for n in x[2])
            source = "nvml"
        elif self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.fh.close()
            sm, mx, reasons = [], [], set()
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(self.NAMES, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            source = "nvidia-smi"
            if not self.out_dir:
                os.remove(self.path)
        else:
            sm, mx, reasons, source = [], [], set(), None
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": source}


def build_case(workload: str):
    from openludwig_b200 import workloads
    try:
        return workloads.build_case(workload)
    except KeyError:
        raise SystemExit(f"unknown workload {workload}")


def launches_per_coarse_step(levels, ddf: bool) -> int:
    """Kernels one coarse step launches through the drop-in path (after the
    first step built the ghost visit lists and Bouzidi links): per level
    sub-step one stream-collide and, with Bouzidi, a gather and a scatter;
    on a refined level one ghost pass per pair of sub-steps, plus one for the
    second sub-step when a block touches the domain boundary; the thermal
    DDF repeats all of it for the temperature populations."""
    total = 0
    for i, lv in enumerate(levels):
        n_sub = 1 << i
        per = n_sub + (2 * n_sub if lv.has_bouzidi and lv.bz_n_links > 0 else 0)
        if lv.ghost is not None:
            if lv.ghost2 is None:
                per += n_sub
            else:
                per += (n_sub // 2) * ((lv.ghost_list.numel() > 1) + (lv.edge_list.numel() > 1))
        total += per * (2 if ddf else 1)
    return total


def describe(workload, p, hosts, world: int = 1) -> dict:
    """The `config` of the JSON line, identical in both arms."""
    return {"workload": workload, "levels": len(hosts),
            "coarse_domain": [p.nx_coarse, p.ny_coarse, p.nz_coarse],
            "blocks_per_level": [h.n_blocks for h in hosts],
            "cells": int(sum(h.n_blocks * 512 for h in hosts)),
            "cell_updates_per_step": int(sum(h.n_blocks * 512 * (1 << i) for i, h in enumerate(hosts))),
            "boundary_cells": int(sum(h.n_boundary for h in hosts)),
            "l2_policy": "state larger than L2 (no flush needed)",
            "parallelism": f"replicas x{world}", "storage": "f32",
            "step": "one coarse step (recursive 2:1 sequence)"}


def relaunch_under_torchrun(gpus: int) -> None:
    """`--gpus N` run directly: start N local ranks through
    torch.distributed.run (rendezvous on 127.0.0.1) and exit with its status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={gpus}", "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    raise SystemExit(subprocess.call(cmd))


def launcher_selftest(a, rank: int, world: int) -> None:
    """The multi-rank plumbing without a GPU (gloo): barrier, a max over the
    ranks' elapsed times, one line from rank 0 with n_gpus = world."""
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
    t = torch.tensor([0.5 + rank], dtype=torch.float64)
    if world > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        print(json.dumps({"metric": "MLUPS", "value": None, "n_gpus": world, "selftest": True,
                          "max_rank_ms": float(t.item()), "steps": a.steps,
                          "warmup": a.warmup}), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def time_cpu_baseline(cfg, p, hosts, budget_s: float = 15.0) -> dict:
    """Oracle (CPU restatement) coarse steps on all host cores within a time budget."""
    from oracle import driver as odrv
    from openludwig_b200.solver import StepSettings
    st = StepSettings.from_config(cfg, cfg.wall_model_enabled)
    s = odrv.settings_dict(st)
    lv = odrv.init_levels(hosts, ddf=bool(cfg.ddf_enabled))
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    upd = sum(h.n_blocks * 512 * (1 << i) for i, h in enumerate(hosts))
    t0 = time.perf_counter()
    n = 0
    while True:
        n += 1
        odrv.recursive_step(lv, s, 0, n, None, 0.0, float(cfg.u_target), dims, np.float32)
        if time.perf_counter() - t0 > budget_s or n >= 50:
            break
    dt = time.perf_counter() - t0
    return {"value": upd * n / dt / 1e6, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{n} coarse step(s) of the workload, FP32 oracle, OpenMP over blocks"}


def bench_batched(a, dev, local, peak_gbs, plain_value) -> dict:
    """Config 4: 48 seeded uneven cases in one pool, FP16-shifted and FP32."""
    from openludwig_b200 import native as NT
    from openludwig_b200.serve_bench import case_makers
    t0 = time.perf_counter()
    cases = [mk() for mk in case_makers(48, 1234, local)]
    prep_s = time.perf_counter() - t0
    upd = sum(c.cell_updates_per_step for c in cases)
    out = {"cases": len(cases), "seed": 1234, "cell_updates_per_step": int(upd),
           "prep_s": prep_s, "workload": "batch_mix 48 (sphere / cube / NACA0012 wing, "
           "16-48 finest cells, 1-3 levels, Re 1e3-1e6), cumulant + WALE"}
    for storage in ("f16", "f32"):
        probe = NT.Context(device=local, budget_bytes=64 << 20, storage=storage)
        need = sum(probe.footprint(c) for c in cases)
        probe.close()
        ctx = NT.Context(device=local, budget_bytes=int(need * 1.2) + (256 << 20), storage=storage)
        for c in cases:
            ctx.add_case(c)
        ctx.step(a.warmup)
        ctx.sync()
        k = max(4, a.steps)
        ms = ctx.step_timed(k)
        mlups = upd * k / (ms / 1e3) / 1e6
        gbs = mlups * 1e6 * B_ALG[storage] / 1e9
        out[storage] = {"MLUPS": mlups, "ms_per_step": ms / k, "roofline_achieved_GBs": gbs,
                        "roofline_frac": gbs / peak_gbs, "bytes_per_cell_update_alg": B_ALG[storage],
                        "launch": ctx.launch()}
        ctx.close()
    out["f16_over_f32_batched"] = out["f16"]["MLUPS"] / out["f32"]["MLUPS"]
    out["f16_over_f32_plain"] = out["f16"]["MLUPS"] / plain_value
    # the plain form on the same mix: each case alone through the FP32 drop-in
    # path (ol_stream_collide / Bouzidi calls per level sub-step, as the
    # reference's driver issues them), one case after another
    serial = serial_plain_mix(a, dev, cases)
    out["serial_f32_dropin_same_mix"] = serial
    out["f16_over_f32_serial_same_mix"] = out["f16"]["MLUPS"] / serial["MLUPS"]
    out["f32_over_f32_serial_same_mix"] = out["f32"]["MLUPS"] / serial["MLUPS"]
    return out


def serial_plain_mix(a, dev, cases) -> dict:
    """The cases one at a time on the plain FP32 drop-in path: per case its
    levels are uploaded, a.warmup coarse steps run, then max(4, a.steps)
    coarse steps are timed with CUDA events; MLUPS = all cases' cell updates
    over the sum of their times."""
    import torch

    from openludwig_b200 import solver as S
    k = max(4, a.steps)
    upd_total, ms_total = 0, 0.0
    stream = torch.cuda.Stream(device=dev)
    for c in cases:
        levels = [S.upload_level(h, dev, ddf=bool(c.cfg.ddf_enabled)) for h in c.levels]
        dims = (c.params.nx_coarse, c.params.ny_coarse, c.params.nz_coarse)
        u = float(c.cfg.u_target)
        with torch.cuda.stream(stream):
            t = 0
            for _ in range(a.warmup):
                t += 1
                S.recursive_step(levels, c.settings, 0, t, None, 0.0, u, dims)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                t += 1
                S.recursive_step(levels, c.settings, 0, t, None, 0.0, u, dims)
            e1.record(stream)
        torch.cuda.synchronize()
        ms_total += e0.elapsed_time(e1)
        upd_total += c.cell_updates_per_step * k
        del levels
    return {"MLUPS": upd_total / (ms_total / 1e3) / 1e6, "ms_total": ms_total, "coarse_steps": k,
            "cases": len(cases), "form": "FP32 drop-in path, one case at a time, eager C-ABI "
            "calls per level sub-step, CUDA events per case"}


def bench_served(a, dev, local, batched) -> dict:
    """A sample of config 5: the config-4 mix plus 10 % large cases, prepared
    on arrival; closed loop (all at t = 0) gives the capacity; then Poisson
    arrivals at 80 % of it; the same requests one at a time on the plain FP32
    drop-in path with the same arrivals."""
    import torch
    from openludwig_b200 import native as NT
    from openludwig_b200 import serving as SV
    from openludwig_b200.serve_bench import case_makers, summary
    n = a.served_requests
    rule = dict(check_every=200, window=2000, tol=1e-3, max_steps=10000)
    budget = min(160 << 30, int(torch.cuda.mem_get_info(dev)[0] * 0.85))
    makers = case_makers(n, 4321, local, large_frac=0.1)
    out = {"requests": n, "config5_requests": 500, "seed": 4321, "large_frac": 0.1,
           "rule": rule, "budget_bytes": budget, "storage": "f16",
           "note": (f"a {n}-request sample of the config-5 stream (500 requests do not fit the "
                    "bench's time); latency counts case preparation")}
    ctx = NT.Context(device=local, budget_bytes=budget, storage="f16")
    closed = SV.Server(ctx, **rule).run([SV.Request(i, 0.0, mk) for i, mk in enumerate(makers)])
    ctx.close()
    # the same closed loop with FP32 storage in the pool (the service's form
    # when storage precision is not traded for bytes)
    ctx = NT.Context(device=local, budget_bytes=budget, storage="f32")
    closed32 = SV.Server(ctx, **rule).run([SV.Request(i, 0.0, mk) for i, mk in enumerate(makers)])
    ctx.close()
    rate = 0.8 * closed["solves_per_hour"] / 3600.0
    arrivals = SV.poisson_arrivals(n, rate, seed=4321)
    ctx = NT.Context(device=local, budget_bytes=budget, storage="f16")
    opened = SV.Server(ctx, **rule).run([SV.Request(i, float(arrivals[i]), mk)
                                          for i, mk in enumerate(makers)])
    ctx.close()
    serial = SV.serial_baseline(makers, arrivals, **rule, device=dev)
    out["capacity_closed_loop"] = summary(closed)
    out["poisson_rate_per_s"] = rate
    out["served"] = summary(opened)
    out["serial_f32_dropin"] = summary(serial)
    out["solves_per_hour"] = opened["solves_per_hour"]
    out["p50_s"], out["p99_s"] = opened["p50_s"], opened["p99_s"]
    out["served_over_serial"] = opened["solves_per_hour"] / serial["solves_per_hour"]
    # capacities: closed-loop served rate against the serial form's rate when
    # it is never idle (its requests over the sum of its solve times)
    out["serial_capacity_solves_per_hour"] = n / serial["busy_s"] * 3600.0
    out["capacity_over_serial"] = closed["solves_per_hour"] / out["serial_capacity_solves_per_hour"]
    out["capacity_closed_loop_f32_storage"] = summary(closed32)
    out["capacity_f32_storage_over_serial"] = (closed32["solves_per_hour"] /
                                               out["serial_capacity_solves_per_hour"])
    return out


def pool_probe(a, local) -> None:
    """The block pool's coarse step of the workload alone, with a chosen
    storage and stream-collide kernel (ol_set_stream_collide_kernel): a.warmup
    steps, then a.steps timed by Context.step_timed (CUDA events)."""
    import torch

    from openludwig_b200 import _native as N
    from openludwig_b200 import build as olbuild
    olbuild.build()
    from openludwig_b200 import native as NT
    from openludwig_b200 import solver as S
    storage, kernel = a.pool_probe.split(":")
    choice = {"auto": 0, "block": 1, "ws": 2}[kernel]
    torch.cuda.set_device(local)
    cfg, mesh, p, hosts = build_case(a.workload)
    case = NT.PreparedCase(cfg, mesh, p, hosts, S.StepSettings.from_config(cfg, cfg.wall_model_enabled))
    upd = sum(h.n_blocks * 512 * (1 << i) for i, h in enumerate(hosts))
    N.call("ol_set_stream_collide_kernel", N.i32(choice), N.i32(0))
    try:
        ctx = NT.Context(device=local, budget_bytes=16 << 30, storage=storage)
        ctx.add_case(case)
        ctx.step(a.warmup)
        ctx.sync()
        k = max(1, a.steps)
        ms = ctx.step_timed(k)
        ctx.close()
    finally:
        N.call("ol_set_stream_collide_kernel", N.i32(0), N.i32(0))
    print(json.dumps({"workload": a.workload, "storage": storage, "kernel": kernel,
                      "coarse_steps": k, "MLUPS": upd * k / (ms / 1e3) / 1e6,
                      "ms_per_step": ms / k}), flush=True)


def kernel_times(a, local) -> None:
    """Per-kernel device time of the drop-in coarse step of the workload:
    a.warmup eager steps, then a.steps steps under the torch profiler
    (CUPTI activity records; caches warm, launches as the C-ABI path issues
    them).  One JSON line: microseconds per coarse step and share, per kernel."""
    import collections

    import torch
    from torch.profiler import ProfilerActivity, profile

    from openludwig_b200 import build as olbuild
    olbuild.build()
    from openludwig_b200 import solver as S
    cfg, mesh, p, hosts = build_case(a.workload)
    dev = torch.device("cuda", local)
    levels = [S.upload_level(h, dev, ddf=bool(cfg.ddf_enabled)) for h in hosts]
    st = S.StepSettings.from_config(cfg, cfg.wall_model_enabled)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    u = float(cfg.u_target)
    t = 0
    for _ in range(a.warmup):
        t += 1
        S.recursive_step(levels, st, 0, t, None, 0.0, u, dims)
    torch.cuda.synchronize()
    n = max(1, a.steps)
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(n):
            t += 1
            S.recursive_step(levels, st, 0, t, None, 0.0, u, dims)
        torch.cuda.synchronize()
    agg = collections.defaultdict(lambda: [0, 0.0])
    for ev in prof.events():
        if ev.device_type == torch.autograd.DeviceType.CUDA:
            agg[ev.name][0] += 1
            agg[ev.name][1] += ev.device_time_total
    total = sum(v[1] for v in agg.values())
    rows = [{"kernel": k, "launches_per_step": c / n, "us_per_step": us / n,
             "share": us / total if total else 0.0}
            for k, (c, us) in sorted(agg.items(), key=lambda kv: -kv[1][1])]
    print(json.dumps({"workload": a.workload, "coarse_steps": n, "warmup": a.warmup,
                      "us_per_step_total": total / n, "kernels": rows}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cube_3lvl")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clocks-dir", default=None,
                    help="also write the clock samples of the timed region to this directory")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched and served blocks")
    ap.add_argument("--served-requests", type=int, default=24,
                    help="requests of the served sample (config 5 asks for 500)")
    ap.add_argument("--launcher-selftest", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--pool-probe", default=None, metavar="STORAGE:KERNEL",
                    help="time only the block pool's coarse step of the workload with storage "
                         "f32|f16 and stream-collide kernel auto|block|ws (e.g. f16:ws), one JSON "
                         "line")
    ap.add_argument("--kernel-times", action="store_true",
                    help="print the device time of each kernel per coarse step of the drop-in "
                         "path (torch profiler, warm, eager launches) instead of the bench line")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)

    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_under_torchrun(a.gpus)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"bench.py: --gpus {a.gpus} but the launcher started {world} rank(s)")
    if a.launcher_selftest:
        launcher_selftest(a, rank, world)
        return

    if a.impl == "reference":
        if rank != 0:
            return
        cfg, mesh, p, hosts = build_case(a.workload)
        from oracle import oracle as orc
        orc.build()
        from oracle import driver as odrv
        from openludwig_b200.solver import StepSettings
        st = StepSettings.from_config(cfg, cfg.wall_model_enabled)
        s = odrv.settings_dict(st)
        lv = odrv.init_levels(hosts, ddf=bool(cfg.ddf_enabled))
        dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
        upd = sum(h.n_blocks * 512 * (1 << i) for i, h in enumerate(hosts))
        # each step: one coarse step of the workload on all host cores (about
        # 1-2 s); W warm-up steps, then exactly K timed steps
        for t in range(1, a.warmup + 1):
            odrv.recursive_step(lv, s, 0, t, None, 0.0, float(cfg.u_target), dims, np.float32)
        t0 = time.perf_counter()
        k = max(1, a.steps)
        for t in range(a.warmup + 1, a.warmup + 1 + k):
            odrv.recursive_step(lv, s, 0, t, None, 0.0, float(cfg.u_target), dims, np.float32)
        dt = time.perf_counter() - t0
        v = upd * k / dt / 1e6
        cells = sum(h.n_blocks * 512 for h in hosts)
        line = {"impl": "reference", "metric": "MLUPS", "value": v, "unit": "MLUPS",
                "n_gpus": a.gpus, "device": "cpu",
                "steps": k, "warmup": a.warmup, "ms_per_step": dt / k * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": describe(a.workload, p, hosts, a.gpus),
                "mlups_reference_formula": cells * k / dt / 1e6,
                "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                                 "sample": f"{k} coarse step(s) of the workload after {a.warmup} "
                                           "warm-up step(s), FP32 oracle, OpenMP over blocks"},
                "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if a.kernel_times:
        if rank == 0:
            kernel_times(a, local)
        return
    if a.pool_probe:
        if rank == 0:
            pool_probe(a, local)
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from openludwig_b200 import replicas
    from openludwig_b200 import build as olbuild
    olbuild.build()
    from openludwig_b200 import _native as N
    from openludwig_b200 import solver as S

    cfg, mesh, p, hosts = build_case(a.workload)
    dev = torch.device("cuda", local)
    levels = [S.upload_level(h, dev, ddf=bool(cfg.ddf_enabled)) for h in hosts]
    st = S.StepSettings.from_config(cfg, cfg.wall_model_enabled)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    u = float(cfg.u_target)
    upd = sum(h.n_blocks * 512 * (1 << i) for i, h in enumerate(hosts))
    # per level sub-step: [ghost pass] + stream-collide + Bouzidi gather/scatter,
    # and the same again for the thermal populations of a DDF case

    stream = torch.cuda.Stream(device=dev)
    state = {"t": 0}

    def coarse_step(t):
        S.recursive_step(levels, st, 0, t, None, 0.0, u, dims)

    # warm-up (also runs the first steps that set up the alternation)
    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            state["t"] += 1
            coarse_step(state["t"])
    torch.cuda.synchronize()

    launches_per_step = launches_per_coarse_step(levels, bool(cfg.ddf_enabled))

    # CUDA graph of two coarse steps (odd + even parity) for the device-resident run
    graph = torch.cuda.CUDAGraph()
    t_graph = state["t"] + 1 if (state["t"] + 1) % 2 == 1 else state["t"] + 2
    with torch.cuda.graph(graph, stream=stream):
        coarse_step(t_graph)
        coarse_step(t_graph + 1)
    torch.cuda.synchronize()
    # (the captured seeds differ from live t only in the inlet-noise seed, which
    # is inactive for this workload: inlet_turbulence_intensity = 0)
    pairs = max(1, (a.steps + 1) // 2)
    nsteps = 2 * pairs
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()

    clk = ClockSampler(local, dev, a.clocks_dir)
    clk.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(pairs):
            graph.replay()
        e1.record(stream)
    torch.cuda.synchronize()
    rate, dt_ms = replicas.job_rate(upd * nsteps, e0.elapsed_time(e1), dev)
    value = rate / 1e6

    # e2e: reference-facing C-ABI calls per level sub-step (step parameters
    # passed from the host each call) + a device-to-host read of the step's
    # FP64 flow statistics every step, into pinned memory, double-buffered:
    # a buffer is reused only after its copy (two steps earlier) has landed
    nb = hosts[0].n_blocks
    partials = torch.empty(int(N.lib().ol_flow_stats_scratch_doubles(nb)), dtype=torch.float64, device=dev)
    dev7 = torch.empty((2, 7), dtype=torch.float64, device=dev)
    host7 = torch.empty((2, 7), dtype=torch.float64, pin_memory=True)
    landed = [torch.cuda.Event(), torch.cuda.Event()]
    import ctypes as C
    ke = max(2, a.steps)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    with torch.cuda.stream(stream):
        ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ee0.record(stream)
        for i in range(ke):
            state["t"] += 1
            coarse_step(state["t"])
            lv0 = levels[0]
            vel = lv0.vel if state["t"] % 2 == 1 else lv0.vel_temp
            slot = i % 2
            if i >= 2:
                landed[slot].synchronize()
                assert host7[slot, 0].item() > 0       # the statistics of step i - 2 arrived
            N.call("ol_flow_stats_device", S._ptr(lv0.rho), S._ptr(vel), S._ptr(lv0.obstacle),
                   N.i32(nb), S._ptr(partials), S._ptr(dev7[slot]), C.c_void_p(stream.cuda_stream))
            host7[slot].copy_(dev7[slot], non_blocking=True)
            landed[slot].record(stream)
        ee1.record(stream)
    torch.cuda.synchronize()
    e2e_rate, e2e_ms = replicas.job_rate(upd * ke, ee0.elapsed_time(ee1), dev)
    e2e = e2e_rate / 1e6
    clocks = clk.stop()
    # host-to-device bytes of a coarse step: what each C-ABI call passes by
    # value (level view, parent view and step parameters per stream-collide;
    # six pointer / scalar arguments per Bouzidi call; the flow statistics call)
    sc_calls = sum(1 << i for i in range(len(levels)))
    bz_calls = sum(1 << i for i, lv in enumerate(levels) if lv.has_bouzidi)
    h2d_per_step = (sc_calls * (C.sizeof(N.LevelView) + C.sizeof(N.ParentView) +
                                C.sizeof(N.StepParams)) + bz_calls * 6 * 8 + 7 * 8)

    # roofline of the dominant kernel: the finest level's ol_stream_collide
    # calls, timed as the pair of sub-steps a refined level takes per parent
    # step (weight 0 with OL_GHOST_PAIR_FIRST, then 1/2 with _SECOND), per call
    fin = levels[-1]
    fdims = tuple(d * (1 << (len(levels) - 1)) for d in dims)
    ptau = levels[-2].tau if len(levels) > 1 else 0.5
    paired = len(levels) > 1 and fin.ghost2 is not None
    calls = []
    for tw, mode in ((0.0, N.OL_GHOST_PAIR_FIRST), (0.5, N.OL_GHOST_PAIR_SECOND)):
        sp = S.step_params(st, fin, ptau, len(levels) == 1, fdims, u, 1, tw, False)
        view = N.LevelView(f_out=S._ptr(fin.f_temp), f_in=S._ptr(fin.f), f_post=None,
                           rho=S._ptr(fin.rho), vel_out=S._ptr(fin.vel_temp),
                           vel_in=S._ptr(fin.vel), obstacle=S._ptr(fin.obstacle),
                           sponge=S._ptr(fin.sponge), wall_dist=S._ptr(fin.wall_dist),
                           neighbor_table=S._ptr(fin.neighbor_table), map_x=S._ptr(fin.map_x),
                           map_y=S._ptr(fin.map_y), map_z=S._ptr(fin.map_z),
                           n_blocks=fin.n_blocks)
        S._ghost_views(view, fin, fin.ghost, fin.ghost2,
                       mode if paired else N.OL_GHOST_UNPAIRED)
        calls.append((view, sp))
    pv = N.ParentView()
    if len(levels) > 1:
        par = levels[-2]
        d = par.host.grid_dim
        pv = N.ParentView(f=S._ptr(par.f), rho=S._ptr(par.rho), vel=S._ptr(par.vel),
                          f_old=S._ptr(par.f_temp), rho_old=S._ptr(par.rho_old),
                          vel_old=S._ptr(par.vel_temp), block_ptr=S._ptr(par.block_ptr),
                          dim_x=d[0], dim_y=d[1], dim_z=d[2], n_blocks=par.n_blocks)
    reps = 10
    sc = C.c_void_p(stream.cuda_stream)
    with torch.cuda.stream(stream):
        for _ in range(3):
            for view, sp in calls:
                N.call("ol_stream_collide", C.byref(view), C.byref(pv), C.byref(sp), sc)
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        for _ in range(reps):
            for view, sp in calls:
                N.call("ol_stream_collide", C.byref(view), C.byref(pv), C.byref(sp), sc)
        r1.record(stream)
    torch.cuda.synchronize()
    k_ms = r0.elapsed_time(r1) / (reps * len(calls))
    alg_bytes = fin.n_blocks * 512 * B_ALG["f32"]
    peak, peak_kind = peaks()
    achieved = alg_bytes / (k_ms / 1e3) / 1e9
    # DRAM bytes per call of the same finest-level launch, from the committed
    # ncu summary of this workload (null when there is none)
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"k_sc_ws_{a.workload}_level{len(levels)}.md")
    if os.path.exists(prof):
        with open(prof) as fh:
            m = re.search(r"^traffic_bytes_per_launch\s*=\s*(\d+)", fh.read(), re.M)
        traffic = int(m.group(1)) if m else None

    # native block-pool path: FP32 and FP16-shifted storage, one CUDA-graph
    # replay per coarse step, timed with events on the context stream
    from openludwig_b200 import native as NT
    case = NT.PreparedCase(cfg, mesh, p, hosts, st)
    native = {}
    for storage in ("f32", "f16"):
        ddf = bool(cfg.ddf_enabled)
        probe = NT.Context(device=local, budget_bytes=64 << 20, storage=storage, ddf=ddf)
        need = probe.footprint(case)
        probe.close()
        ctx = NT.Context(device=local, budget_bytes=int(need * 1.25) + (64 << 20), storage=storage,
                         ddf=ddf)
        cid = ctx.add_case(case)
        ctx.step(a.warmup)
        ctx.sync()
        n_rate, ms = replicas.job_rate(upd * nsteps, ctx.step_timed(nsteps), dev)
        native[storage] = {"MLUPS": n_rate / 1e6,
                           "ms_per_step": ms / nsteps,
                           "launches_per_step": ctx.stats()["launches"] // max(1, a.warmup + nsteps),
                           "bytes_per_cell_update_alg": B_ALG[storage]}
        ctx.close()
    native["f16_over_f32_plain"] = native["f16"]["MLUPS"] / value

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            from oracle import oracle as orc
            orc.build()
            cpu = time_cpu_baseline(cfg, p, hosts, budget_s=15.0)
        except Exception as ex:  # the baseline is reported, never the target
            cpu = {"value": None, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"unavailable: {ex}"}

    extras = {}
    if rank == 0 and world == 1 and not a.no_extras:
        peak_gbs = peaks()[0]
        extras["batched"] = bench_batched(a, dev, local, peak_gbs, value)
        extras["served"] = bench_served(a, dev, local, extras["batched"])

    if rank == 0:
        cells = sum(h.n_blocks * 512 for h in hosts)
        line = {
            "metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": nsteps,
            "warmup": a.warmup, "ms_per_step": dt_ms / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": describe(a.workload, p, hosts, world),
            "mlups_reference_formula": value * cells / upd,
            "e2e": {"value": e2e, "unit": "MLUPS", "h2d_bytes_per_step": h2d_per_step,
                    "d2h_bytes_per_step": 7 * 8},
            "gpu_launches": launches_per_step * nsteps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "ol_stream_collide on the finest level (k_ghost_fill + "
                                   "k_sc_ws), mean over the pair of sub-steps per "
                                   "parent step",
                         "peak_source": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": k_ms},
            "clocks": clocks,
            "native": native,
            **extras,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        del graph
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
