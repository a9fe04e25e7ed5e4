"""The oracle's per-cell restatement run on the GPU (oracle/_build/
libolorc_gpu.so, built from ol_oracle_gpu.cu): the accuracy oracle in FP64 at
full benchmark sizes.

TEST INFRASTRUCTURE: imported only by tests/.  The kernel set here has the
interface of the CPU oracle's (stream_collide, bouzidi, thermal, copyto) over
torch CUDA tensors, so oracle.driver runs the reference's per-level step and
2:1 recursion on it unchanged:

    levels = gpu.init_levels(hosts, torch.float64, device=dev)
    driver.recursive_step(levels, s, 0, t, None, 0.0, u, dims, np.float64, k=gpu)

The oracle's own buffers (separate f_post, f_old / rho_old / vel_old copied
as copy_to_old! does) are kept, and all host arrays of a level (masks,
tables, q-map, boundary-cell lists) get device copies.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import types
from pathlib import Path

import numpy as np
import torch

from . import driver as odrv
from .oracle import StepParamsC, ThermalParamsC, _fill

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libolorc_gpu.so"
_lib = None


def build(force: bool = False) -> Path:
    srcs = [HERE / "ol_oracle_gpu.cu", HERE / "ol_oracle_cell.h", HERE / "Makefile"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        r = subprocess.run(["make", "-C", str(HERE), "gpu"] + (["-B"] if force else []),
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"GPU oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        for name in ("orcg_stream_collide_f32", "orcg_stream_collide_f64", "orcg_bouzidi_f32",
                     "orcg_bouzidi_f64", "orcg_thermal_f32", "orcg_thermal_f64"):
            getattr(_lib, name).restype = C.c_int
    return _lib


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"GPU oracle {what}: CUDA error {rc}")


def _suffix(dtype) -> str:
    return "f32" if dtype in (np.float32, torch.float32) else "f64"


def copyto(dst: torch.Tensor, src: torch.Tensor) -> None:
    dst.copy_(src)


def stream_collide(lv: dict, pv: dict | None, params: dict, dtype=np.float64) -> None:
    sp = _fill(StepParamsC, params)
    pv = pv or {}
    dims = pv.get("dim", (0, 0, 0))
    fn = getattr(lib(), "orcg_stream_collide_" + _suffix(dtype))
    _check(fn(_p(lv["f_out"]), _p(lv["f_in"]), _p(lv.get("f_post")), _p(lv["rho"]),
              _p(lv["vel_out"]), _p(lv["vel_in"]), _p(lv["obstacle"]), _p(lv["sponge"]),
              _p(lv.get("wall_dist")), _p(lv["neighbor_table"]), _p(lv["map_x"]), _p(lv["map_y"]),
              _p(lv["map_z"]), C.c_int32(lv["n_blocks"]), _p(pv.get("f")), _p(pv.get("rho")),
              _p(pv.get("vel")), _p(pv.get("f_old")), _p(pv.get("rho_old")),
              _p(pv.get("vel_old")), _p(pv.get("block_ptr")), C.c_int32(dims[0]),
              C.c_int32(dims[1]), C.c_int32(dims[2]), C.c_int32(pv.get("n_blocks", 0)),
              C.byref(sp), _stream()), "stream_collide")


def bouzidi(f_out, f_post, q_map, cell_block, cx, cy, cz, neighbor_table, n_blocks, q_min,
            dtype=np.float64) -> None:
    fn = getattr(lib(), "orcg_bouzidi_" + _suffix(dtype))
    _check(fn(_p(f_out), _p(f_post), _p(q_map), _p(cell_block), _p(cx), _p(cy), _p(cz),
              C.c_int32(int(cell_block.numel())), _p(neighbor_table), C.c_int32(n_blocks),
              C.c_float(q_min), _stream()), "bouzidi")


def thermal(tv: dict, pv: dict | None, params: dict, dtype=np.float64) -> None:
    tp = _fill(ThermalParamsC, params)
    pv = pv or {}
    dims = pv.get("dim", (0, 0, 0))
    fn = getattr(lib(), "orcg_thermal_" + _suffix(dtype))
    _check(fn(_p(tv["g_out"]), _p(tv["g_in"]), _p(tv.get("g_post")), _p(tv["T"]), _p(tv["vel"]),
              _p(tv["obstacle"]), _p(tv["sponge"]), _p(tv["neighbor_table"]), _p(tv["map_x"]),
              _p(tv["map_y"]), _p(tv["map_z"]), C.c_int32(tv["n_blocks"]), _p(pv.get("g")),
              _p(pv.get("T")), _p(pv.get("vel")), _p(pv.get("g_old")), _p(pv.get("T_old")),
              _p(pv.get("vel_old")), _p(pv.get("block_ptr")), C.c_int32(dims[0]),
              C.c_int32(dims[1]), C.c_int32(dims[2]), C.c_int32(pv.get("n_blocks", 0)),
              C.byref(tp), _stream()), "thermal")


def restrict(*args, **kw) -> None:
    raise NotImplementedError("fine-to-coarse restriction has no GPU oracle; use the CPU oracle")


_ARRAYS = ("obstacle", "sponge", "wall_dist", "neighbor_table", "map_x", "map_y", "map_z",
           "block_ptr", "cell_block", "cell_x", "cell_y", "cell_z")


def device_host(h, device) -> types.SimpleNamespace:
    """A level's host description with every array on the device."""
    d = types.SimpleNamespace(level_id=h.level_id, tau=h.tau, tau_g=h.tau_g, bouzidi=h.bouzidi,
                              n_boundary=h.n_boundary, n_blocks=h.n_blocks, grid_dim=h.grid_dim)
    for name in _ARRAYS:
        a = getattr(h, name, None)
        setattr(d, name, None if a is None else
                torch.from_numpy(np.ascontiguousarray(a)).to(device))
    q = getattr(h, "q_map", None)
    d.q_map = None if q is None else torch.from_numpy(
        np.ascontiguousarray(q).view(np.int16)).to(device)
    return d


def init_levels(hosts, dtype=torch.float64, ddf=False, t_init=1.0, device=None):
    """main.jl:113-173 initial state (f = w_k, rho = 1, u = 0) on the device."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    npd = np.float32 if dtype == torch.float32 else np.float64
    w = torch.from_numpy(odrv._w(npd)).to(dev)
    out = []
    for h in hosts:
        S = 512 * h.n_blocks
        f = w[:, None].expand(27, S).reshape(-1).clone()

        def z(n):
            return torch.zeros(n, dtype=dtype, device=dev)

        lv = odrv.OLevel(device_host(h, dev), f.clone(), f.clone(), torch.zeros_like(f), f.clone(),
                         torch.ones(S, dtype=dtype, device=dev),
                         torch.ones(S, dtype=dtype, device=dev), z(3 * S), z(3 * S), z(3 * S))
        if ddf:
            g = f * t_init
            lv.g, lv.g_temp, lv.g_post, lv.g_old = g.clone(), g.clone(), g.clone(), g.clone()
            lv.T = torch.full((S,), t_init, dtype=dtype, device=dev)
            lv.T_old = lv.T.clone()
        out.append(lv)
    return out
