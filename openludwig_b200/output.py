"""Merged flow output: export_merged_mesh_sync (io_vtk.jl:6-129).

The reference copies every level's rho, velocity, obstacle (and temperature)
to the host, picks the blocks that are not covered by all 8 children, gathers
their cells into the arrays of one VTK unstructured grid (9^3 corner points
and one VOXEL cell per lattice cell), replaces NaN and +-Inf by 0 and writes
a compressed .vtu.  Here the selection is host topology (static per case),
the gather runs on the device (ol_pack_merged_fields, one launch on the
solver's stream), the packed arrays come back with one asynchronous copy
each into pinned memory, and write_vtu writes them (raw appended binary).

  export_block_lists(hosts)         -> per-level 0-based ids of the exported blocks
  MergedOutput(levels).pack(t_step) -> enqueue the gather + copies, returns a Snapshot
  Snapshot.wait()                   -> dict of numpy arrays
  write_vtu(path, arrays)           -> flow_%06d.vtu as the reference names it
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np
import torch

from . import _native as N

BS = 8
POINTS_PER_BLOCK = (BS + 1) ** 3
VTK_VOXEL = 11


def export_block_lists(hosts) -> list[np.ndarray]:
    """io_vtk.jl:10-38: a block of level l is exported unless all 8 of its
    children (2b-1 + {0,1} per axis, 1-based) exist on level l + 1; the
    finest level exports every block.  Order: block index within a level."""
    out = []
    for lvl, h in enumerate(hosts):
        coords = np.asarray(h.coords, dtype=np.int64)
        if lvl + 1 < len(hosts):
            child = {tuple(c) for c in np.asarray(hosts[lvl + 1].coords, dtype=np.int64)}
            keep = []
            for b, (bx, by, bz) in enumerate(coords):
                n = sum((2 * bx - 1 + dx, 2 * by - 1 + dy, 2 * bz - 1 + dz) in child
                        for dz in (0, 1) for dy in (0, 1) for dx in (0, 1))
                if n != 8:
                    keep.append(b)
            out.append(np.asarray(keep, dtype=np.int32))
        else:
            out.append(np.arange(h.n_blocks, dtype=np.int32))
    return out


class Snapshot:
    """Packed arrays on their way to pinned host memory."""

    def __init__(self, host: dict, event: torch.cuda.Event, t_step: int):
        self.host, self.event, self.t_step = host, event, t_step

    def ready(self) -> bool:
        return self.event.query()

    def wait(self) -> dict:
        self.event.synchronize()
        return {k: v.numpy() for k, v in self.host.items()}


class MergedOutput:
    """Device gather of the merged output of a list of solver.DeviceLevel.
    Buffers are allocated once; pack() may be called every output step."""

    FIELDS = ("points", "rho", "vel", "vel_mag", "obstacle", "level", "temperature")

    def __init__(self, levels, with_temperature: bool | None = None):
        self.levels = levels
        dev = levels[0].rho.device
        self.lists = [torch.from_numpy(np.append(l, -1).astype(np.int32)).to(dev)
                      for l in export_block_lists([lv.host for lv in levels])]
        self.n_export = [int(x.numel()) - 1 for x in self.lists]
        nb = sum(self.n_export)
        self.n_blocks = nb
        temp = (with_temperature if with_temperature is not None
                else any(lv.temperature is not None for lv in levels))
        shapes = {"points": (nb * POINTS_PER_BLOCK, 3), "rho": (nb * 512,), "vel": (nb * 512, 3),
                  "vel_mag": (nb * 512,), "obstacle": (nb * 512,), "level": (nb * 512,)}
        if temp:
            shapes["temperature"] = (nb * 512,)
        dtypes = {"obstacle": torch.uint8, "level": torch.int32}
        self.dev = {k: torch.empty(s, dtype=dtypes.get(k, torch.float32), device=dev)
                    for k, s in shapes.items()}
        self.host = [{k: torch.empty(s, dtype=dtypes.get(k, torch.float32), pin_memory=True)
                      for k, s in shapes.items()} for _ in range(2)]
        self.events = [None, None]
        self.turn = 0

    def pack(self, t_step: int, stream: torch.cuda.Stream | None = None) -> Snapshot:
        """Gather step t_step's state (vel_temp on even steps, vel on odd ones,
        io_vtk.jl:48) and start its copies; two snapshots may be in flight."""
        s = stream or torch.cuda.current_stream()
        lvs = (N.OutputLevel * len(self.levels))()
        for i, (lv, lst, n) in enumerate(zip(self.levels, self.lists, self.n_export)):
            vel = lv.vel_temp if t_step % 2 == 0 else lv.vel
            lvs[i] = N.OutputLevel(
                rho=lv.rho.data_ptr(), vel=vel.data_ptr(), obstacle=lv.obstacle.data_ptr(),
                temperature=lv.temperature.data_ptr() if lv.temperature is not None else None,
                map_x=lv.map_x.data_ptr(), map_y=lv.map_y.data_ptr(), map_z=lv.map_z.data_ptr(),
                blocks=lst.data_ptr(), n_export=n, n_blocks=lv.n_blocks,
                level_id=lv.host.level_id, dx=float(np.float32(lv.host.dx)))
        out = N.OutputFields(**{k: (self.dev[k].data_ptr() if k in self.dev else None)
                                for k in self.FIELDS})
        k = self.turn
        self.turn ^= 1
        if self.events[k] is not None:
            self.events[k].synchronize()   # the copy into this buffer has landed
        with torch.cuda.stream(s):
            N.call("ol_pack_merged_fields", lvs, N.i32(len(self.levels)), C.byref(out),
                   C.c_void_p(s.cuda_stream))
            for name, t in self.dev.items():
                self.host[k][name].copy_(t, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self.events[k] = ev
        return Snapshot(self.host[k], ev, t_step)


def voxel_connectivity(n_blocks: int) -> np.ndarray:
    """The 8 point ids of each cell, 0-based (io_vtk.jl:85-94), [n*512, 8] int64."""
    c = np.arange(512)
    x, y, z = c % BS, (c // BS) % BS, c // (BS * BS)
    base = x + (BS + 1) * y + (BS + 1) ** 2 * z
    sy, sz = BS + 1, (BS + 1) ** 2
    corner = np.array([0, 1, sy, sy + 1, sz, sz + 1, sz + sy, sz + sy + 1])
    one = base[:, None] + corner[None, :]
    blocks = np.arange(n_blocks, dtype=np.int64)[:, None, None] * POINTS_PER_BLOCK
    return (blocks + one[None]).reshape(-1, 8)


def write_vtu(path: str, arrays: dict) -> None:
    """An UnstructuredGrid .vtu of the packed arrays (raw appended binary,
    UInt64 block headers): points, VOXEL cells and the cell fields the
    reference writes (Density, Velocity, VelocityMagnitude, Obstacle, Level,
    Temperature)."""
    pts = np.ascontiguousarray(arrays["points"], dtype=np.float32).reshape(-1, 3)
    n_blocks = pts.shape[0] // POINTS_PER_BLOCK
    n_cells = n_blocks * 512
    conn = voxel_connectivity(n_blocks)
    blobs = [("Points", None, pts, "Float32", 3),
             ("connectivity", "Cells", conn.reshape(-1), "Int64", 1),
             ("offsets", "Cells", np.arange(8, 8 * n_cells + 1, 8, dtype=np.int64), "Int64", 1),
             ("types", "Cells", np.full(n_cells, VTK_VOXEL, dtype=np.uint8), "UInt8", 1)]
    names = [("Density", "rho", "Float32", 1), ("Velocity", "vel", "Float32", 3),
             ("VelocityMagnitude", "vel_mag", "Float32", 1), ("Obstacle", "obstacle", "UInt8", 1),
             ("Level", "level", "Int32", 1), ("Temperature", "temperature", "Float32", 1)]
    np_t = {"Float32": np.float32, "UInt8": np.uint8, "Int32": np.int32, "Int64": np.int64}
    for vtk_name, key, typ, nc in names:
        if key in arrays:
            blobs.append((vtk_name, "CellData", np.ascontiguousarray(arrays[key], np_t[typ]), typ, nc))
    offset = 0
    entries = []
    for name, section, data, typ, nc in blobs:
        entries.append((name, section, typ, nc, offset))
        offset += 8 + data.nbytes
    def tag(name, typ, nc, off):
        comp = f' NumberOfComponents="{nc}"' if nc > 1 else ""
        return (f'<DataArray type="{typ}" Name="{name}"{comp} format="appended" '
                f'offset="{off}"/>')
    xml = ['<?xml version="1.0"?>',
           '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
           'header_type="UInt64">', '<UnstructuredGrid>',
           f'<Piece NumberOfPoints="{pts.shape[0]}" NumberOfCells="{n_cells}">']
    for section in (None, "Cells", "CellData"):
        xml.append({None: "<Points>", "Cells": "<Cells>", "CellData": "<CellData>"}[section])
        xml += [tag(n, t, c, o) for n, s, t, c, o in entries if s == section]
        xml.append({None: "</Points>", "Cells": "</Cells>", "CellData": "</CellData>"}[section])
    xml += ["</Piece>", "</UnstructuredGrid>", '<AppendedData encoding="raw">']
    with open(path, "wb") as fh:
        fh.write(("\n".join(xml) + "\n_").encode())
        for _, _, data, _, _ in blobs:
            fh.write(struct.pack("<Q", data.nbytes))
            fh.write(data.tobytes())
        fh.write(b"\n</AppendedData>\n</VTKFile>\n")


def _bench(workload: str = "cube_3lvl", reps: int = 10) -> dict:
    """Time the device gather of one merged output of a benchmark workload
    (state after three coarse steps) against the reference's route: every
    level's full rho / vel / obstacle copied to the host, then the exported
    blocks gathered there (io_vtk.jl:46-107, here with numpy)."""
    import time
    from . import solver as S
    from .workloads import build_case
    cfg, mesh, p, hosts = build_case(workload)
    dev = torch.device("cuda", 0)
    levels = [S.upload_level(h, dev) for h in hosts]
    st = S.StepSettings.from_config(cfg, cfg.wall_model_enabled)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    for t in range(1, 4):
        S.recursive_step(levels, st, 0, t, None, 0.0, float(cfg.u_target), dims)
    torch.cuda.synchronize()
    mo = MergedOutput(levels)
    mo.pack(3).wait()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s = torch.cuda.current_stream()
    lvs = (N.OutputLevel * len(levels))()
    for i, (lv, lst, n) in enumerate(zip(levels, mo.lists, mo.n_export)):
        lvs[i] = N.OutputLevel(rho=lv.rho.data_ptr(), vel=lv.vel.data_ptr(),
                               obstacle=lv.obstacle.data_ptr(), temperature=None,
                               map_x=lv.map_x.data_ptr(), map_y=lv.map_y.data_ptr(),
                               map_z=lv.map_z.data_ptr(), blocks=lst.data_ptr(), n_export=n,
                               n_blocks=lv.n_blocks, level_id=lv.host.level_id,
                               dx=float(np.float32(lv.host.dx)))
    out = N.OutputFields(**{k: (mo.dev[k].data_ptr() if k in mo.dev else None)
                            for k in MergedOutput.FIELDS})
    lvs_ms = []
    for _ in range(reps):   # the gather kernel alone
        e0.record(s)
        N.call("ol_pack_merged_fields", lvs, N.i32(len(levels)), C.byref(out),
               C.c_void_p(s.cuda_stream))
        e1.record(s)
        torch.cuda.synchronize()
        lvs_ms.append(e0.elapsed_time(e1))
    t0 = time.perf_counter()
    for _ in range(reps):
        mo.pack(3).wait()
    dev_ms = (time.perf_counter() - t0) / reps * 1e3
    t0 = time.perf_counter()
    for _ in range(3):
        parts = []
        for lv, lst in zip(levels, export_block_lists(hosts)):
            r, v, o = lv.rho.cpu().numpy(), lv.vel.cpu().numpy(), lv.obstacle.cpu().numpy()
            sel = (lst[:, None] * 512 + np.arange(512)[None, :]).reshape(-1)
            S_ = r.shape[0]
            parts.append((r[sel], np.stack([v[sel], v[S_ + sel], v[2 * S_ + sel]], 1), o[sel]))
    host_ms = (time.perf_counter() - t0) / 3 * 1e3
    n_cells = mo.n_blocks * 512
    kernel_ms = float(np.median(lvs_ms))
    bytes_moved = n_cells * (17 + 4 + 12 + 4 + 1 + 4) + mo.n_blocks * POINTS_PER_BLOCK * 12
    return {"workload": workload, "exported_cells": n_cells, "kernel_ms": kernel_ms,
            "kernel_GBs": bytes_moved / kernel_ms / 1e6,
            "device_gather_and_copy_ms": dev_ms, "host_route_ms": host_ms}


if __name__ == "__main__":
    import json
    import sys
    print(json.dumps(_bench(*(sys.argv[1:2] or ["cube_3lvl"]))))
