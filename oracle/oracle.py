"""ctypes wrapper of the CPU oracle (oracle/_build/libolorc.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The oracle restates the reference's Julia
algorithm for the LBM time step, its host preprocessing, the surface forces
and the merged flow output (see the headers of ol_oracle_kernels.cpp and
ol_oracle_domain.cpp, and merged_output below); parity against the
reference itself is unpinned because the reference ships no tests, golden
vectors or fixtures and its Julia toolchain is absent here.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libolorc.so"

_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off, OpenMP)."""
    srcs = [HERE / "ol_oracle_kernels.cpp", HERE / "ol_oracle_domain.cpp",
            HERE / "ol_oracle_cell.h", HERE / "Makefile"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        r = subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


copyto = np.copyto


class StepParamsC(C.Structure):
    from openludwig_b200._native import STEP_FIELDS as _f
    _fields_ = _f


class ThermalParamsC(C.Structure):
    from openludwig_b200._native import THERMAL_FIELDS as _f
    _fields_ = _f


def _fill(struct_cls, d: dict):
    s = struct_cls()
    for name, _ in struct_cls._fields_:
        if name in d:
            setattr(s, name, d[name])
    return s


def stream_collide(lv: dict, pv: dict | None, params: dict, dtype=np.float32) -> None:
    """One level sub-step in place on host arrays (see ol_stream_collide).
    lv keys: f_out f_in f_post rho vel_out vel_in obstacle sponge wall_dist
    neighbor_table map_x map_y map_z n_blocks; pv keys: f rho vel f_old
    rho_old vel_old block_ptr dim n_blocks (or None on level 1)."""
    fn = lib().orc_stream_collide_f32 if dtype == np.float32 else lib().orc_stream_collide_f64
    sp = _fill(StepParamsC, params)
    pv = pv or {}
    dims = pv.get("dim", (0, 0, 0))
    fn.restype = None
    fn(_p(lv["f_out"]), _p(lv["f_in"]), _p(lv.get("f_post")), _p(lv["rho"]), _p(lv["vel_out"]),
       _p(lv["vel_in"]), _p(lv["obstacle"]), _p(lv["sponge"]), _p(lv.get("wall_dist")),
       _p(lv["neighbor_table"]), _p(lv["map_x"]), _p(lv["map_y"]), _p(lv["map_z"]),
       C.c_int32(lv["n_blocks"]), _p(pv.get("f")), _p(pv.get("rho")), _p(pv.get("vel")),
       _p(pv.get("f_old")), _p(pv.get("rho_old")), _p(pv.get("vel_old")),
       _p(pv.get("block_ptr")), C.c_int32(dims[0]), C.c_int32(dims[1]), C.c_int32(dims[2]),
       C.c_int32(pv.get("n_blocks", 0)), C.byref(sp))


def bouzidi(f_out, f_post, q_map, cell_block, cx, cy, cz, neighbor_table, n_blocks, q_min,
            dtype=np.float32) -> None:
    fn = lib().orc_bouzidi_f32 if dtype == np.float32 else lib().orc_bouzidi_f64
    fn.restype = None
    fn(_p(f_out), _p(f_post), _p(q_map), _p(cell_block), _p(cx), _p(cy), _p(cz),
       C.c_int32(len(cell_block)), _p(neighbor_table), C.c_int32(n_blocks), C.c_float(q_min))


def restrict(f_f, obs_f, mx, my, mz, n_f, f_c, rho_c, vel_c, obs_c, block_ptr, dims, n_c,
             tau_f, tau_c, compressible, dtype=np.float32) -> None:
    """Fine-to-coarse restriction in place on the coarse arrays (ol_restrict)."""
    fn = lib().orc_restrict_f32 if dtype == np.float32 else lib().orc_restrict_f64
    fn.restype = None
    fn(_p(f_f), _p(obs_f), _p(mx), _p(my), _p(mz), C.c_int32(n_f), _p(f_c), _p(rho_c), _p(vel_c),
       _p(obs_c), _p(block_ptr), C.c_int32(dims[0]), C.c_int32(dims[1]), C.c_int32(dims[2]),
       C.c_int32(n_c), C.c_float(tau_f), C.c_float(tau_c), C.c_int32(int(compressible)))


def thermal(tv: dict, pv: dict | None, params: dict, dtype=np.float32) -> None:
    fn = lib().orc_thermal_f32 if dtype == np.float32 else lib().orc_thermal_f64
    tp = _fill(ThermalParamsC, params)
    pv = pv or {}
    dims = pv.get("dim", (0, 0, 0))
    fn.restype = None
    fn(_p(tv["g_out"]), _p(tv["g_in"]), _p(tv.get("g_post")), _p(tv["T"]), _p(tv["vel"]),
       _p(tv["obstacle"]), _p(tv["sponge"]), _p(tv["neighbor_table"]), _p(tv["map_x"]),
       _p(tv["map_y"]), _p(tv["map_z"]), C.c_int32(tv["n_blocks"]), _p(pv.get("g")),
       _p(pv.get("T")), _p(pv.get("vel")), _p(pv.get("g_old")), _p(pv.get("T_old")),
       _p(pv.get("vel_old")), _p(pv.get("block_ptr")), C.c_int32(dims[0]), C.c_int32(dims[1]),
       C.c_int32(dims[2]), C.c_int32(pv.get("n_blocks", 0)), C.byref(tp))


# ------------------------------------------------------------------ domain

def level_blocks(lvl, tris, dx, offset, dims, prev=None, prev_bs_phys=0.0, wake_box=None,
                 margin_layers=2) -> np.ndarray:
    t = np.ascontiguousarray(tris, dtype=np.float64)
    off = np.ascontiguousarray(offset, dtype=np.float64)
    pv = np.ascontiguousarray(prev if prev is not None else np.zeros((0, 3)), dtype=np.int32)
    wb = np.ascontiguousarray(wake_box if wake_box is not None else np.zeros(6), dtype=np.float64)
    cap = int(np.prod(dims)) if lvl == 1 else 1 << 20
    while True:
        out = np.zeros((cap, 3), dtype=np.int32)
        fn = lib().orc_level_blocks
        fn.restype = C.c_int
        n = fn(C.c_int(lvl), _p(t), C.c_int(t.shape[0]), C.c_double(dx), _p(off), C.c_int(dims[0]),
               C.c_int(dims[1]), C.c_int(dims[2]), _p(pv), C.c_int(pv.shape[0]),
               C.c_double(prev_bs_phys), C.c_int(1 if wake_box is not None else 0), _p(wb),
               C.c_int(margin_layers), _p(out), C.c_int(cap))
        if n >= 0:
            return out[:n].copy()
        cap = -n


def neighbor_table(coords, dims) -> np.ndarray:
    c = np.ascontiguousarray(coords, dtype=np.int32)
    out = np.zeros(27 * c.shape[0], dtype=np.int32)
    lib().orc_neighbor_table(_p(c), C.c_int(c.shape[0]), C.c_int(dims[0]), C.c_int(dims[1]),
                             C.c_int(dims[2]), _p(out))
    return out


def voxelize(coords, tris, dx, offset) -> np.ndarray:
    c = np.ascontiguousarray(coords, dtype=np.int32)
    t = np.ascontiguousarray(tris, dtype=np.float64)
    off = np.ascontiguousarray(offset, dtype=np.float64)
    out = np.zeros(c.shape[0] * 512, dtype=np.uint8)
    lib().orc_voxelize(_p(c), C.c_int(c.shape[0]), _p(t), C.c_int(t.shape[0]), C.c_double(dx),
                       _p(off), _p(out))
    return out


def flood_fill(coords, dims, obstacle) -> np.ndarray:
    c = np.ascontiguousarray(coords, dtype=np.int32)
    o = np.ascontiguousarray(obstacle, dtype=np.uint8).copy()
    lib().orc_flood_fill(_p(c), C.c_int(c.shape[0]), C.c_int(dims[0]), C.c_int(dims[1]),
                         C.c_int(dims[2]), _p(o))
    return o


def sponge(coords, dx, domain_size, thickness, symmetric) -> np.ndarray:
    c = np.ascontiguousarray(coords, dtype=np.int32)
    out = np.zeros(c.shape[0] * 512, dtype=np.float32)
    lib().orc_sponge(_p(c), C.c_int(c.shape[0]), C.c_double(dx), C.c_double(domain_size[0]),
                     C.c_double(domain_size[1]), C.c_double(domain_size[2]),
                     C.c_float(thickness), C.c_int(1 if symmetric else 0), _p(out))
    return out


def wall_dist(coords, obstacle, dx) -> np.ndarray:
    c = np.ascontiguousarray(coords, dtype=np.int32)
    o = np.ascontiguousarray(obstacle, dtype=np.uint8)
    out = np.full(c.shape[0] * 512, 100.0, dtype=np.float32)
    lib().orc_wall_dist(_p(c), C.c_int(c.shape[0]), _p(o), C.c_double(dx), _p(out))
    return out


def bouzidi_qmap(coords, tris, dx, offset):
    c = np.ascontiguousarray(coords, dtype=np.int32)
    t = np.ascontiguousarray(tris, dtype=np.float64)
    off = np.ascontiguousarray(offset, dtype=np.float64)
    n = c.shape[0]
    q = np.zeros(n * 512 * 27, dtype=np.uint16)
    tri = np.zeros(n * 512 * 27, dtype=np.int32)
    cap = n * 512
    cells = np.zeros((max(cap, 1), 4), dtype=np.int32)
    fn = lib().orc_bouzidi_qmap
    fn.restype = C.c_int
    cnt = fn(_p(c), C.c_int(n), _p(t), C.c_int(t.shape[0]), C.c_double(dx), _p(off), _p(q),
             _p(tri), _p(cells), C.c_int(cap))
    return q, tri, cells[:cnt].copy()


class ForceParamsC(C.Structure):
    from openludwig_b200._native import ForceParams as _F
    _fields_ = _F._fields_


def surface_forces(mesh_arrays, rho, vel, obstacle, block_ptr, n_blocks, fp_struct):
    """Per-triangle (p, tau_x, tau_y, tau_z) maps and the nine force/moment sums.
    mesh_arrays: float32 [7, n] (cx cy cz nx ny nz area)."""
    m = np.ascontiguousarray(mesh_arrays, dtype=np.float32)
    n = m.shape[1]
    maps = np.zeros((4, n), np.float32)
    out = np.zeros(9, np.float64)
    fp = ForceParamsC()
    C.memmove(C.byref(fp), C.byref(fp_struct), C.sizeof(fp))
    lib().orc_surface_forces(*[_p(m[i]) for i in range(7)], C.c_int32(n), _p(rho), _p(vel),
                             _p(obstacle), _p(block_ptr), C.c_int32(n_blocks), C.byref(fp),
                             _p(maps[0]), _p(maps[1]), _p(maps[2]), _p(maps[3]), _p(out))
    return out, maps


def surface_net_forces(mesh_arrays, rho, vel, obstacle, block_ptr, n_blocks, fp_struct,
                       closed_body: bool):
    """Two-sided per-triangle net forces: returns maps [8, n] (p+, tau+ xyz,
    p-, tau- xyz) and net [3, n] (Fx, Fy, Fz)."""
    m = np.ascontiguousarray(mesh_arrays, dtype=np.float32)
    n = m.shape[1]
    maps = np.zeros((8, n), np.float32)
    net = np.zeros((3, n), np.float32)
    fp = ForceParamsC()
    C.memmove(C.byref(fp), C.byref(fp_struct), C.sizeof(fp))
    lib().orc_surface_net_forces(*[_p(m[i]) for i in range(7)], C.c_int32(n), _p(rho), _p(vel),
                                 _p(obstacle), _p(block_ptr), C.c_int32(n_blocks), C.byref(fp),
                                 C.c_int32(1 if closed_body else 0), _p(maps), _p(net))
    return maps, net


def merged_output(levels: list, t_step: int) -> dict:
    """export_merged_mesh_sync (io_vtk.jl:6-129) restated with numpy loops
    over blocks: levels = [dict(coords [n,3] 1-based, rho, vel, vel_temp,
    obstacle, temperature or None, dx, level_id)], all flat Float32 / UInt8
    host arrays in the reference layout.  Returns the arrays the reference
    hands to vtk_grid (points [P,3], rho, vel [C,3], vel_mag, obstacle, level,
    temperature when any level has one)."""
    bs = 8
    valid = []
    for lvl, L in enumerate(levels):                                 # io_vtk.jl:19-38
        nxt = None
        if lvl + 1 < len(levels):
            nxt = {tuple(int(v) for v in c) for c in levels[lvl + 1]["coords"]}
        for b, (bx, by, bz) in enumerate(L["coords"]):
            bx, by, bz = int(bx), int(by), int(bz)
            export = True
            if nxt is not None:
                children = 0
                for dbz in (0, 1):
                    for dby in (0, 1):
                        for dbx in (0, 1):
                            if (2 * bx - 1 + dbx, 2 * by - 1 + dby, 2 * bz - 1 + dbz) in nxt:
                                children += 1
                export = children != 8
            if export:
                valid.append((lvl, b, bx, by, bz))
    n = len(valid)
    ddf = any(L.get("temperature") is not None for L in levels)
    pts = np.empty((n * 729, 3), np.float32)
    rho = np.empty(n * 512, np.float32)
    vel = np.empty((n * 512, 3), np.float32)
    obs = np.empty(n * 512, np.uint8)
    lev = np.empty(n * 512, np.int32)
    temp = np.zeros(n * 512, np.float32) if ddf else None
    px, py, pz = np.meshgrid(np.arange(9), np.arange(9), np.arange(9), indexing="ij")
    px, py, pz = px.T.reshape(-1), py.T.reshape(-1), pz.T.reshape(-1)   # x fastest
    for i, (lvl, b, bx, by, bz) in enumerate(valid):                 # io_vtk.jl:68-107
        L = levels[lvl]
        dx = np.float32(L["dx"])
        S = L["rho"].shape[0]
        v = L["vel_temp"] if t_step % 2 == 0 else L["vel"]
        o = np.float32((bx - 1) * 8), np.float32((by - 1) * 8), np.float32((bz - 1) * 8)
        sl = slice(i * 729, (i + 1) * 729)
        pts[sl, 0] = (o[0] + px.astype(np.float32)) * dx
        pts[sl, 1] = (o[1] + py.astype(np.float32)) * dx
        pts[sl, 2] = (o[2] + pz.astype(np.float32)) * dx
        c = slice(i * 512, (i + 1) * 512)
        src = slice(b * 512, (b + 1) * 512)
        rho[c] = L["rho"][src]
        vel[c, 0] = v[src]
        vel[c, 1] = v[S + b * 512:S + (b + 1) * 512]
        vel[c, 2] = v[2 * S + b * 512:2 * S + (b + 1) * 512]
        obs[c] = (L["obstacle"][src] != 0).astype(np.uint8)
        lev[c] = L["level_id"]
        if ddf and L.get("temperature") is not None:
            temp[c] = L["temperature"][src]
    for a in (rho, vel, temp):                                       # io_vtk.jl:111-115
        if a is not None:
            a[~np.isfinite(a)] = 0.0
    vmag = np.sqrt(vel[:, 0] * vel[:, 0] + vel[:, 1] * vel[:, 1] + vel[:, 2] * vel[:, 2])
    out = dict(points=pts, rho=rho, vel=vel, vel_mag=vmag, obstacle=obs, level=lev)
    if ddf:
        out["temperature"] = temp
    return out


class ScaleInC(C.Structure):
    _fields_ = [("mesh_min", C.c_double * 3), ("mesh_max", C.c_double * 3),
                ("ref_length_cfg", C.c_double), ("ref_dim", C.c_int32),
                ("ref_chord_cfg", C.c_double), ("ref_area_cfg", C.c_double),
                ("symmetric", C.c_int32), ("moment_center", C.c_double * 3),
                ("u_phys", C.c_double), ("nu_phys", C.c_double), ("rho_phys", C.c_double),
                ("surface_resolution", C.c_int32), ("u_lattice", C.c_float),
                ("tau_min", C.c_float), ("upstream", C.c_double), ("downstream", C.c_double),
                ("lateral", C.c_double), ("height", C.c_double), ("block_size", C.c_int32),
                ("min_coarse_blocks", C.c_int32), ("num_levels_cfg", C.c_int32),
                ("auto_levels", C.c_int32), ("max_levels", C.c_int32),
                ("ddf_enabled", C.c_int32), ("prandtl", C.c_double)]


class ScaleOutC(C.Structure):
    _fields_ = [("num_levels", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
                ("nz", C.c_int32), ("bx", C.c_int32), ("by", C.c_int32), ("bz", C.c_int32),
                ("ref_length", C.c_double), ("ref_chord", C.c_double), ("ref_area", C.c_double),
                ("re", C.c_double), ("tau_fine", C.c_double), ("domain", C.c_double * 3),
                ("offset", C.c_double * 3), ("moment_center", C.c_double * 3),
                ("dx_fine", C.c_double), ("dx_coarse", C.c_double), ("dx_levels", C.c_double * 16),
                ("length_scale", C.c_double), ("velocity_scale", C.c_double),
                ("time_scale", C.c_double), ("nu_lattice", C.c_double),
                ("force_scale", C.c_double), ("tau_levels", C.c_float * 16),
                ("tau_g_fine", C.c_double), ("tau_g_levels", C.c_float * 16)]


def domain_scaling(cfg, mesh_min, mesh_max) -> dict:
    """compute_domain_from_mesh (physics_scaling.jl:83-191) from a CaseConfig
    and the mesh bounds; returns the scaled quantities as a dict."""
    s = ScaleInC()
    s.mesh_min[:] = [float(v) for v in mesh_min]
    s.mesh_max[:] = [float(v) for v in mesh_max]
    s.ref_length_cfg = cfg.reference_length_for_meshing
    s.ref_dim = {"x": 0, "y": 1, "z": 2}.get(cfg.reference_dimension, 3)
    s.ref_chord_cfg, s.ref_area_cfg = cfg.reference_chord_config, cfg.reference_area_config
    s.symmetric = int(bool(cfg.symmetric_analysis))
    s.moment_center[:] = [float(v) for v in cfg.moment_center]
    s.u_phys, s.nu_phys = cfg.flow_velocity, cfg.fluid_kinematic_viscosity
    s.rho_phys = cfg.fluid_density
    s.surface_resolution = cfg.surface_resolution
    s.u_lattice, s.tau_min = cfg.u_target, cfg.tau_min
    s.upstream, s.downstream = cfg.domain_upstream, cfg.domain_downstream
    s.lateral, s.height = cfg.domain_lateral, cfg.domain_height
    s.block_size, s.min_coarse_blocks = cfg.block_size, cfg.min_coarse_blocks
    s.num_levels_cfg, s.auto_levels = cfg.num_levels_config, int(bool(cfg.auto_levels))
    s.max_levels, s.ddf_enabled = cfg.max_levels, int(bool(cfg.ddf_enabled))
    s.prandtl = cfg.ddf_prandtl
    o = ScaleOutC()
    fn = lib().orc_domain_scaling
    fn.restype = C.c_int
    if fn(C.byref(s), C.byref(o)) != 0:
        raise ValueError("level count outside 1..16")
    nl = o.num_levels
    return dict(num_levels=nl, nx_coarse=o.nx, ny_coarse=o.ny, nz_coarse=o.nz, bx_max=o.bx,
                by_max=o.by, bz_max=o.bz, reference_length=o.ref_length,
                reference_chord=o.ref_chord, reference_area=o.ref_area, re_number=o.re,
                tau_fine=o.tau_fine, domain_size=tuple(o.domain), mesh_offset=tuple(o.offset),
                moment_center=tuple(o.moment_center), dx_fine=o.dx_fine, dx_coarse=o.dx_coarse,
                dx_levels=list(o.dx_levels[:nl]), length_scale=o.length_scale,
                velocity_scale=o.velocity_scale, time_scale=o.time_scale,
                nu_lattice=o.nu_lattice, force_scale=o.force_scale,
                tau_levels=[float(v) for v in o.tau_levels[:nl]], tau_g_fine=o.tau_g_fine,
                tau_g_levels=[float(v) for v in o.tau_g_levels[:nl]] if cfg.ddf_enabled else [])


def double_to_half_bits(x: float) -> int:
    fn = lib().orc_double_to_half
    fn.restype = C.c_uint16
    return int(fn(C.c_double(x)))


def gradient_noise(gx: int, gy: int, gz: int, seed: int) -> float:
    fn = lib().orc_gradient_noise
    fn.restype = C.c_float
    return float(fn(C.c_int32(gx), C.c_int32(gy), C.c_int32(gz), C.c_int32(seed)))


def half_to_float(h: int) -> float:
    fn = lib().orc_half_to_float
    fn.restype = C.c_float
    return float(fn(C.c_uint16(h)))


os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
