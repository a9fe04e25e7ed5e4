"""Oracle time-step driver: the reference's per-level step and 2:1 recursion
(timestep.jl:1-159, solver_control.jl:6-218, blocks.jl:241-252) restated over
host numpy arrays, calling the CPU oracle kernels.

TEST INFRASTRUCTURE (see oracle.py).  Unlike the product driver it keeps the
reference's separate f_post and f_old/rho_old/vel_old buffers and copies
them exactly as copy_to_old! does, so the two drivers are independent.
"""
from __future__ import annotations

import dataclasses as dc

import numpy as np

from . import oracle as orc


def _w(dtype):
    w = []
    for cz in (-1, 0, 1):
        for cy in (-1, 0, 1):
            for cx in (-1, 0, 1):
                d2 = cx * cx + cy * cy + cz * cz
                if dtype == np.float32:
                    w.append(np.float32(8) / np.float32(27) if d2 == 0 else np.float32(2) / np.float32(27)
                             if d2 == 1 else np.float32(1) / np.float32(54) if d2 == 2
                             else np.float32(1) / np.float32(216))
                else:
                    w.append(8 / 27 if d2 == 0 else 2 / 27 if d2 == 1 else 1 / 54 if d2 == 2 else 1 / 216)
    return np.array(w, dtype=dtype)


@dc.dataclass
class OLevel:
    host: object          # domain.HostLevel
    f: np.ndarray
    f_temp: np.ndarray
    f_post: np.ndarray
    f_old: np.ndarray
    rho: np.ndarray
    rho_old: np.ndarray
    vel: np.ndarray
    vel_temp: np.ndarray
    vel_old: np.ndarray
    g: np.ndarray | None = None
    g_temp: np.ndarray | None = None
    g_post: np.ndarray | None = None
    g_old: np.ndarray | None = None
    T: np.ndarray | None = None
    T_old: np.ndarray | None = None


def init_levels(hosts, dtype=np.float32, ddf=False, t_init=1.0):
    """main.jl:113-173 initial state."""
    out = []
    w = _w(dtype)
    for h in hosts:
        S = 512 * h.n_blocks
        f = np.repeat(w, S).astype(dtype)
        lv = OLevel(h, f.copy(), f.copy(), np.zeros_like(f), f.copy(),
                    np.ones(S, dtype), np.ones(S, dtype), np.zeros(3 * S, dtype),
                    np.zeros(3 * S, dtype), np.zeros(3 * S, dtype))
        if ddf:
            g = (np.repeat(w, S) * dtype(t_init)).astype(dtype)
            lv.g, lv.g_temp, lv.g_post, lv.g_old = g.copy(), g.copy(), g.copy(), g.copy()
            lv.T = np.full(S, t_init, dtype)
            lv.T_old = np.full(S, t_init, dtype)
        out.append(lv)
    return out


def _level_dict(lv: OLevel, f_out, f_in, vel_out, vel_in, store_post):
    h = lv.host
    return dict(f_out=f_out, f_in=f_in, f_post=lv.f_post if store_post else None, rho=lv.rho,
                vel_out=vel_out, vel_in=vel_in, obstacle=h.obstacle, sponge=h.sponge,
                wall_dist=h.wall_dist, neighbor_table=h.neighbor_table, map_x=h.map_x,
                map_y=h.map_y, map_z=h.map_z, n_blocks=h.n_blocks)


def perform_timestep(s: dict, lv: OLevel, parent, f_out, f_in, vel_out, vel_in, g_out, g_in,
                     u: float, t_sub: int, tw: float, domain_dims, dtype, k=orc):
    """timestep.jl:1-159 on one level; `k` is the kernel set (the CPU oracle,
    or oracle.gpu over device tensors)."""
    h = lv.host
    is_l1 = parent is None
    scale = 1 << (h.level_id - 1)
    dims = tuple(d * scale for d in domain_dims)
    bz = h.bouzidi and h.n_boundary > 0
    params = dict(s)
    params.update(tau_molecular=h.tau, tau_parent=parent["tau"] if parent else 0.5,
                  is_level_1=int(is_l1), nx_global=dims[0], ny_global=dims[1], nz_global=dims[2],
                  u_inlet=u, time_step_seed=t_sub % 1000000, store_post_collision=int(bz),
                  temporal_weight=tw)
    pv = None
    if parent is not None:
        pv = dict(f=parent["f"], rho=parent["rho"], vel=parent["vel"], f_old=parent["f_old"],
                  rho_old=parent["rho_old"], vel_old=parent["vel_old"],
                  block_ptr=parent["block_ptr"], dim=parent["dim"], n_blocks=parent["n_blocks"])
    k.stream_collide(_level_dict(lv, f_out, f_in, vel_out, vel_in, bz), pv, params, dtype)
    if bz:
        k.bouzidi(f_out, lv.f_post, h.q_map, h.cell_block, h.cell_x, h.cell_y, h.cell_z,
                  h.neighbor_table, h.n_blocks, s["q_min"], dtype)
    if s.get("ddf") and g_out is not None:
        tp = dict(tau_g=h.tau_g, tau_g_parent=parent["tau_g"] if parent else 0.5,
                  is_level_1=int(is_l1), is_symmetric=s["is_symmetric"], nx_global=dims[0],
                  ny_global=dims[1], nz_global=dims[2], u_inlet=u, T_inlet=s["T_inlet"],
                  T_wall=s["T_wall"], wall_bc_adiabatic=s["wall_bc_adiabatic"],
                  store_post_collision=int(bz), temporal_weight=tw,
                  use_temporal_interp=s["use_temporal_interp"],
                  sponge_blend_distributions=s["sponge_blend_distributions"])
        tv = dict(g_out=g_out, g_in=g_in, g_post=lv.g_post if bz else None, T=lv.T, vel=vel_out,
                  obstacle=h.obstacle, sponge=h.sponge, neighbor_table=h.neighbor_table,
                  map_x=h.map_x, map_y=h.map_y, map_z=h.map_z, n_blocks=h.n_blocks)
        tpv = None
        if parent is not None:
            tpv = dict(g=parent["g"], T=parent["T"], vel=parent["vel"], g_old=parent["g_old"],
                       T_old=parent["T_old"], vel_old=parent["vel_old"],
                       block_ptr=parent["block_ptr"], dim=parent["dim"], n_blocks=parent["n_blocks"])
        k.thermal(tv, tpv, tp, dtype)
        if bz:
            k.bouzidi(g_out, lv.g_post, h.q_map, h.cell_block, h.cell_x, h.cell_y, h.cell_z,
                      h.neighbor_table, h.n_blocks, s["q_min"], dtype)


def recursive_step(levels, s, lvl, t_sub, parent, tw, u, domain_dims, dtype, k=orc):
    """solver_control.jl:6-98 (copy_to_old! before a parent step, children
    at (2t, tw 0) and (2t+1, tw 1/2))."""
    if lvl >= len(levels):
        return
    lv = levels[lvl]
    if t_sub % 2 == 0:
        f_in, f_out, vel_in, vel_out = lv.f, lv.f_temp, lv.vel, lv.vel_temp
        g_in, g_out = lv.g, lv.g_temp
    else:
        f_in, f_out, vel_in, vel_out = lv.f_temp, lv.f, lv.vel_temp, lv.vel
        g_in, g_out = lv.g_temp, lv.g
    has_children = lvl + 1 < len(levels)
    if has_children and s["use_temporal_interp"]:
        k.copyto(lv.f_old, f_in)
        k.copyto(lv.rho_old, lv.rho)
        k.copyto(lv.vel_old, vel_in)
        if s.get("ddf") and lv.g is not None:
            k.copyto(lv.g_old, g_in)
            k.copyto(lv.T_old, lv.T)
    perform_timestep(s, lv, parent, f_out, f_in, vel_out, vel_in, g_out, g_in, u, t_sub,
                     0.0 if parent is None else tw, domain_dims, dtype, k)
    if has_children:
        h = lv.host
        me = dict(f=f_out, rho=lv.rho, vel=vel_out, f_old=lv.f_old, rho_old=lv.rho_old,
                  vel_old=lv.vel_old, block_ptr=h.block_ptr, dim=h.grid_dim, n_blocks=h.n_blocks,
                  tau=h.tau, tau_g=h.tau_g, g=g_out, T=lv.T, g_old=lv.g_old, T_old=lv.T_old)
        recursive_step(levels, s, lvl + 1, 2 * t_sub, me, 0.0, u, domain_dims, dtype, k)
        recursive_step(levels, s, lvl + 1, 2 * t_sub + 1, me, 0.5, u, domain_dims, dtype, k)
        if s.get("restriction"):
            c = levels[lvl + 1]   # its second sub-step (odd t_sub) wrote f and vel
            k.restrict(c.f, c.host.obstacle, c.host.map_x, c.host.map_y, c.host.map_z,
                         c.host.n_blocks, f_out, lv.rho, vel_out, h.obstacle, h.block_ptr,
                         h.grid_dim, h.n_blocks, c.host.tau, h.tau, s["compressible_corr"], dtype)


def settings_dict(st) -> dict:
    """Convert solver.StepSettings to the oracle's parameter dictionary."""
    return dict(op=st.op, c_wale=st.c_wale, nu_sgs_background=st.nu_sgs_bg,
                is_symmetric=st.is_symmetric, wall_model_active=st.wall_model,
                inlet_turbulence=st.inlet_turbulence, use_temporal_interp=st.use_temporal_interp,
                sponge_blend_distributions=st.sponge_blend, omega_bulk=st.omega_bulk,
                omega_3=st.omega_3, omega_4=st.omega_4, adaptive_omega4=st.adaptive_omega4,
                lambda_param=st.lambda_param, limiter_type=st.limiter,
                compressible_corr=st.compressible, q_min=st.q_min, ddf=st.ddf,
                T_inlet=st.t_inlet, T_wall=st.t_wall, wall_bc_adiabatic=st.wall_bc_adiabatic,
                restriction=st.restriction)
