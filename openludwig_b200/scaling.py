"""Domain size, level count, grid spacing, tau per level and unit scales from
the mesh bounds (solver/physics_scaling.jl:63-191)."""
from __future__ import annotations

import dataclasses as dc
import math

import numpy as np

from .config import CaseConfig


@dc.dataclass
class DomainParams:
    num_levels: int
    mesh_min: tuple
    mesh_max: tuple
    mesh_center: tuple
    mesh_extent: tuple
    reference_length: float
    reference_chord: float
    reference_area: float
    moment_center: tuple
    domain_size: tuple
    mesh_offset: tuple
    dx_fine: float
    dx_coarse: float
    dx_levels: list
    nx_coarse: int
    ny_coarse: int
    nz_coarse: int
    bx_max: int
    by_max: int
    bz_max: int
    nu_lattice: float
    tau_levels: list          # float32 values
    re_number: float
    u_physical: float
    rho_physical: float
    nu_physical: float
    length_scale: float
    time_scale: float
    velocity_scale: float
    force_scale: float
    tau_fine: float
    tau_g_fine: float
    tau_g_levels: list


def compute_tau(Re: float, resolution: int, u_lattice: float) -> float:
    """physics_scaling.jl:63-66."""
    nu = float(u_lattice) * resolution / Re
    return 3.0 * nu + 0.5


def max_levels_for_domain(domain_size: float, dx_fine: float, block_size: int, min_blocks: int) -> int:
    ratio = domain_size / (dx_fine * min_blocks * block_size)
    return 1 if ratio < 1.0 else int(math.floor(1 + math.log2(ratio)))


def f32(x: float) -> float:
    return float(np.float32(x))


def compute_domain_from_mesh(cfg: CaseConfig, mesh_min: tuple, mesh_max: tuple) -> DomainParams:
    """physics_scaling.jl:83-191."""
    mc = tuple((mesh_min[i] + mesh_max[i]) / 2 for i in range(3))
    me = tuple(mesh_max[i] - mesh_min[i] for i in range(3))
    if cfg.reference_length_for_meshing > 0:
        L = cfg.reference_length_for_meshing
    else:
        L = {"x": me[0], "y": me[1], "z": me[2]}.get(cfg.reference_dimension, max(me))
    chord = cfg.reference_chord_config if cfg.reference_chord_config > 0 else me[0]
    if cfg.reference_area_config > 0:
        area = cfg.reference_area_config
    else:
        area = me[1] * me[2] * 2 if cfg.symmetric_analysis else me[1] * me[2]
    u_phys, nu_phys, rho_phys = cfg.flow_velocity, cfg.fluid_kinematic_viscosity, cfg.fluid_density
    Re = u_phys * L / nu_phys
    tau_fine = max(compute_tau(Re, cfg.surface_resolution, cfg.u_target), cfg.tau_min)
    dom_x = L * (cfg.domain_upstream + cfg.domain_downstream) + me[0]
    dom_y = (mesh_max[1] + L * cfg.domain_lateral) if cfg.symmetric_analysis else (me[1] + 2 * L * cfg.domain_lateral)
    dom_z = me[2] + 2 * L * cfg.domain_height
    dx_fine = L / cfg.surface_resolution
    max_lv = max_levels_for_domain(min(dom_x, dom_y, dom_z), dx_fine, cfg.block_size, cfg.min_coarse_blocks)
    if cfg.num_levels_config > 0:
        nl = min(cfg.num_levels_config, max_lv)
    else:
        nl = min(max_lv, cfg.max_levels) if cfg.auto_levels else min(8, max_lv)
    dx_coarse = dx_fine * 2 ** (nl - 1)
    dx_levels = [dx_fine * 2 ** (nl - l) for l in range(1, nl + 1)]
    bs = cfg.block_size
    nx = max(bs, int(math.ceil(math.ceil(dom_x / dx_coarse) / bs) * bs))
    ny = max(bs, int(math.ceil(math.ceil(dom_y / dx_coarse) / bs) * bs))
    nz = max(bs, int(math.ceil(math.ceil(dom_z / dx_coarse) / bs) * bs))
    dom_x, dom_y, dom_z = nx * dx_coarse, ny * dx_coarse, nz * dx_coarse
    mesh_x = L * cfg.domain_upstream
    mesh_y = 0.0 if cfg.symmetric_analysis else (dom_y / 2 - mc[1])
    mesh_z = dom_z / 2 - mc[2]
    offset = (mesh_x - mesh_min[0], mesh_y, mesh_z)
    length_scale = dx_fine
    velocity_scale = u_phys / float(cfg.u_target)
    time_scale = length_scale / velocity_scale
    nu_lat = nu_phys * time_scale / (length_scale ** 2)
    tau_levels = []
    for l in range(1, nl + 1):
        t = tau_fine if l == nl else 0.5 + (tau_fine - 0.5) * 2.0 ** (nl - l)
        tau_levels.append(f32(t))
    force_scale = rho_phys * length_scale ** 4 / time_scale ** 2
    mcr = [float(v) for v in cfg.moment_center]
    moment_center = (mesh_min[0] + offset[0] + mcr[0] * chord,
                     mc[1] + offset[1] + mcr[1] * chord,
                     mc[2] + offset[2] + mcr[2] * chord)
    tau_g_fine, tau_g_levels = 0.0, []
    if cfg.ddf_enabled:
        kappa = nu_lat / cfg.ddf_prandtl
        tau_g_fine = 0.5 + 3.0 * kappa
        for l in range(1, nl + 1):
            t = tau_g_fine if l == nl else 0.5 + (tau_g_fine - 0.5) * 2.0 ** (nl - l)
            tau_g_levels.append(f32(t))
    return DomainParams(
        num_levels=nl, mesh_min=tuple(mesh_min), mesh_max=tuple(mesh_max), mesh_center=mc,
        mesh_extent=me, reference_length=L, reference_chord=chord, reference_area=area,
        moment_center=moment_center, domain_size=(dom_x, dom_y, dom_z), mesh_offset=offset,
        dx_fine=dx_fine, dx_coarse=dx_coarse, dx_levels=dx_levels, nx_coarse=nx, ny_coarse=ny,
        nz_coarse=nz, bx_max=nx // bs, by_max=ny // bs, bz_max=nz // bs, nu_lattice=nu_lat,
        tau_levels=tau_levels, re_number=Re, u_physical=u_phys, rho_physical=rho_phys,
        nu_physical=nu_phys, length_scale=length_scale, time_scale=time_scale,
        velocity_scale=velocity_scale, force_scale=force_scale, tau_fine=tau_fine,
        tau_g_fine=tau_g_fine, tau_g_levels=tau_g_levels)
