"""Synthetic stand-ins for the benchmark workloads.

The reference has no benchmark suite; these cases reproduce the shapes of the
five benchmark configurations with seeded, generated geometry:

  sphere_1lvl   128x64x64 single level, D = 16 cells icosphere (1280 triangles),
                Re = 1000, u = 0.05, cumulant, Bouzidi, no WALE
  cube_3lvl     cube of side 16/32/64 cells on levels 1..3 rotated alpha = 10 deg,
                coarsest 160x80x80, Re = 1e5, cumulant + WALE (0.5) + WMLES
  sphere_ddf    5120-triangle icosphere, D = 48 finest cells, 2 levels,
                Ma = 0.6 (u = 0.346), O(u^4) + thermal DDF
  batch_mix     48 seeded cases: sphere / cube / NACA0012 wing, 16..48 finest
                cells, 1..3 levels, Re log-uniform [1e3, 1e6]
Each returns a CaseConfig (the YAML keys the reference reads) and the
rotated body mesh, ready for scaling.compute_domain_from_mesh.
"""
from __future__ import annotations

import dataclasses as dc
import math

import numpy as np

from . import geometry as geo
from .config import CaseConfig, f32


def base_config(**kw) -> CaseConfig:
    c = CaseConfig()
    c.stl_scale = 1.0
    c.reference_length_for_meshing = 1.0
    c.reference_chord_config = 1.0
    c.fluid_density = 1.0
    c.flow_velocity = 1.0
    c.inlet_turbulence_intensity = f32(0.0)
    c.boundary_method = "bouzidi"
    c.bouzidi_levels = 1
    c.forces_enabled = True
    c.ramp_steps = 0
    c.diag_freq = 100
    c.async_depth = 8
    c.sponge_thickness = f32(0.10)
    c.cumulant_limiter = "factored"
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def sphere_1lvl(resolution: int = 16):
    """128x64x64 sphere case (single level, Bouzidi, no WALE)."""
    c = base_config(surface_resolution=resolution, num_levels_config=1,
                    domain_upstream=2.0, domain_downstream=5.0, domain_lateral=1.5,
                    domain_height=1.5, u_target=f32(0.05), c_wale=f32(0.0),
                    fluid_kinematic_viscosity=1e-3, reference_area_full_model=math.pi / 4,
                    steps=2000)
    c.reference_area_config = c.reference_area_full_model
    mesh = geo.icosphere(3, radius=0.5)
    return c, mesh


def cube_3lvl(alpha_deg: float = 10.0):
    """Three-level refined cube (coarsest 160x80x80, finest side 64 cells)."""
    c = base_config(surface_resolution=64, num_levels_config=3,
                    domain_upstream=3.0, domain_downstream=5.8, domain_lateral=2.0,
                    domain_height=1.9, u_target=f32(0.05), c_wale=f32(0.5),
                    wall_model_enabled=True, fluid_kinematic_viscosity=1e-5,
                    alpha_deg=alpha_deg, reference_area_full_model=1.0, steps=2500)
    c.reference_area_config = 1.0
    mesh = geo.rotate_mesh(geo.cube(1.0), alpha_deg, 0.0)
    return c, mesh


def sphere_ddf():
    """Compressible thermal sphere: O(u^4) + DDF, 2 levels, D = 48 finest."""
    c = base_config(surface_resolution=48, num_levels_config=2,
                    domain_upstream=1.5, domain_downstream=3.0, domain_lateral=1.5,
                    domain_height=1.5, u_target=f32(0.346), c_wale=f32(0.5),
                    fluid_kinematic_viscosity=1e-6, compressibility_correction=True,
                    ddf_enabled=True, reference_area_full_model=math.pi / 4, steps=4000)
    c.reference_area_config = c.reference_area_full_model
    mesh = geo.icosphere(4, radius=0.5)
    return c, mesh


def build_case(workload: str):
    """(cfg, mesh, domain params, host levels) of a named benchmark workload."""
    from . import domain, scaling
    makers = {"cube_3lvl": cube_3lvl, "sphere_1lvl": sphere_1lvl, "sphere_ddf": sphere_ddf}
    cfg, mesh = makers[workload]()
    p = scaling.compute_domain_from_mesh(cfg, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(cfg, mesh, p)
    return cfg, mesh, p, hosts


@dc.dataclass
class MixCase:
    kind: str
    size_cells: int
    levels: int
    re: float
    alpha: float
    beta: float


def batch_mix(n: int = 48, seed: int = 1234, large_frac: float = 0.0) -> list[MixCase]:
    """Seeded draw of the uneven batch: geometry, finest size, depth, Re, angles."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        if large_frac > 0 and rng.random() < large_frac:
            kind, size, lv = ["sphere", "cube", "wing"][rng.integers(3)], 64, 3
        else:
            kind = ["sphere", "cube", "wing"][rng.integers(3)]
            size = int([16, 24, 32, 48][rng.integers(4)])
            lv = int(rng.integers(1, 4))
        re = float(10 ** rng.uniform(3, 6))
        out.append(MixCase(kind, size, lv, re, float(rng.uniform(-4, 12)),
                           float(rng.uniform(-5, 5))))
    return out


def mix_case_config(m: MixCase):
    """CaseConfig + mesh of one batch case (FP16-shifted, cumulant + WALE)."""
    # finest body size `size_cells`; coarse spacing 2^(levels-1) times larger
    c = base_config(surface_resolution=m.size_cells, num_levels_config=m.levels,
                    domain_upstream=1.5, domain_downstream=3.0, domain_lateral=1.0,
                    domain_height=1.0, u_target=f32(0.05), c_wale=f32(0.5),
                    fluid_kinematic_viscosity=1.0 / m.re, alpha_deg=m.alpha, beta_deg=m.beta,
                    steps=100000)
    if m.kind == "sphere":
        mesh = geo.icosphere(4, radius=0.5)
        c.reference_area_full_model = math.pi / 4
    elif m.kind == "cube":
        mesh = geo.cube(1.0)
        c.reference_area_full_model = 1.0
    else:
        mesh = geo.naca0012_wing(chord=1.0, span=3.0)
        c.reference_area_full_model = 3.0
        c.domain_lateral = 0.75
    c.reference_area_config = c.reference_area_full_model
    mesh = geo.rotate_mesh(mesh, m.alpha, m.beta)
    return c, mesh
