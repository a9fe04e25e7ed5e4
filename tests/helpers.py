"""Shared builders for the tests: small cases with the shapes of the
benchmark workloads, seeded perturbed states, and comparison helpers."""
from __future__ import annotations

import math

import numpy as np

from openludwig_b200 import domain, geometry as geo, scaling, workloads
from openludwig_b200.config import f32


def small_sphere_case(resolution: int = 8, levels: int = 1, bouzidi: bool = True, **kw):
    """A sphere case like the 128x64x64 workload at a reduced resolution
    (resolution 8 -> 64x32x32 cells, 128 blocks on level 1)."""
    c, mesh = workloads.sphere_1lvl(resolution)
    c.num_levels_config = levels
    if levels > 1:
        c.domain_upstream, c.domain_downstream = 1.0, 2.0
        c.domain_lateral = c.domain_height = 1.0
        c.min_coarse_blocks = 2
    if not bouzidi:
        c.boundary_method = "bounce_back"
    for k, v in kw.items():
        setattr(c, k, v)
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    return c, mesh, p, hosts


def interior_refined_case():
    """Two-level cube (48 finest cells, Re 1.6e5, alpha 3.2, beta -1.9) whose
    refined level lies inside the domain: all its absent-neighbour values
    are coarse-to-fine (4096 fine blocks, 1352 at the interface)."""
    m = workloads.MixCase("cube", 48, 2, 158378.0, 3.18, -1.94)
    c, mesh = workloads.mix_case_config(m)
    c.ramp_steps = 0
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    return c, mesh, p, hosts


def lattice():
    cx, cy, cz = [], [], []
    for z in (-1, 0, 1):
        for y in (-1, 0, 1):
            for x in (-1, 0, 1):
                cx.append(x); cy.append(y); cz.append(z)
    return np.array(cx), np.array(cy), np.array(cz)


def weights32():
    cx, cy, cz = lattice()
    d2 = cx * cx + cy * cy + cz * cz
    w = np.where(d2 == 0, np.float32(8) / np.float32(27),
                 np.where(d2 == 1, np.float32(2) / np.float32(27),
                          np.where(d2 == 2, np.float32(1) / np.float32(54),
                                   np.float32(1) / np.float32(216))))
    return w.astype(np.float32)


def perturbed_state(n_blocks: int, seed: int, amp: float = 0.05, u0: float = 0.05):
    """f = f_eq(rho ~ 1, u ~ (u0, 0, 0) + noise) * (1 + amp * noise): every
    population positive, a non-trivial flow for every collision branch."""
    rng = np.random.default_rng(seed)
    S = 512 * n_blocks
    cx, cy, cz = lattice()
    w = weights32().astype(np.float64)
    rho = 1.0 + 0.01 * rng.standard_normal(S)
    ux = u0 + 0.02 * rng.standard_normal(S)
    uy = 0.02 * rng.standard_normal(S)
    uz = 0.02 * rng.standard_normal(S)
    f = np.empty((27, S))
    for k in range(27):
        cu = cx[k] * ux + cy[k] * uy + cz[k] * uz
        usq = ux * ux + uy * uy + uz * uz
        f[k] = rho * w[k] * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * usq)
    f *= 1.0 + amp * rng.standard_normal(f.shape)
    vel = np.concatenate([ux, uy, uz]) + 0.005 * rng.standard_normal(3 * S)
    return f.reshape(-1).astype(np.float32), vel.astype(np.float32)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def max_abs(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))
