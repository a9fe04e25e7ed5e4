"""Case scaling (physics_scaling.jl:63-191): the product's
scaling.compute_domain_from_mesh against the oracle's independent C++
restatement (orc_domain_scaling), value for value, on the benchmark
workloads, the seeded batch mix, the reference's own case folders (values
recorded in tests/golden/reference_cases.json) and variants that reach every
branch (symmetric half model, reference dimension y / z / maximum, automatic
level count, thermal DDF, configured chord and area, moment centre).

Known answers pin the formulas on numbers worked by hand:
* the 128x64x64 sphere: Re = 1000, tau = 1/2 + 3 * 0.05 * 16 / 1000;
* the cube of the three-level workload: nu_lat < (tau_min - 1/2) / 3, so the
  finest tau clamps to tau_min = Float32(0.501) and the coarser levels double
  the excess: tau_l = 1/2 + 0.001 * 2^(3 - l);
* the reference's cube case folder: u_lattice 0.08, 75 cells per metre,
  Re = U L / nu from its YAML."""
import dataclasses as dc
import json
import math
from pathlib import Path

import numpy as np
import pytest

from openludwig_b200 import config, scaling, workloads
from oracle import oracle as orc

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_cases.json").read_text())

FIELDS = ["num_levels", "nx_coarse", "ny_coarse", "nz_coarse", "bx_max", "by_max", "bz_max",
          "reference_length", "reference_chord", "reference_area", "re_number", "tau_fine",
          "domain_size", "mesh_offset", "moment_center", "dx_fine", "dx_coarse", "dx_levels",
          "length_scale", "velocity_scale", "time_scale", "nu_lattice", "force_scale",
          "tau_levels", "tau_g_fine", "tau_g_levels"]


@pytest.fixture(scope="module", autouse=True)
def _oracle():
    orc.build()


def _cases():
    out = []
    for name in ("sphere_1lvl", "cube_3lvl", "sphere_ddf"):
        c, m = getattr(workloads, name)()
        out.append((name, c, m.min_bounds, m.max_bounds))
    for i, mc in enumerate(workloads.batch_mix(12, seed=1234, large_frac=0.25)):
        c, m = workloads.mix_case_config(mc)
        out.append((f"mix{i}_{mc.kind}{mc.size_cells}x{mc.levels}", c, m.min_bounds, m.max_bounds))
    for name, entry in GOLD["cases"].items():
        c = config.CaseConfig()
        for k, v in entry["config"].items():
            setattr(c, k, v)
        out.append((name, c, tuple(entry["stl"]["min_bounds"]), tuple(entry["stl"]["max_bounds"])))
    base, m = workloads.sphere_1lvl()
    lo, hi = m.min_bounds, m.max_bounds
    variants = {
        "symmetric": dict(symmetric_analysis=True, reference_area_config=0.0),
        "ref_dim_y": dict(reference_length_for_meshing=0.0, reference_dimension="y"),
        "ref_dim_z": dict(reference_length_for_meshing=0.0, reference_dimension="z"),
        "ref_dim_max": dict(reference_length_for_meshing=0.0, reference_dimension="max"),
        "auto_levels": dict(num_levels_config=0, auto_levels=True, max_levels=3),
        "default_levels": dict(num_levels_config=0, auto_levels=False),
        "ddf": dict(ddf_enabled=True, ddf_prandtl=0.71, num_levels_config=2),
        "chord_moment": dict(reference_chord_config=0.0, moment_center=[0.25, 0.1, -0.05]),
        "physical_units": dict(flow_velocity=30.0, fluid_kinematic_viscosity=1.5e-5,
                               fluid_density=1.225, surface_resolution=40),
    }
    for name, kw in variants.items():
        c = dc.replace(base)
        for k, v in kw.items():
            setattr(c, k, v)
        out.append((name, c, lo, hi))
    return out


CASES = _cases()


@pytest.mark.parametrize("name,cfg,lo,hi", CASES, ids=[c[0] for c in CASES])
def test_scaling_matches_oracle_restatement(name, cfg, lo, hi):
    p = scaling.compute_domain_from_mesh(cfg, lo, hi)
    o = orc.domain_scaling(cfg, lo, hi)
    for k in FIELDS:
        mine, ref = getattr(p, k), o[k]
        if isinstance(mine, (tuple, list)):
            mine, ref = list(mine), list(ref)
        assert mine == ref, (name, k, mine, ref)


def test_known_answers():
    c, m = workloads.sphere_1lvl()
    p = scaling.compute_domain_from_mesh(c, m.min_bounds, m.max_bounds)
    assert (p.nx_coarse, p.ny_coarse, p.nz_coarse, p.num_levels) == (128, 64, 64, 1)
    assert p.re_number == pytest.approx(1000.0)
    assert p.tau_levels == [float(np.float32(0.5 + 3 * float(np.float32(0.05)) * 16 / 1000))]

    c, m = workloads.cube_3lvl()
    p = scaling.compute_domain_from_mesh(c, m.min_bounds, m.max_bounds)
    assert (p.nx_coarse, p.ny_coarse, p.nz_coarse, p.num_levels) == (160, 80, 80, 3)
    assert p.nu_lattice < (float(np.float32(0.501)) - 0.5) / 3
    t = float(np.float32(0.501))
    assert p.tau_fine == t
    assert p.tau_levels == [float(np.float32(0.5 + (t - 0.5) * 2.0 ** (3 - l))) for l in (1, 2, 3)]
    assert p.dx_levels == [p.dx_fine * 4, p.dx_fine * 2, p.dx_fine]

    entry = GOLD["cases"]["cube1m_Re1e3"]
    c = config.CaseConfig()
    for k, v in entry["config"].items():
        setattr(c, k, v)
    p = scaling.compute_domain_from_mesh(c, tuple(entry["stl"]["min_bounds"]),
                                         tuple(entry["stl"]["max_bounds"]))
    L = 1.0   # unit cube, reference dimension x
    re = c.flow_velocity * L / c.fluid_kinematic_viscosity
    assert p.re_number == re
    assert p.tau_fine == max(3.0 * float(np.float32(0.08)) * 75 / re + 0.5, float(np.float32(0.501)))
    assert p.dx_fine == L / 75
    assert p.time_scale == p.dx_fine / (c.flow_velocity / float(np.float32(0.08)))


def test_thermal_levels_follow_prandtl():
    c, m = workloads.sphere_ddf()
    p = scaling.compute_domain_from_mesh(c, m.min_bounds, m.max_bounds)
    kappa = p.nu_lattice / c.ddf_prandtl
    assert p.tau_g_fine == 0.5 + 3.0 * kappa
    nl = p.num_levels
    assert p.tau_g_levels[-1] == float(np.float32(p.tau_g_fine))
    assert p.tau_g_levels[0] == float(np.float32(0.5 + (p.tau_g_fine - 0.5) * 2.0 ** (nl - 1)))
    assert math.isclose(p.force_scale,
                        p.rho_physical * p.length_scale ** 4 / p.time_scale ** 2, rel_tol=1e-15)
