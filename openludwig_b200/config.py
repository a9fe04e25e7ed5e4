"""Case YAML loader: the same keys, defaults and validation as the reference's
``load_case_configuration`` (io/config_loader.jl:133-329), returned as one
``CaseConfig`` object instead of ~90 mutable globals.

A case directory holds ``config.yaml`` plus the STL file(s) it names; a list
file (``cases_to_run.yaml``) names case directories under ``CASES/``
(main.jl:413-483).
"""
from __future__ import annotations

import dataclasses as dc
import math
from pathlib import Path
from typing import Any

import yaml

VALID_COLLISION_OPERATORS = {"regularized_bgk", "cumulant"}
VALID_CUMULANT_LIMITERS = {"none", "factored", "positivity"}


class ConfigError(ValueError):
    """Missing key, unknown enum value or unreadable case (config_loader.jl errors)."""


def f32(x: float) -> float:
    """Round through binary32, as the reference's Float32(...) globals do."""
    import numpy as np
    return float(np.float32(x))


_MISSING = object()


def safe_get(d: Any, *keys: str, default: Any = _MISSING) -> Any:
    """config_loader.jl:122-131: walk nested keys; a missing key without a
    default is an error; an explicit null takes the default."""
    cur = d
    for i, k in enumerate(keys):
        if cur is None or not isinstance(cur, dict) or k not in cur:
            if default is not _MISSING:
                return default
            raise ConfigError("Missing config key: " + " -> ".join(keys[: i + 1]))
        cur = cur[k]
    if cur is None and default is not _MISSING:
        return default
    return cur


@dc.dataclass
class CaseConfig:
    case_dir: str = ""
    stl_files: list = dc.field(default_factory=list)
    stl_scale: float = 1.0
    out_dir_name: str = "RESULTS"
    surface_resolution: int = 200
    num_levels_config: int = 0
    minimum_facet_size: float = 0.0
    symmetric_analysis: bool = False
    alpha_deg: float = 0.0
    beta_deg: float = 0.0
    reference_area_full_model: float = 0.0
    reference_area_config: float = 0.0
    reference_chord_config: float = 0.0
    reference_length_for_meshing: float = 0.0
    reference_dimension: str = "x"
    fluid_density: float = 1.225
    fluid_kinematic_viscosity: float = 1.5e-5
    flow_velocity: float = 10.0
    domain_length_covered: float = 0.0
    steps: int = 1000
    ramp_steps: int = 1500
    output_freq: int = 100
    collision_operator: str = "cumulant"
    u_target: float = f32(0.08)
    c_wale: float = f32(0.20)
    tau_min: float = f32(0.501)
    tau_safety_factor: float = f32(1.0)
    inlet_turbulence_intensity: float = f32(0.01)
    nu_sgs_background: float = f32(0.0)
    sponge_blend_distributions: bool = False
    temporal_interpolation: bool = True
    fine_to_coarse_restriction: bool = False   # opt-in extension, not in the reference
    cumulant_omega_bulk: float = f32(1.0)
    cumulant_omega_3: float = f32(1.0)
    cumulant_omega_4: float = f32(1.0)
    cumulant_adaptive_omega4: bool = True
    cumulant_lambda_param: float = f32(1.0 / 6.0)
    cumulant_limiter: str = "factored"
    compressibility_correction: bool = False
    ddf_enabled: bool = False
    ddf_prandtl: float = 0.71
    ddf_t_inlet: float = 1.0
    ddf_t_wall: float = 1.0
    ddf_t_initial: float = 1.0
    ddf_wall_bc: str = "adiabatic"
    auto_levels: bool = False
    max_levels: int = 12
    min_coarse_blocks: int = 4
    wall_model_enabled: bool = False
    wall_model_type: str = "equilibrium"
    wall_model_yplus_target: float = 30.0
    domain_upstream: float = 0.75
    domain_downstream: float = 1.5
    domain_lateral: float = 0.75
    domain_height: float = 0.75
    sponge_thickness: float = f32(0.10)
    block_size: int = 8
    refinement_margin: int = 2
    refinement_strategy: str = "geometry_first"
    wake_enabled: bool = False
    wake_length: float = 0.25
    wake_width_factor: float = 0.1
    wake_height_factor: float = 0.1
    boundary_method: str = "bounce_back"
    bouzidi_levels: int = 1
    q_min_threshold: float = f32(0.001)
    forces_enabled: bool = False
    force_output_freq_config: int = 0
    moment_center: list = dc.field(default_factory=lambda: [0.25, 0.0, 0.0])
    net_force_export: bool = False
    diag_freq: int = 500
    async_depth: int = 8

    @property
    def force_output_freq(self) -> int:
        return self.diag_freq if self.force_output_freq_config == 0 else self.force_output_freq_config

    @property
    def limiter_code(self) -> int:
        return {"none": 0, "factored": 1, "positivity": 2}[self.cumulant_limiter]

    @property
    def operator_code(self) -> int:
        return 0 if self.collision_operator == "cumulant" else 1


def config_from_dict(cfg: dict, case_dir: str = ".") -> CaseConfig:
    """Parse an already-loaded YAML mapping (config_loader.jl:143-281)."""
    c = CaseConfig(case_dir=str(case_dir))
    raw = safe_get(cfg, "basic", "stl_file")
    if isinstance(raw, str):
        names = [raw]
    elif isinstance(raw, list):
        names = [str(s) for s in raw]
    else:
        raise ConfigError(f"stl_file must be a string or list of strings, got: {type(raw).__name__}")
    c.stl_files = [str(Path(case_dir) / n) for n in names]
    c.stl_scale = float(safe_get(cfg, "basic", "stl_scale"))
    c.out_dir_name = safe_get(cfg, "basic", "simulation", "output_dir")
    c.surface_resolution = int(safe_get(cfg, "basic", "surface_resolution"))
    c.num_levels_config = int(safe_get(cfg, "basic", "num_levels"))
    c.minimum_facet_size = float(safe_get(cfg, "basic", "minimum_facet_size", default=0.0))
    c.symmetric_analysis = bool(safe_get(cfg, "advanced", "refinement", "symmetric_analysis", default=False))
    c.alpha_deg = float(safe_get(cfg, "basic", "alpha", default=0.0))
    c.beta_deg = float(safe_get(cfg, "basic", "beta", default=0.0))
    if c.symmetric_analysis and c.beta_deg != 0.0:
        c.beta_deg = 0.0  # config_loader.jl:165-168
    c.reference_area_full_model = float(safe_get(cfg, "basic", "reference_area_of_full_model", default=0.0))
    c.reference_area_config = (c.reference_area_full_model / 2.0 if c.symmetric_analysis
                               else c.reference_area_full_model)
    c.reference_chord_config = float(safe_get(cfg, "basic", "reference_chord", default=0.0))
    c.reference_length_for_meshing = float(safe_get(cfg, "basic", "reference_length_for_meshing", default=0.0))
    c.reference_dimension = str(safe_get(cfg, "basic", "reference_dimension", default="x"))
    c.fluid_density = float(safe_get(cfg, "basic", "fluid", "density", default=1.225))
    c.fluid_kinematic_viscosity = float(safe_get(cfg, "basic", "fluid", "kinematic_viscosity", default=1.5e-5))
    c.flow_velocity = float(safe_get(cfg, "basic", "flow", "velocity", default=10.0))
    c.domain_length_covered = float(safe_get(cfg, "basic", "simulation", "domain_length_covered", default=0.0))
    c.steps = int(safe_get(cfg, "basic", "simulation", "steps", default=0))
    c.ramp_steps = int(safe_get(cfg, "basic", "simulation", "ramp_steps"))
    c.output_freq = int(safe_get(cfg, "basic", "simulation", "output_freq"))
    op = str(safe_get(cfg, "advanced", "numerics", "collision_operator", default="cumulant"))
    if op not in VALID_COLLISION_OPERATORS:
        raise ConfigError(f'Unknown collision_operator: "{op}". Valid options: '
                          + ", ".join(sorted(VALID_COLLISION_OPERATORS)))
    c.collision_operator = op
    g = lambda *k, d: safe_get(cfg, "advanced", "numerics", *k, default=d)  # noqa: E731
    c.u_target = f32(g("u_lattice", d=0.08))
    c.c_wale = f32(g("c_wale", d=0.20))
    c.tau_min = f32(g("tau_min", d=0.501))
    c.tau_safety_factor = f32(g("tau_safety_factor", d=1.0))
    c.inlet_turbulence_intensity = f32(g("inlet_turbulence_intensity", d=0.01))
    c.nu_sgs_background = f32(g("nu_sgs_background", d=0.0))
    c.sponge_blend_distributions = bool(g("sponge_blend_distributions", d=False))
    c.temporal_interpolation = bool(g("temporal_interpolation", d=True))
    c.fine_to_coarse_restriction = bool(g("fine_to_coarse_restriction", d=False))
    c.cumulant_omega_bulk = f32(g("cumulant", "omega_bulk", d=1.0))
    c.cumulant_omega_3 = f32(g("cumulant", "omega_3", d=1.0))
    c.cumulant_omega_4 = f32(g("cumulant", "omega_4", d=1.0))
    c.cumulant_adaptive_omega4 = bool(g("cumulant", "adaptive_omega_4", d=True))
    c.cumulant_lambda_param = f32(g("cumulant", "lambda_param", d=1.0 / 6.0))
    lim = str(g("cumulant", "limiter", d="factored"))
    if lim not in VALID_CUMULANT_LIMITERS:
        raise ConfigError(f'Unknown cumulant limiter: "{lim}". Valid: '
                          + ", ".join(sorted(VALID_CUMULANT_LIMITERS)))
    c.cumulant_limiter = lim
    c.compressibility_correction = bool(g("compressibility_correction", d=False))
    c.ddf_enabled = c.compressibility_correction  # config_loader.jl:225
    if c.ddf_enabled:
        t = lambda k, d: safe_get(cfg, "advanced", "thermal", k, default=d)  # noqa: E731
        c.ddf_prandtl = float(t("prandtl", 0.71))
        c.ddf_t_inlet = float(t("t_inlet", 1.0))
        c.ddf_t_wall = float(t("t_wall", 1.0))
        c.ddf_t_initial = float(t("t_initial", 1.0))
        bc = str(t("wall_bc", "adiabatic"))
        if bc not in ("adiabatic", "isothermal"):
            raise ConfigError(f'Unknown thermal wall_bc: "{bc}". Valid: adiabatic, isothermal')
        c.ddf_wall_bc = bc
    h = lambda *k, d: safe_get(cfg, "advanced", "high_re", *k, default=d)  # noqa: E731
    c.auto_levels = bool(h("auto_levels", d=False))
    c.max_levels = int(h("max_levels", d=12))
    c.min_coarse_blocks = int(h("min_coarse_blocks", d=4))
    c.wall_model_enabled = bool(h("wall_model", "enabled", d=False))
    c.wall_model_type = str(h("wall_model", "type", d="equilibrium"))
    c.wall_model_yplus_target = float(h("wall_model", "y_plus_target", d=30.0))
    dm = lambda k, d: safe_get(cfg, "advanced", "domain", k, default=d)  # noqa: E731
    c.domain_upstream = float(dm("upstream", 0.75))
    c.domain_downstream = float(dm("downstream", 1.5))
    c.domain_lateral = float(dm("lateral", 0.75))
    c.domain_height = float(dm("height", 0.75))
    c.sponge_thickness = f32(dm("sponge_thickness", 0.10))
    r = lambda k, d: safe_get(cfg, "advanced", "refinement", k, default=d)  # noqa: E731
    c.block_size = int(r("block_size", 8))
    if c.block_size != 8:
        raise ConfigError("block_size must be 8 (the kernels are built for 8^3 blocks)")
    c.refinement_margin = int(r("margin", 2))
    c.refinement_strategy = str(r("strategy", "geometry_first"))
    c.wake_enabled = bool(r("wake_enabled", False))
    c.wake_length = float(r("wake_length", 0.25))
    c.wake_width_factor = float(r("wake_width_factor", 0.1))
    c.wake_height_factor = float(r("wake_height_factor", 0.1))
    c.boundary_method = str(safe_get(cfg, "advanced", "boundary", "method", default="bouzidi"))
    c.bouzidi_levels = int(safe_get(cfg, "advanced", "boundary", "bouzidi_levels", default=1))
    c.q_min_threshold = f32(safe_get(cfg, "advanced", "boundary", "q_min_threshold", default=0.001))
    c.forces_enabled = bool(safe_get(cfg, "advanced", "forces", "enabled", default=True))
    c.force_output_freq_config = int(safe_get(cfg, "advanced", "forces", "output_freq", default=0))
    c.moment_center = list(safe_get(cfg, "advanced", "forces", "moment_center", default=[0.25, 0.0, 0.0]))
    c.net_force_export = bool(safe_get(cfg, "advanced", "forces", "net_force_export", default=False))
    c.diag_freq = int(safe_get(cfg, "advanced", "diagnostics", "freq", default=500))
    c.async_depth = int(safe_get(cfg, "advanced", "gpu", "async_depth", default=8))
    return c


def load_case_configuration(case_dir: str | Path) -> CaseConfig:
    """Load ``<case_dir>/config.yaml`` (config_loader.jl:133-141)."""
    d = Path(case_dir)
    if not d.is_dir():
        raise ConfigError(f"Case folder not found: {d}")
    p = d / "config.yaml"
    if not p.is_file():
        raise ConfigError(f"config.yaml not found: {p}")
    with open(p) as fh:
        cfg = yaml.safe_load(fh)
    return config_from_dict(cfg, str(d))


def load_case_list(list_file: str | Path) -> list[str]:
    """``cases_to_run.yaml`` -> case folder names (main.jl:413-420)."""
    with open(list_file) as fh:
        d = yaml.safe_load(fh) or {}
    return [str(x) for x in (d.get("case_folders") or [])]


def steps_from_domain_length(cfg: CaseConfig, domain_x_phys: float, u_physical: float,
                             time_scale: float) -> int:
    """main.jl:79-89: steps for ``domain_length_covered`` traversals, rounded up
    to a multiple of the diagnostics period."""
    t_needed = cfg.domain_length_covered * domain_x_phys / u_physical
    n = int(math.ceil(t_needed / time_scale))
    return int(math.ceil(n / cfg.diag_freq)) * cfg.diag_freq
