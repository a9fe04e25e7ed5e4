"""Generate tests/golden/reference_cases.json from the reference's own case
data (CASES/<case>/config.yaml and the STL it names).

The reference ships no tests or golden vectors for the solver path; its case
folders are the only reference-produced inputs.  This script reads them where
the reference is mounted and records what the reference's loaders produce
from them: the configuration values config_loader.jl:133-281 would set (the
expected values below were read off the YAML text and the defaults in
config_loader.jl:5-119), the facet count and bounds of the parsed STL
(geometry.jl:385-429) and the triangle count after longest-edge subdivision
(geometry.jl:174-258).  Run it from the repository root, naming the
reference checkout as the argument or in OL_REFERENCE_ROOT:

    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from openludwig_b200 import config, geometry  # noqa: E402

CASES = ["cube1m_Re1e3", "ball1m_Re1e3"]
KEYS = ["surface_resolution", "num_levels_config", "cumulant_limiter", "c_wale", "u_target",
        "minimum_facet_size", "tau_min", "collision_operator", "domain_upstream",
        "domain_downstream", "domain_lateral", "domain_height", "refinement_margin",
        "wake_enabled", "boundary_method", "bouzidi_levels", "q_min_threshold", "diag_freq",
        "ramp_steps", "flow_velocity", "fluid_kinematic_viscosity", "reference_area_config",
        "compressibility_correction", "ddf_enabled", "cumulant_adaptive_omega4",
        "cumulant_lambda_param", "inlet_turbulence_intensity", "temporal_interpolation",
        "domain_length_covered"]


def main(ref: str) -> None:
    out = {"source": "reference CASES folders", "cases": {}}
    for name in CASES:
        case_dir = Path(ref) / "CASES" / name
        c = config.load_case_configuration(case_dir)
        m = geometry.load_mesh(c.stl_files[0], c.stl_scale, 0.0)
        entry = {"config": {k: getattr(c, k) for k in KEYS},
                 "stl": {"file": Path(c.stl_files[0]).name, "n_triangles": m.n,
                         "min_bounds": list(m.min_bounds), "max_bounds": list(m.max_bounds),
                         "area": float(m.areas.sum())}}
        if c.minimum_facet_size > 0 and m.n < 100:
            entry["stl"]["n_after_subdivision"] = geometry.subdivide_mesh(m, c.minimum_facet_size).n
        out["cases"][name] = entry
    out["case_list_head"] = config.load_case_list(Path(ref) / "cases_to_run.yaml")[:4]
    (Path(__file__).parent / "reference_cases.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OL_REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set OL_REFERENCE_ROOT)")
    main(ref)
