"""The C-ABI library builds for sm_100a, loads without a GPU, and exports every
function declared in include/*.h (no compute calls: this runs on CPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"OL_API\s+[\w\s\*]*?\b(ol_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from openludwig_b200 import build
    path = build.build()
    return ctypes.CDLL(str(path))


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("ol_stream_collide", "ol_bouzidi", "ol_bouzidi_sparse", "ol_thermal",
                     "ol_surface_forces", "ol_init_equilibrium", "ol_flow_stats",
                     "ol_ctx_create", "ol_ctx_step", "ol_last_error",
                     # per-case control and the coefficient record
                     "ol_ctx_case_step", "ol_ctx_case_coefficients",
                     # serving through the C ABI
                     "ol_server_create", "ol_serve_submit", "ol_serve_advance", "ol_serve_poll",
                     "ol_serve_history", "ol_server_destroy",
                     # kernel and launch-shape control
                     "ol_set_stream_collide_kernel", "ol_ctx_set_launch", "ol_pipeline_fault"):
        assert required in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert missing == []


def test_version_and_error_string_without_gpu(lib):
    lib.ol_version.restype = ctypes.c_char_p
    lib.ol_last_error.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.ol_version()
    assert isinstance(lib.ol_last_error(), bytes)


def test_argument_errors_are_reported_not_raised(lib):
    """Null views are rejected with OL_ERR_ARG before any CUDA call."""
    lib.ol_stream_collide.restype = ctypes.c_int
    rc = lib.ol_stream_collide(None, None, None, None)
    assert rc == 1
    lib.ol_last_error.restype = ctypes.c_char_p
    assert b"null" in lib.ol_last_error()
    lib.ol_ctx_create.restype = ctypes.c_int
    assert lib.ol_ctx_create(None, 0, ctypes.c_size_t(1 << 20), 0) == 1
    # serving and per-case entry points check their arguments first too
    assert lib.ol_server_create(None, None, None) == 1
    assert lib.ol_serve_submit(None, None, None, ctypes.c_double(0.0), None) == 1
    assert lib.ol_serve_advance(None, None, None) == 1
    assert lib.ol_ctx_case_step(None, 0, 1, ctypes.c_float(-1.0)) == 1
    assert lib.ol_ctx_case_coefficients(None, 0, None, None) == 1
    assert lib.ol_set_stream_collide_kernel(7, 0) == 1
    assert lib.ol_fe_map_forces(None, None, None) == 1


def test_ctypes_struct_layouts_match_header(tmp_path):
    """Every POD struct of the ABI has the same size in C and in the binding."""
    import shutil
    import subprocess
    import sys
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    sys.path.insert(0, str(ROOT))
    from openludwig_b200 import _native as N
    names = {"ol_case_desc": N.CaseDesc, "ol_level_desc": N.LevelDesc,
             "ol_step_params": N.StepParams, "ol_thermal_params": N.ThermalParams,
             "ol_force_params": N.ForceParams, "ol_level_view": N.LevelView,
             "ol_parent_view": N.ParentView, "ol_thermal_view": N.ThermalView,
             "ol_surface_mesh": N.SurfaceMesh, "ol_restrict_view": N.RestrictView,
             "ol_net_force_maps": N.NetForceMaps, "ol_output_level": N.OutputLevel,
             "ol_output_fields": N.OutputFields, "ol_bouzidi_link": N.BouzidiLink,
             "ol_coeff_ref": N.CoeffRef, "ol_serve_rule": N.ServeRule,
             "ol_serve_result": N.ServeResult, "ol_fe_map_view": N.FeMapView}
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "openludwig_b200.h"\nint main(void){\n' +
                   "".join(f'printf("%zu\\n", sizeof({n}));\n' for n in names) + "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert [int(v) for v in out] == [ctypes.sizeof(t) for t in names.values()]
