"""ctypes binding of libopenludwig_b200.so (the C ABI in include/openludwig_b200.h).

The library is built in-tree by ``openludwig_b200.build``; loading fails
loudly when it is missing -- there is no CPU fallback for the time step.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from .build import library_path

OL_OK = 0
OL_OP_CUMULANT = 0
OL_OP_REGULARIZED_BGK = 1
OL_LIMITER_NONE, OL_LIMITER_FACTORED, OL_LIMITER_POSITIVITY = 0, 1, 2
OL_STORE_F32, OL_STORE_F16, OL_STORE_DDF = 0, 1, 2
OL_GHOST_UNPAIRED, OL_GHOST_PAIR_FIRST, OL_GHOST_PAIR_SECOND = 0, 1, 2

vp = C.c_void_p
i32 = C.c_int32
f32 = C.c_float


class LevelView(C.Structure):
    _fields_ = [("f_out", vp), ("f_in", vp), ("f_post", vp), ("rho", vp), ("vel_out", vp),
                ("vel_in", vp), ("obstacle", vp), ("sponge", vp), ("wall_dist", vp),
                ("neighbor_table", vp), ("map_x", vp), ("map_y", vp), ("map_z", vp),
                ("ghost", vp), ("n_blocks", i32), ("ghost_next", vp), ("ghost_mode", i32),
                ("ghost_blocks", vp), ("n_ghost_blocks", i32)]


class ParentView(C.Structure):
    _fields_ = [("f", vp), ("rho", vp), ("vel", vp), ("f_old", vp), ("rho_old", vp),
                ("vel_old", vp), ("block_ptr", vp), ("dim_x", i32), ("dim_y", i32),
                ("dim_z", i32), ("n_blocks", i32)]


STEP_FIELDS = [("op", i32), ("tau_molecular", f32), ("tau_parent", f32), ("c_wale", f32),
               ("nu_sgs_background", f32), ("is_level_1", i32), ("is_symmetric", i32),
               ("nx_global", i32), ("ny_global", i32), ("nz_global", i32), ("u_inlet", f32),
               ("wall_model_active", i32), ("time_step_seed", i32),
               ("store_post_collision", i32), ("inlet_turbulence", f32),
               ("temporal_weight", f32), ("use_temporal_interp", i32),
               ("sponge_blend_distributions", i32), ("omega_bulk", f32), ("omega_3", f32),
               ("omega_4", f32), ("adaptive_omega4", i32), ("lambda_param", f32),
               ("limiter_type", i32), ("compressible_corr", i32)]


class StepParams(C.Structure):
    _fields_ = STEP_FIELDS


class ThermalView(C.Structure):
    _fields_ = [("g_out", vp), ("g_in", vp), ("g_post", vp), ("temperature", vp), ("vel", vp),
                ("obstacle", vp), ("sponge", vp), ("neighbor_table", vp), ("map_x", vp),
                ("map_y", vp), ("map_z", vp), ("n_blocks", i32),
                ("pg", vp), ("pT", vp), ("pvel", vp), ("pg_old", vp), ("pT_old", vp),
                ("pvel_old", vp), ("p_block_ptr", vp), ("p_dim_x", i32), ("p_dim_y", i32),
                ("p_dim_z", i32), ("p_n_blocks", i32), ("ghost", vp), ("ghost_next", vp),
                ("ghost_mode", i32), ("ghost_blocks", vp), ("n_ghost_blocks", i32)]


THERMAL_FIELDS = [("tau_g", f32), ("tau_g_parent", f32), ("is_level_1", i32),
                  ("is_symmetric", i32), ("nx_global", i32), ("ny_global", i32),
                  ("nz_global", i32), ("u_inlet", f32), ("T_inlet", f32), ("T_wall", f32),
                  ("wall_bc_adiabatic", i32), ("store_post_collision", i32),
                  ("temporal_weight", f32), ("use_temporal_interp", i32),
                  ("sponge_blend_distributions", i32)]


class ThermalParams(C.Structure):
    _fields_ = THERMAL_FIELDS


class RestrictView(C.Structure):
    _fields_ = [("f_fine", vp), ("obstacle_fine", vp), ("map_x", vp), ("map_y", vp),
                ("map_z", vp), ("n_fine", i32), ("f_coarse", vp), ("rho_coarse", vp),
                ("vel_coarse", vp), ("obstacle_coarse", vp), ("block_ptr", vp), ("dim_x", i32),
                ("dim_y", i32), ("dim_z", i32), ("n_coarse", i32), ("tau_fine", f32),
                ("tau_coarse", f32), ("compressible", i32)]


class FeMapView(C.Structure):
    _fields_ = [("node_xyz", vp), ("tri_xyz", vp), ("tri_force", vp), ("node_begin", vp),
                ("tri_begin", vp), ("n_nodes", i32), ("n_tris", i32), ("n_objects", i32),
                ("tri_nodes", vp), ("tri_node_force", vp), ("nodal_force", vp), ("scratch", vp)]


class SurfaceMesh(C.Structure):
    _fields_ = [("cx", vp), ("cy", vp), ("cz", vp), ("nx", vp), ("ny", vp), ("nz", vp),
                ("area", vp), ("n_triangles", i32)]


class NetForceMaps(C.Structure):
    _fields_ = [("p_plus", vp), ("sx_plus", vp), ("sy_plus", vp), ("sz_plus", vp),
                ("p_minus", vp), ("sx_minus", vp), ("sy_minus", vp), ("sz_minus", vp),
                ("net_fx", vp), ("net_fy", vp), ("net_fz", vp)]


class BouzidiLink(C.Structure):
    _fields_ = [("cell", i32), ("far_cell", i32), ("q", f32), ("k", i32)]


class OutputLevel(C.Structure):
    _fields_ = [("rho", vp), ("vel", vp), ("obstacle", vp), ("temperature", vp), ("map_x", vp),
                ("map_y", vp), ("map_z", vp), ("blocks", vp), ("n_export", i32),
                ("n_blocks", i32), ("level_id", i32), ("dx", f32)]


class OutputFields(C.Structure):
    _fields_ = [("points", vp), ("rho", vp), ("vel", vp), ("vel_mag", vp), ("obstacle", vp),
                ("level", vp), ("temperature", vp)]


class ForceParams(C.Structure):
    _fields_ = [("dx", f32), ("dim_x", i32), ("dim_y", i32), ("dim_z", i32),
                ("offset_x", f32), ("offset_y", f32), ("offset_z", f32),
                ("pressure_scale", f32), ("stress_scale", f32), ("tau_molecular", f32),
                ("search_radius", i32), ("c_wale", f32), ("nu_sgs_bg", f32),
                ("ref_x", f32), ("ref_y", f32), ("ref_z", f32)]


class LevelDesc(C.Structure):
    _fields_ = [("n_blocks", i32), ("map_x", vp), ("map_y", vp), ("map_z", vp),
                ("neighbor_table", vp), ("block_ptr", vp), ("dim_x", i32), ("dim_y", i32),
                ("dim_z", i32), ("obstacle", vp), ("sponge", vp), ("wall_dist", vp),
                ("n_boundary", i32), ("q_map", vp), ("cell_block", vp), ("cell_x", vp),
                ("cell_y", vp), ("cell_z", vp), ("tau", f32), ("tau_g", f32),
                ("store_scale", f32)]


class CaseDesc(C.Structure):
    _fields_ = [("n_levels", i32), ("levels", C.POINTER(LevelDesc)), ("nx", i32), ("ny", i32),
                ("nz", i32), ("params", StepParams), ("ddf", i32), ("tparams", ThermalParams),
                ("n_triangles", i32), ("tri_cx", vp), ("tri_cy", vp), ("tri_cz", vp),
                ("tri_nx", vp), ("tri_ny", vp), ("tri_nz", vp), ("tri_area", vp),
                ("force", ForceParams), ("u_target", f32), ("ramp_steps", i32),
                ("async_depth", i32), ("q_min_threshold", f32), ("T_initial", f32)]


class CoeffRef(C.Structure):
    _fields_ = [("rho_ref", C.c_double), ("u_ref", C.c_double), ("area_ref", C.c_double),
                ("chord_ref", C.c_double), ("symmetric", i32)]


class ServeRule(C.Structure):
    _fields_ = [("check_every", i32), ("window", i32), ("tol", C.c_double),
                ("max_steps", i32), ("min_steps", i32)]


class ServeResult(C.Structure):
    _fields_ = [("rid", i32), ("steps", i32), ("status", i32), ("converged", i32),
                ("arrival_s", C.c_double), ("admit_s", C.c_double), ("finish_s", C.c_double),
                ("coeff", C.c_double * 12)]


OL_SC_KERNEL_AUTO, OL_SC_KERNEL_BLOCK, OL_SC_KERNEL_WS = 0, 1, 2
OL_LAUNCH_WS, OL_LAUNCH_PIPELINED, OL_LAUNCH_PER_ITEM = -2, -1, 0


class OLError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


_LIB: C.CDLL | None = None

# name -> (restype, argtypes)
_SIGS = {
    "ol_stream_collide": (C.c_int, [C.POINTER(LevelView), C.POINTER(ParentView),
                                    C.POINTER(StepParams), vp]),
    "ol_bouzidi": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, i32, vp, i32, f32, vp]),
    "ol_bouzidi_sparse": (C.c_int, [vp, vp, vp, vp, vp, vp, i32, vp, i32, f32, vp, vp]),
    "ol_bouzidi_sparse_noalloc": (C.c_int, [vp, vp, vp, vp, vp, vp, i32, vp, i32, f32, vp]),
    "ol_bouzidi_build_links": (C.c_int, [vp, vp, vp, vp, vp, i32, vp, i32, f32, vp, vp, vp]),
    "ol_bouzidi_apply_links": (C.c_int, [vp, vp, i32, i32, vp, vp]),
    "ol_thermal": (C.c_int, [C.POINTER(ThermalView), C.POINTER(ThermalParams), vp]),
    "ol_restrict": (C.c_int, [C.POINTER(RestrictView), vp]),
    "ol_voxelize": (C.c_int, [vp, i32, vp, i32, vp, vp, C.c_double, C.POINTER(C.c_double), vp,
                              vp]),
    "ol_bouzidi_qmap": (C.c_int, [vp, i32, vp, i32, vp, vp, C.c_double, C.POINTER(C.c_double),
                                  vp, vp, vp, vp]),
    "ol_init_equilibrium": (C.c_int, [vp, vp, vp, vp, vp, i32, vp]),
    "ol_surface_forces": (C.c_int, [C.POINTER(SurfaceMesh), vp, vp, vp, vp, i32,
                                    C.POINTER(ForceParams), vp, vp, vp, vp, vp,
                                    C.POINTER(C.c_double), vp]),
    "ol_surface_forces_scratch_doubles": (C.c_size_t, [i32]),
    "ol_surface_net_forces": (C.c_int, [C.POINTER(SurfaceMesh), vp, vp, vp, vp, i32,
                                        C.POINTER(ForceParams), i32, C.POINTER(NetForceMaps),
                                        vp]),
    "ol_flow_stats": (C.c_int, [vp, vp, vp, i32, vp, C.POINTER(C.c_double), vp]),
    "ol_flow_stats_scratch_doubles": (C.c_size_t, [i32]),
    "ol_flow_stats_device": (C.c_int, [vp, vp, vp, i32, vp, vp, vp]),
    "ol_pack_merged_fields": (C.c_int, [C.POINTER(OutputLevel), i32, C.POINTER(OutputFields), vp]),
    "ol_ghost_floats": (C.c_int64, [i32]),
    "ol_ctx_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_size_t, C.c_int]),
    "ol_ctx_destroy": (C.c_int, [vp]),
    "ol_ctx_case_footprint": (C.c_int, [vp, C.POINTER(CaseDesc), C.POINTER(C.c_size_t)]),
    "ol_ctx_case_add": (C.c_int, [vp, C.POINTER(CaseDesc), C.POINTER(i32)]),
    "ol_ctx_case_remove": (C.c_int, [vp, i32]),
    "ol_ctx_step": (C.c_int, [vp, i32]),
    "ol_ctx_sync": (C.c_int, [vp]),
    "ol_ctx_step_timed": (C.c_int, [vp, i32, C.POINTER(C.c_float)]),
    "ol_ctx_case_forces": (C.c_int, [vp, i32, C.POINTER(C.c_double)]),
    "ol_ctx_case_download": (C.c_int, [vp, i32, i32, vp, vp, vp]),
    "ol_ctx_case_download_thermal": (C.c_int, [vp, i32, i32, vp, vp]),
    "ol_ctx_case_info": (C.c_int, [vp, i32, C.POINTER(C.c_int64), C.POINTER(i32)]),
    "ol_ctx_autotune": (C.c_int, [vp, i32]),
    "ol_ctx_set_launch": (C.c_int, [vp, i32]),
    "ol_ctx_get_launch": (C.c_int, [vp, C.POINTER(i32)]),
    "ol_ctx_get_variant_launch": (C.c_int, [vp, i32, i32, i32, C.POINTER(i32)]),
    "ol_ctx_case_step": (C.c_int, [vp, i32, i32, f32]),
    "ol_ctx_case_coefficients": (C.c_int, [vp, i32, C.POINTER(CoeffRef), C.POINTER(C.c_double)]),
    "ol_set_stream_collide_kernel": (C.c_int, [i32, i32]),
    "ol_pipeline_fault": (C.c_int, [C.POINTER(i32)]),
    "ol_staging_tables": (C.c_int, [vp, i32, vp, i32, C.POINTER(i32)]),
    "ol_server_create": (C.c_int, [C.POINTER(vp), vp, C.POINTER(ServeRule)]),
    "ol_server_destroy": (C.c_int, [vp]),
    "ol_server_clock": (C.c_int, [vp, C.POINTER(C.c_double)]),
    "ol_serve_submit": (C.c_int, [vp, C.POINTER(CaseDesc), C.POINTER(CoeffRef), C.c_double,
                                  C.POINTER(i32)]),
    "ol_serve_advance": (C.c_int, [vp, C.POINTER(i32), C.POINTER(i32)]),
    "ol_serve_poll": (C.c_int, [vp, C.POINTER(ServeResult), i32, C.POINTER(i32)]),
    "ol_serve_history": (C.c_int, [vp, i32, C.POINTER(C.c_double), i32, C.POINTER(i32)]),
    "ol_ctx_stats": (C.c_int, [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                               C.POINTER(i32), C.POINTER(C.c_int64)]),
    "ol_fe_map_scratch_bytes": (C.c_size_t, [i32]),
    "ol_fe_map_forces": (C.c_int, [C.POINTER(FeMapView), C.POINTER(i32), vp]),
    "ol_last_error": (C.c_char_p, []),
    "ol_version": (C.c_char_p, []),
}


def lib() -> C.CDLL:
    """Load the library (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is None:
        path = Path(library_path())
        if not path.exists():
            raise RuntimeError(
                f"{path} is missing: build it with `python -m openludwig_b200.build` "
                "(the CUDA path has no fallback)")
        L = C.CDLL(str(path))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(fn_name: str, rc: int) -> None:
    if rc != OL_OK:
        msg = lib().ol_last_error().decode(errors="replace")
        raise OLError(fn_name, rc, msg)


def call(fn_name: str, *args) -> None:
    check(fn_name, getattr(lib(), fn_name)(*args))
