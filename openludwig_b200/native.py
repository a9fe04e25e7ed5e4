"""Native multi-case context (ol_ctx_* in the C ABI): a device block pool with
FP32 or FP16-shifted population storage, persistent batched kernels, and a
coarse step replayed from a CUDA graph for every resident case.

    ctx = Context(budget_bytes=8 << 30, storage="f16")
    cid = ctx.add_case(case)          # case = prepare_case(cfg, mesh)
    ctx.step(100); ctx.sync()
    f = ctx.forces(cid)               # ForceResult with Cd, Cl, Cs, Cm...
    ctx.remove_case(cid)
"""
from __future__ import annotations

import ctypes as C
import dataclasses as dc

import numpy as np

from . import _native as N
from .config import CaseConfig
from .domain import HostLevel, setup_multilevel_domain
from .geometry import SolverMesh
from .scaling import DomainParams, compute_domain_from_mesh
from .solver import StepSettings

# FP16 shift scale per level: stored value = binary16((f - w) * scale / w).
# A power of two keeps the encode/decode exact apart from the binary16
# rounding; 256 keeps relative deviations of 1e-6..255 in the normal range.
DEFAULT_F16_SCALE = 256.0


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dc.dataclass
class PreparedCase:
    """Host-side description of a case, ready for Context.add_case."""
    cfg: CaseConfig
    mesh: SolverMesh
    params: DomainParams
    levels: list
    settings: StepSettings
    name: str = ""

    @property
    def cell_updates_per_step(self) -> int:
        return sum(h.n_blocks * 512 * (1 << i) for i, h in enumerate(self.levels))

    @property
    def cells(self) -> int:
        return sum(h.n_blocks * 512 for h in self.levels)


def prepare_case(cfg: CaseConfig, mesh: SolverMesh, name: str = "",
                 device: int | None = None) -> PreparedCase:
    """Domain scaling + multi-level domain build; device: CUDA device for the
    voxelisation and Bouzidi q-map (None = all on the host)."""
    p = compute_domain_from_mesh(cfg, mesh.min_bounds, mesh.max_bounds)
    hosts = setup_multilevel_domain(cfg, mesh, p, device=device)
    st = StepSettings.from_config(cfg, cfg.wall_model_enabled)
    return PreparedCase(cfg, mesh, p, hosts, st, name)


@dc.dataclass
class ForceResult:
    """integrate_surface_forces! outputs (surface.jl:828-910)."""
    Fx_p: float
    Fy_p: float
    Fz_p: float
    Fx_v: float
    Fy_v: float
    Fz_v: float
    Mx: float
    My: float
    Mz: float
    Cd: float = 0.0
    Cl: float = 0.0
    Cs: float = 0.0
    Cmx: float = 0.0
    Cmy: float = 0.0
    Cmz: float = 0.0


def coefficients(raw, rho_ref, u_ref, area_ref, chord_ref, symmetric=False) -> ForceResult:
    """Symmetry doubling and Cd/Cl/Cs/Cm (surface.jl:873-910)."""
    Fx_p, Fy_p, Fz_p, Fx_v, Fy_v, Fz_v, Mx, My, Mz = (float(v) for v in raw)
    if symmetric:
        Fx_p *= 2.0; Fz_p *= 2.0; Fx_v *= 2.0; Fz_v *= 2.0; My *= 2.0
        Fy_p = Fy_v = 0.0
        Mx = Mz = 0.0
    r = ForceResult(Fx_p, Fy_p, Fz_p, Fx_v, Fy_v, Fz_v, Mx, My, Mz)
    q_inf = 0.5 * rho_ref * u_ref ** 2
    F_ref = q_inf * area_ref
    M_ref = F_ref * chord_ref
    Fx, Fy, Fz = Fx_p + Fx_v, Fy_p + Fy_v, Fz_p + Fz_v
    if F_ref > 1e-10:
        r.Cd, r.Cl, r.Cs = Fx / F_ref, Fz / F_ref, Fy / F_ref
    if M_ref > 1e-10:
        r.Cmx, r.Cmy, r.Cmz = Mx / M_ref, My / M_ref, Mz / M_ref
    return r


def coeff_ref(case: PreparedCase) -> N.CoeffRef:
    """Reference values of a case's force coefficients (surface.jl:873-910)."""
    p = case.params
    return N.CoeffRef(rho_ref=p.rho_physical, u_ref=p.u_physical, area_ref=p.reference_area,
                      chord_ref=p.reference_chord, symmetric=int(bool(case.cfg.symmetric_analysis)))


COEFF_NAMES = ("Cd", "Cl", "Cs", "Cmx", "Cmy", "Cmz", "Fx", "Fy", "Fz", "Mx", "My", "Mz")


def force_params(case: PreparedCase, search_radius: int = 5) -> N.ForceParams:
    """map_surface_stresses! scalars (surface.jl:766-790) on the finest level."""
    p, cfg = case.params, case.cfg
    fin: HostLevel = case.levels[-1]
    vs = p.velocity_scale
    ps = float(np.float32(p.rho_physical * vs * vs))
    mc = p.moment_center
    off = p.mesh_offset
    return N.ForceParams(dx=float(np.float32(fin.dx)), dim_x=fin.grid_dim[0], dim_y=fin.grid_dim[1],
                         dim_z=fin.grid_dim[2], offset_x=off[0], offset_y=off[1], offset_z=off[2],
                         pressure_scale=ps, stress_scale=ps, tau_molecular=fin.tau,
                         search_radius=search_radius, c_wale=cfg.c_wale,
                         nu_sgs_bg=cfg.nu_sgs_background, ref_x=mc[0], ref_y=mc[1], ref_z=mc[2])


class _CaseKeep:
    """Keeps the numpy buffers referenced by an ol_case_desc alive."""

    def __init__(self):
        self.arrays = []

    def keep(self, a):
        a = np.ascontiguousarray(a)
        self.arrays.append(a)
        return _p(a)


def build_case_desc(case: PreparedCase, f16_scale: float = DEFAULT_F16_SCALE):
    keep = _CaseKeep()
    cfg, p, st = case.cfg, case.params, case.settings
    lv = (N.LevelDesc * len(case.levels))()
    for i, h in enumerate(case.levels):
        d = lv[i]
        d.n_blocks = h.n_blocks
        d.map_x, d.map_y, d.map_z = keep.keep(h.map_x), keep.keep(h.map_y), keep.keep(h.map_z)
        d.neighbor_table = keep.keep(h.neighbor_table)
        d.block_ptr = keep.keep(h.block_ptr)
        d.dim_x, d.dim_y, d.dim_z = h.grid_dim
        d.obstacle = keep.keep(h.obstacle)
        d.sponge = keep.keep(h.sponge)
        d.wall_dist = keep.keep(h.wall_dist)
        d.n_boundary = h.n_boundary if h.bouzidi else 0
        if d.n_boundary:
            d.q_map = keep.keep(h.q_map)
            d.cell_block = keep.keep(h.cell_block)
            d.cell_x, d.cell_y, d.cell_z = keep.keep(h.cell_x), keep.keep(h.cell_y), keep.keep(h.cell_z)
        d.tau = h.tau
        d.tau_g = h.tau_g if h.tau_g else 0.5
        d.store_scale = f16_scale * (1 << i)
    cd = N.CaseDesc()
    cd.n_levels = len(case.levels)
    cd.levels = C.cast(lv, C.POINTER(N.LevelDesc))
    keep.arrays.append(lv)
    cd.nx, cd.ny, cd.nz = p.nx_coarse, p.ny_coarse, p.nz_coarse
    sp = cd.params
    sp.op = st.op
    sp.c_wale = st.c_wale
    sp.nu_sgs_background = st.nu_sgs_bg
    sp.is_symmetric = st.is_symmetric
    sp.wall_model_active = st.wall_model
    sp.inlet_turbulence = st.inlet_turbulence
    sp.use_temporal_interp = st.use_temporal_interp
    sp.sponge_blend_distributions = st.sponge_blend
    sp.omega_bulk, sp.omega_3, sp.omega_4 = st.omega_bulk, st.omega_3, st.omega_4
    sp.adaptive_omega4 = st.adaptive_omega4
    sp.lambda_param = st.lambda_param
    sp.limiter_type = st.limiter
    sp.compressible_corr = st.compressible
    cd.ddf = st.ddf
    tp = cd.tparams
    tp.is_symmetric = st.is_symmetric
    tp.T_inlet, tp.T_wall = st.t_inlet, st.t_wall
    tp.wall_bc_adiabatic = st.wall_bc_adiabatic
    tp.use_temporal_interp = st.use_temporal_interp
    tp.sponge_blend_distributions = st.sponge_blend
    m = case.mesh
    cd.n_triangles = m.n if cfg.forces_enabled else 0
    if cd.n_triangles:
        cen, nrm, area = m.centers.astype(np.float32), m.normals.astype(np.float32), m.areas.astype(np.float32)
        cd.tri_cx, cd.tri_cy, cd.tri_cz = keep.keep(cen[:, 0]), keep.keep(cen[:, 1]), keep.keep(cen[:, 2])
        cd.tri_nx, cd.tri_ny, cd.tri_nz = keep.keep(nrm[:, 0]), keep.keep(nrm[:, 1]), keep.keep(nrm[:, 2])
        cd.tri_area = keep.keep(area)
    cd.force = force_params(case)
    cd.u_target = cfg.u_target
    cd.ramp_steps = cfg.ramp_steps
    cd.async_depth = cfg.async_depth
    cd.q_min_threshold = cfg.q_min_threshold
    cd.T_initial = cfg.ddf_t_initial
    return cd, keep


class Context:
    """One device, one block pool, many cases advanced together."""

    def __init__(self, device: int = 0, budget_bytes: int = 4 << 30, storage: str = "f16",
                 ddf: bool = False, f16_scale: float = DEFAULT_F16_SCALE):
        kind = (N.OL_STORE_F16 if storage == "f16" else N.OL_STORE_F32) | (2 if ddf else 0)
        self._h = C.c_void_p()
        N.call("ol_ctx_create", C.byref(self._h), device, C.c_size_t(budget_bytes), kind)
        self.storage = storage
        self.f16_scale = f16_scale
        self.cases: dict[int, PreparedCase] = {}

    def close(self) -> None:
        if self._h:
            N.call("ol_ctx_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def footprint(self, case: PreparedCase) -> int:
        cd, keep = build_case_desc(case, self.f16_scale)
        out = C.c_size_t()
        N.call("ol_ctx_case_footprint", self._h, C.byref(cd), C.byref(out))
        return int(out.value)

    def add_case(self, case: PreparedCase) -> int:
        cd, keep = build_case_desc(case, self.f16_scale)
        cid = C.c_int32()
        N.call("ol_ctx_case_add", self._h, C.byref(cd), C.byref(cid))
        self.cases[cid.value] = case
        return cid.value

    def remove_case(self, cid: int) -> None:
        N.call("ol_ctx_case_remove", self._h, cid)
        self.cases.pop(cid, None)

    def step(self, n: int = 1) -> None:
        N.call("ol_ctx_step", self._h, n)

    def step_timed(self, n: int) -> float:
        """Advance n coarse steps; device milliseconds from CUDA events."""
        ms = C.c_float()
        N.call("ol_ctx_step_timed", self._h, n, C.byref(ms))
        return float(ms.value)

    def sync(self) -> None:
        N.call("ol_ctx_sync", self._h)

    def forces_raw(self, cid: int) -> np.ndarray:
        out = (C.c_double * 9)()
        N.call("ol_ctx_case_forces", self._h, cid, out)
        return np.array(out[:], dtype=np.float64)

    def forces(self, cid: int) -> ForceResult:
        case = self.cases[cid]
        p = case.params
        return coefficients(self.forces_raw(cid), p.rho_physical, p.u_physical, p.reference_area,
                            p.reference_chord, case.cfg.symmetric_analysis)

    def coefficient_record(self, cid: int) -> dict:
        """ol_ctx_case_coefficients: Cd, Cl, Cs, Cmx..z and the total forces
        and moments of a case, computed by the library."""
        out = (C.c_double * 12)()
        ref = coeff_ref(self.cases[cid])
        N.call("ol_ctx_case_coefficients", self._h, cid, C.byref(ref), out)
        return dict(zip(COEFF_NAMES, out[:]))

    def case_step(self, cid: int, n: int, u_in: float = -1.0) -> None:
        """Advance one case alone (ol_ctx_case_step); u_in >= 0 fixes its
        inlet speed from now on."""
        N.call("ol_ctx_case_step", self._h, cid, n, u_in)

    def download(self, cid: int, level: int = 1, f: bool = False):
        h = self.cases[cid].levels[level - 1]
        n = h.n_blocks * 512
        rho = np.empty(n, np.float32)
        vel = np.empty(3 * n, np.float32)
        ff = np.empty(27 * n, np.float32) if f else None
        N.call("ol_ctx_case_download", self._h, cid, level, _p(rho), _p(vel), _p(ff))
        return rho, vel, ff

    def download_thermal(self, cid: int, level: int = 1, g: bool = False):
        """Temperature (and decoded thermal populations) of a DDF case."""
        h = self.cases[cid].levels[level - 1]
        n = h.n_blocks * 512
        T = np.empty(n, np.float32)
        gg = np.empty(27 * n, np.float32) if g else None
        N.call("ol_ctx_case_download_thermal", self._h, cid, level, _p(T), _p(gg))
        return T, gg

    def info(self, cid: int) -> tuple[int, int]:
        steps = C.c_int64()
        status = C.c_int32()
        N.call("ol_ctx_case_info", self._h, cid, C.byref(steps), C.byref(status))
        return int(steps.value), int(status.value)

    def autotune(self, trials: int = 3) -> None:
        N.call("ol_ctx_autotune", self._h, trials)

    def set_launch(self, shape: int) -> None:
        """Launch shape of the stream-collide launches (OL_LAUNCH_*, 1, 2)."""
        N.call("ol_ctx_set_launch", self._h, shape)

    def launch(self) -> int:
        out = C.c_int32()
        N.call("ol_ctx_get_launch", self._h, C.byref(out))
        return int(out.value)

    def variant_launch(self, op: int, wale: bool, ddf: bool = False) -> int:
        """Launch shape of one collision variant's stream-collide launches."""
        out = C.c_int32()
        N.call("ol_ctx_get_variant_launch", self._h, op, int(bool(wale)), int(bool(ddf)),
               C.byref(out))
        return int(out.value)

    def stats(self) -> dict:
        used, budget = C.c_size_t(), C.c_size_t()
        n, launches = C.c_int32(), C.c_int64()
        N.call("ol_ctx_stats", self._h, C.byref(used), C.byref(budget), C.byref(n), C.byref(launches))
        return {"used": used.value, "budget": budget.value, "cases": n.value,
                "launches": launches.value}
