"""Device-resident levels and the time-step driver, mirroring the reference's
solver path through the C ABI:

  perform_timestep_v2!   (collision/timestep.jl:1-159)  -> perform_timestep
  recursive_step!        (solver/solver_control.jl:6-98) -> recursive_step
  execute_timestep_batch! (solver_control.jl:199-218)   -> execute_timestep_batch
  main.jl:208-315 loop (ramp, diagnostics, forces)      -> Simulation.run

Buffers are torch CUDA tensors in the reference layout; every kernel is a
call into libopenludwig_b200.so on the current torch stream.  There is no
CPU fallback: without a CUDA device or the built library the calls raise.

Differences from the reference that do not change results:
  * copy_to_old! (blocks.jl:241-252) copies f_in and vel_in before a parent
    step; the children only read that state while the parent's f_in is
    untouched, so f_old / vel_old alias f_in / vel_in and only rho (which the
    step overwrites in place) is copied.
  * Bouzidi runs in the sparse two-phase form (gather corrected links, then
    scatter) over the level's static list of cut links, so the dense
    post-collision copy f_post is never written.
"""
from __future__ import annotations

import ctypes as C
import dataclasses as dc
import math

import numpy as np
import torch

from . import _native as N
from .config import CaseConfig
from .domain import HostLevel
from .scaling import DomainParams

BS = 8


def _ptr(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@dc.dataclass
class DeviceLevel:
    host: HostLevel
    f: torch.Tensor
    f_temp: torch.Tensor
    rho: torch.Tensor
    rho_old: torch.Tensor
    vel: torch.Tensor
    vel_temp: torch.Tensor
    obstacle: torch.Tensor
    sponge: torch.Tensor
    wall_dist: torch.Tensor
    neighbor_table: torch.Tensor
    map_x: torch.Tensor
    map_y: torch.Tensor
    map_z: torch.Tensor
    block_ptr: torch.Tensor
    q_map: torch.Tensor | None = None
    cell_block: torch.Tensor | None = None
    cell_x: torch.Tensor | None = None
    cell_y: torch.Tensor | None = None
    cell_z: torch.Tensor | None = None
    bouzidi_scratch: torch.Tensor | None = None
    f_post: torch.Tensor | None = None
    # absent-neighbour pull sources, precomputed by a separate pass (optional)
    ghost: torch.Tensor | None = None
    ghost_g: torch.Tensor | None = None   # the same for the thermal populations
    # second scratch of a refined level: the pair's first sub-step writes the
    # second one's coarse-to-fine values there (ol_level_view.ghost_mode)
    ghost2: torch.Tensor | None = None
    ghost_g2: torch.Tensor | None = None
    # blocks the ghost pass visits: those with an absent neighbour, and those
    # with one not wholly inside the domain (second sub-step of a pair); each
    # list ends with one unused entry
    ghost_list: torch.Tensor | None = None
    edge_list: torch.Tensor | None = None
    # Bouzidi links (cells x directions with q in (q_min, 1]), built once
    bz_links: torch.Tensor | None = None
    bz_n_links: int = 0
    # thermal DDF
    g: torch.Tensor | None = None
    g_temp: torch.Tensor | None = None
    temperature: torch.Tensor | None = None
    temperature_old: torch.Tensor | None = None
    # aliases of the parent state read by the children (set per step)
    f_old: torch.Tensor | None = None
    vel_old: torch.Tensor | None = None
    g_old: torch.Tensor | None = None

    @property
    def n_blocks(self) -> int:
        return self.host.n_blocks

    @property
    def tau(self) -> float:
        return self.host.tau

    @property
    def has_bouzidi(self) -> bool:
        return self.host.bouzidi and self.host.n_boundary > 0


def upload_level(h: HostLevel, device: torch.device, ddf: bool = False, t_init: float = 1.0,
                 reference_bouzidi: bool = False, ghost: bool | None = None) -> DeviceLevel:
    """adapt(backend, g) + the initial state of main.jl:113-173.

    ghost: allocate the level's ol_level_view.ghost scratch, so that the
    boundary values of absent neighbours are evaluated by their own pass
    (identical results).  None = on refined levels only: their level
    interfaces need coarse-to-fine interpolation, which that pass makes
    cheaper; level 1 only has the cheap domain-boundary values."""
    if ghost is None:
        ghost = h.level_id > 1
    n = h.n_blocks
    S = 512 * n
    dev = device
    t = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    f = torch.empty(S * 27, dtype=torch.float32, device=dev)
    ft = torch.empty_like(f)
    rho_old = torch.ones(S, dtype=torch.float32, device=dev)
    vel_old = torch.zeros(S * 3, dtype=torch.float32, device=dev)
    f_old = torch.empty_like(f)
    N.call("ol_init_equilibrium", _ptr(f), _ptr(ft), _ptr(f_old), _ptr(rho_old), _ptr(vel_old),
           N.i32(n), _stream())
    del f_old, vel_old
    lv = DeviceLevel(
        host=h, f=f, f_temp=ft,
        rho=torch.ones(S, dtype=torch.float32, device=dev), rho_old=rho_old,
        vel=torch.zeros(S * 3, dtype=torch.float32, device=dev),
        vel_temp=torch.zeros(S * 3, dtype=torch.float32, device=dev),
        obstacle=t(h.obstacle), sponge=t(h.sponge), wall_dist=t(h.wall_dist),
        neighbor_table=t(h.neighbor_table), map_x=t(h.map_x), map_y=t(h.map_y),
        map_z=t(h.map_z), block_ptr=t(h.block_ptr))
    if h.bouzidi and h.n_boundary > 0:
        lv.q_map = t(h.q_map.view(np.int16))
        lv.cell_block, lv.cell_x = t(h.cell_block), t(h.cell_x)
        lv.cell_y, lv.cell_z = t(h.cell_y), t(h.cell_z)
        lv.bouzidi_scratch = torch.empty(27 * h.n_boundary, dtype=torch.float32, device=dev)
        if reference_bouzidi:
            lv.f_post = torch.zeros(S * 27, dtype=torch.float32, device=dev)
    if ghost:
        lv.ghost = torch.empty(int(N.lib().ol_ghost_floats(N.i32(n))), dtype=torch.float32,
                               device=dev)
        if h.level_id > 1:
            lv.ghost2 = torch.empty_like(lv.ghost)
    if ddf:
        if ghost:
            lv.ghost_g = torch.empty_like(lv.ghost)
            if h.level_id > 1:
                lv.ghost_g2 = torch.empty_like(lv.ghost)
        w = torch.tensor(lattice_weights(), dtype=torch.float32, device=dev)
        lv.g = (w[:, None] * t_init).expand(27, S).reshape(-1).clone()
        lv.g_temp = lv.g.clone()
        lv.temperature = torch.full((S,), t_init, dtype=torch.float32, device=dev)
        lv.temperature_old = lv.temperature.clone()
    return lv


# Out-of-block pulls a block makes from its neighbour in direction d: 484
# from a face neighbour (22 x 22 cell-direction pairs), 22 from an edge, 1
# from a corner (3176 in all).
_PULLS_FROM_NEIGHBOUR = np.array(
    [{0: 0, 1: 484, 2: 22, 3: 1}[abs(d % 3 - 1) + abs((d // 3) % 3 - 1) + abs(d // 9 - 1)]
     for d in range(27)], dtype=np.int64)


def ghost_block_lists(h: HostLevel, dims) -> tuple[np.ndarray, np.ndarray]:
    """0-based ids (int32) of the blocks with an absent neighbour, and of
    those with an absent neighbour block not wholly inside the level's
    domain (dims = its size in cells): the ghost pass's visit lists.  Each
    list is ordered by the number of absent-neighbour pulls, largest first
    (ties by block id), so the pass's last CTAs are its shortest ones."""
    n = h.n_blocks
    missing = np.asarray(h.neighbor_table).reshape(27, n) <= 0     # [dir, block]
    d = np.arange(27)
    inside = np.ones((27, n), dtype=bool)
    for m, off, nc in ((h.map_x, d % 3 - 1, dims[0]), (h.map_y, (d // 3) % 3 - 1, dims[1]),
                       (h.map_z, d // 9 - 1, dims[2])):
        c = np.asarray(m, dtype=np.int64)[None, :] + off[:, None]
        inside &= (c >= 1) & (c * BS <= nc)

    def by_work(sel):
        ids = np.nonzero(sel.any(axis=0))[0]
        work = (sel[:, ids] * _PULLS_FROM_NEIGHBOUR[:, None]).sum(axis=0)
        return ids[np.argsort(-work, kind="stable")].astype(np.int32)

    return by_work(missing), by_work(missing & ~inside)


def lattice_weights() -> list:
    out = []
    for cz in (-1, 0, 1):
        for cy in (-1, 0, 1):
            for cx in (-1, 0, 1):
                d2 = cx * cx + cy * cy + cz * cz
                num, den = ((8, 27) if d2 == 0 else (2, 27) if d2 == 1 else (1, 54) if d2 == 2
                            else (1, 216))
                out.append(float(np.float32(num) / np.float32(den)))
    return out


@dc.dataclass
class StepSettings:
    """The scalars perform_timestep_v2! reads from globals (timestep.jl:39-49)."""
    op: int = 0
    c_wale: float = 0.2
    nu_sgs_bg: float = 0.0
    is_symmetric: int = 0
    wall_model: int = 0
    inlet_turbulence: float = 0.0
    use_temporal_interp: int = 1
    sponge_blend: int = 0
    omega_bulk: float = 1.0
    omega_3: float = 1.0
    omega_4: float = 1.0
    adaptive_omega4: int = 1
    lambda_param: float = 1.0 / 6.0
    limiter: int = 1
    compressible: int = 0
    q_min: float = 0.001
    ddf: int = 0
    t_inlet: float = 1.0
    t_wall: float = 1.0
    wall_bc_adiabatic: int = 1
    # fine-to-coarse restriction after each pair of child sub-steps (opt-in;
    # the reference couples the levels coarse to fine only)
    restriction: int = 0

    @staticmethod
    def from_config(cfg: CaseConfig, wall_model_active: bool) -> "StepSettings":
        return StepSettings(op=cfg.operator_code, c_wale=cfg.c_wale, nu_sgs_bg=cfg.nu_sgs_background,
                            is_symmetric=int(cfg.symmetric_analysis), wall_model=int(wall_model_active),
                            inlet_turbulence=cfg.inlet_turbulence_intensity,
                            use_temporal_interp=int(cfg.temporal_interpolation),
                            sponge_blend=int(cfg.sponge_blend_distributions),
                            omega_bulk=cfg.cumulant_omega_bulk, omega_3=cfg.cumulant_omega_3,
                            omega_4=cfg.cumulant_omega_4,
                            adaptive_omega4=int(cfg.cumulant_adaptive_omega4),
                            lambda_param=cfg.cumulant_lambda_param, limiter=cfg.limiter_code,
                            compressible=int(cfg.compressibility_correction),
                            q_min=cfg.q_min_threshold, ddf=int(cfg.ddf_enabled),
                            t_inlet=cfg.ddf_t_inlet, t_wall=cfg.ddf_t_wall,
                            wall_bc_adiabatic=int(cfg.ddf_wall_bc == "adiabatic"),
                            restriction=int(cfg.fine_to_coarse_restriction))


def step_params(s: StepSettings, lv: DeviceLevel, parent_tau: float, is_l1: bool, dims, u: float,
                t_sub: int, tw: float, store_post: bool) -> N.StepParams:
    sp = N.StepParams()
    sp.op = s.op
    sp.tau_molecular = lv.tau
    sp.tau_parent = parent_tau
    sp.c_wale = s.c_wale
    sp.nu_sgs_background = s.nu_sgs_bg
    sp.is_level_1 = int(is_l1)
    sp.is_symmetric = s.is_symmetric
    sp.nx_global, sp.ny_global, sp.nz_global = dims
    sp.u_inlet = u
    sp.wall_model_active = s.wall_model
    sp.time_step_seed = t_sub % 1000000
    sp.store_post_collision = int(store_post)
    sp.inlet_turbulence = s.inlet_turbulence
    sp.temporal_weight = tw
    sp.use_temporal_interp = s.use_temporal_interp
    sp.sponge_blend_distributions = s.sponge_blend
    sp.omega_bulk, sp.omega_3, sp.omega_4 = s.omega_bulk, s.omega_3, s.omega_4
    sp.adaptive_omega4 = s.adaptive_omega4
    sp.lambda_param = s.lambda_param
    sp.limiter_type = s.limiter
    sp.compressible_corr = s.compressible
    return sp


@dc.dataclass
class ParentRef:
    lv: DeviceLevel
    f_new: torch.Tensor
    vel_new: torch.Tensor
    g_new: torch.Tensor | None


def _ghost_views(view, lv: DeviceLevel, ghost, ghost2, mode: int) -> None:
    """Set a view's ghost, ghost_next, ghost_mode and visit list: mode 1 =
    first sub-step of a pair (also fills ghost2), 2 = second (reads ghost2),
    0 = unpaired."""
    if ghost is None or ghost2 is None:
        mode = N.OL_GHOST_UNPAIRED
    view.ghost_mode = mode
    view.ghost = _ptr(ghost2 if mode == N.OL_GHOST_PAIR_SECOND else ghost)
    view.ghost_next = _ptr(ghost2) if mode == N.OL_GHOST_PAIR_FIRST else None
    lst = lv.edge_list if mode == N.OL_GHOST_PAIR_SECOND else lv.ghost_list
    if ghost is not None and lst is not None:
        view.ghost_blocks, view.n_ghost_blocks = _ptr(lst), int(lst.numel()) - 1


def perform_timestep(s: StepSettings, lv: DeviceLevel, parent: ParentRef | None, f_out, f_in,
                     vel_out, vel_in, u: float, t_sub: int, tw: float, domain_dims,
                     g_out=None, g_in=None, ghost_mode: int = 0) -> None:
    """timestep.jl:1-159: flow kernel, Bouzidi, thermal kernel, thermal Bouzidi.
    ghost_mode pairs the two sub-steps of a refined level per parent step
    (N.OL_GHOST_PAIR_FIRST at weight 0, N.OL_GHOST_PAIR_SECOND at 1/2)."""
    n = lv.n_blocks
    if n == 0:
        return
    is_l1 = parent is None
    scale = 1 << (lv.host.level_id - 1)
    dims = (domain_dims[0] * scale, domain_dims[1] * scale, domain_dims[2] * scale)
    ref_post = lv.f_post is not None
    if lv.ghost is not None and lv.ghost_list is None:   # static: computed on first use
        # one trailing entry keeps an empty list's pointer non-null (a null
        # list means "every block"); the view passes the true length
        gl, el = ghost_block_lists(lv.host, dims)
        lv.ghost_list = torch.from_numpy(np.append(gl, -1).astype(np.int32)).to(lv.f.device)
        lv.edge_list = torch.from_numpy(np.append(el, -1).astype(np.int32)).to(lv.f.device)
    sp = step_params(s, lv, parent.lv.tau if parent else 0.5, is_l1, dims, u, t_sub, tw,
                     lv.has_bouzidi and ref_post)
    view = N.LevelView(f_out=_ptr(f_out), f_in=_ptr(f_in), f_post=_ptr(lv.f_post),
                       rho=_ptr(lv.rho), vel_out=_ptr(vel_out), vel_in=_ptr(vel_in),
                       obstacle=_ptr(lv.obstacle), sponge=_ptr(lv.sponge),
                       wall_dist=_ptr(lv.wall_dist), neighbor_table=_ptr(lv.neighbor_table),
                       map_x=_ptr(lv.map_x), map_y=_ptr(lv.map_y), map_z=_ptr(lv.map_z),
                       n_blocks=n)
    _ghost_views(view, lv, lv.ghost, lv.ghost2, ghost_mode)
    pv = N.ParentView()
    if parent is not None:
        p = parent.lv
        d = p.host.grid_dim
        pv = N.ParentView(f=_ptr(parent.f_new), rho=_ptr(p.rho), vel=_ptr(parent.vel_new),
                          f_old=_ptr(p.f_old), rho_old=_ptr(p.rho_old), vel_old=_ptr(p.vel_old),
                          block_ptr=_ptr(p.block_ptr), dim_x=d[0], dim_y=d[1], dim_z=d[2],
                          n_blocks=p.n_blocks)
    st = _stream()
    N.call("ol_stream_collide", C.byref(view), C.byref(pv), C.byref(sp), st)
    if lv.has_bouzidi:
        h = lv.host
        if ref_post:
            N.call("ol_bouzidi", _ptr(f_out), _ptr(lv.f_post), _ptr(lv.q_map), _ptr(lv.cell_block),
                   _ptr(lv.cell_x), _ptr(lv.cell_y), _ptr(lv.cell_z), N.i32(h.n_boundary),
                   _ptr(lv.neighbor_table), N.i32(n), N.f32(s.q_min), st)
        else:
            if lv.bz_links is None:
                build_bouzidi_links(lv, s.q_min)
            N.call("ol_bouzidi_apply_links", _ptr(f_out), _ptr(lv.bz_links),
                   N.i32(lv.bz_n_links), N.i32(n), _ptr(lv.bouzidi_scratch), st)
    if s.ddf and g_out is not None:
        tp = N.ThermalParams(tau_g=lv.host.tau_g, tau_g_parent=parent.lv.host.tau_g if parent else 0.5,
                             is_level_1=int(is_l1), is_symmetric=s.is_symmetric,
                             nx_global=dims[0], ny_global=dims[1], nz_global=dims[2], u_inlet=u,
                             T_inlet=s.t_inlet, T_wall=s.t_wall,
                             wall_bc_adiabatic=s.wall_bc_adiabatic, store_post_collision=0,
                             temporal_weight=tw, use_temporal_interp=s.use_temporal_interp,
                             sponge_blend_distributions=s.sponge_blend)
        tv = N.ThermalView(g_out=_ptr(g_out), g_in=_ptr(g_in), g_post=None,
                           temperature=_ptr(lv.temperature), vel=_ptr(vel_out),
                           obstacle=_ptr(lv.obstacle), sponge=_ptr(lv.sponge),
                           neighbor_table=_ptr(lv.neighbor_table), map_x=_ptr(lv.map_x),
                           map_y=_ptr(lv.map_y), map_z=_ptr(lv.map_z), n_blocks=n)
        _ghost_views(tv, lv, lv.ghost_g, lv.ghost_g2, ghost_mode)
        if parent is not None:
            p = parent.lv
            d = p.host.grid_dim
            tv.pg, tv.pT, tv.pvel = _ptr(parent.g_new), _ptr(p.temperature), _ptr(parent.vel_new)
            tv.pg_old, tv.pT_old, tv.pvel_old = _ptr(p.g_old), _ptr(p.temperature_old), _ptr(p.vel_old)
            tv.p_block_ptr = _ptr(p.block_ptr)
            tv.p_dim_x, tv.p_dim_y, tv.p_dim_z = d
            tv.p_n_blocks = p.n_blocks
        N.call("ol_thermal", C.byref(tv), C.byref(tp), st)
        if lv.has_bouzidi:
            if lv.bz_links is None:
                build_bouzidi_links(lv, s.q_min)
            N.call("ol_bouzidi_apply_links", _ptr(g_out), _ptr(lv.bz_links),
                   N.i32(lv.bz_n_links), N.i32(n), _ptr(lv.bouzidi_scratch), st)


def recursive_step(levels: list, s: StepSettings, lvl: int, t_sub: int, parent: ParentRef | None,
                   tw: float, u: float, domain_dims, ghost_mode: int = 0) -> None:
    """solver_control.jl:6-197 (recursive_step! and recursive_step_temporal!).
    A child's two sub-steps per parent step share one ghost pass (ghost_mode)."""
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
    if has_children and s.use_temporal_interp:
        # copy_to_old!: f_old / vel_old alias the untouched pull sources
        lv.f_old, lv.vel_old = f_in, vel_in
        lv.rho_old.copy_(lv.rho)
        if s.ddf and lv.g is not None:
            lv.g_old = g_in
            lv.temperature_old.copy_(lv.temperature)
    perform_timestep(s, lv, parent, f_out, f_in, vel_out, vel_in, u, t_sub,
                     0.0 if parent is None else tw, domain_dims,
                     g_out=g_out if s.ddf else None, g_in=g_in if s.ddf else None,
                     ghost_mode=ghost_mode)
    if has_children:
        me = ParentRef(lv, f_out, vel_out, g_out if s.ddf else None)
        recursive_step(levels, s, lvl + 1, 2 * t_sub, me, 0.0, u, domain_dims,
                       N.OL_GHOST_PAIR_FIRST)
        recursive_step(levels, s, lvl + 1, 2 * t_sub + 1, me, 0.5, u, domain_dims,
                       N.OL_GHOST_PAIR_SECOND)
        if s.restriction:
            # the child's second sub-step (odd t_sub) wrote f and vel
            restrict_level(levels[lvl + 1], me, s)


def build_bouzidi_links(lv: DeviceLevel, q_min: float) -> None:
    """The level's Bouzidi link list (ol_bouzidi_build_links): static, built
    on first use; the correction then visits only those links."""
    h = lv.host
    links = torch.empty((27 * h.n_boundary + 1) * 4, dtype=torch.int32, device=lv.f.device)
    count = torch.zeros(1, dtype=torch.int32, device=lv.f.device)
    N.call("ol_bouzidi_build_links", _ptr(lv.q_map), _ptr(lv.cell_block), _ptr(lv.cell_x),
           _ptr(lv.cell_y), _ptr(lv.cell_z), N.i32(h.n_boundary), _ptr(lv.neighbor_table),
           N.i32(lv.n_blocks), N.f32(q_min), _ptr(links), _ptr(count), _stream())
    lv.bz_n_links = int(count.item())
    lv.bz_links = links


def restrict_level(child: DeviceLevel, parent: ParentRef, s: StepSettings) -> None:
    """Fine-to-coarse restriction (ol_restrict) of the child's newest state
    into the parent's newest state; an opt-in extension of the reference."""
    p = parent.lv
    d = p.host.grid_dim
    v = N.RestrictView(f_fine=_ptr(child.f), obstacle_fine=_ptr(child.obstacle),
                       map_x=_ptr(child.map_x), map_y=_ptr(child.map_y), map_z=_ptr(child.map_z),
                       n_fine=child.n_blocks, f_coarse=_ptr(parent.f_new), rho_coarse=_ptr(p.rho),
                       vel_coarse=_ptr(parent.vel_new), obstacle_coarse=_ptr(p.obstacle),
                       block_ptr=_ptr(p.block_ptr), dim_x=d[0], dim_y=d[1], dim_z=d[2],
                       n_coarse=p.n_blocks, tau_fine=child.tau, tau_coarse=p.tau,
                       compressible=s.compressible)
    N.call("ol_restrict", C.byref(v), _stream())


def execute_timestep_batch(levels, s: StepSettings, t_start: int, batch: int, u: float,
                           domain_dims) -> None:
    """solver_control.jl:199-218."""
    for off in range(batch):
        recursive_step(levels, s, 0, t_start + off, None, 0.0, u, domain_dims)


@dc.dataclass
class Batch:
    """One pass of main.jl's time loop (main.jl:212-313): steps t..end at one
    inlet velocity u; diag_step / out_step are the diagnostics and output
    steps that fall inside the batch (None when none does)."""
    t: int
    end: int
    actual: int
    u: float
    diag_step: int | None
    out_step: int | None


def main_loop_batches(first: int, last: int, async_depth: int, diag_freq: int,
                      output_freq: int, ramp_steps: int, u_target: float):
    """main.jl:212-313 schedule: batches of async_depth steps, the inlet
    velocity of a batch evaluated at its end step; a diagnostics step is
    the multiple of diag_freq that the batch crosses (also checked on the
    run's last batch); an output step likewise for output_freq."""
    batch = max(1, async_depth)
    of = max(1, output_freq)
    t = first
    while t <= last:
        end = min(t + batch - 1, last)
        actual = end - t + 1
        diag = out = None
        if end % diag_freq < actual or end == last:
            d = (end // diag_freq) * diag_freq
            if t <= d <= end:
                diag = d
        if end % of < actual:
            o = (end // of) * of
            if t <= o <= end:
                out = o
        yield Batch(t, end, actual, ramp_velocity(u_target, end, ramp_steps), diag, out)
        t = end + 1


def ramp_velocity(u_target: float, batch_end: int, ramp_steps: int) -> float:
    """main.jl:217-218: cosine ramp evaluated once per batch at its end step,
    in Float32: prog = 0.5f0 (1 - cos(Float32(pi) batch_end / ramp)).  The
    Float32 argument is formed as Julia forms it (Float32 product, then
    Float32 quotient); cos is taken in double and rounded once to Float32,
    which is how Julia's cos(::Float32) works too (Float64 kernel, one
    rounding), so the two agree except where cos lies within that kernel's
    error of a Float32 rounding midpoint (then by one ulp of u)."""
    if ramp_steps > 0 and batch_end <= ramp_steps:
        prog = np.float32(0.5) * (np.float32(1.0) - np.float32(math.cos(np.float32(math.pi) * batch_end / ramp_steps)))
    else:
        prog = np.float32(1.0)
    return float(np.float32(u_target) * np.float32(prog))


def cells_total(levels) -> int:
    return sum(lv.n_blocks * 512 for lv in levels)


def cell_updates_per_coarse_step(levels) -> int:
    """True cell updates: level l advances 2^(l-1) times per coarse step."""
    return sum(lv.n_blocks * 512 * (1 << i) for i, lv in enumerate(levels))


# --------------------------------------------------------------------- forces

@dc.dataclass
class DeviceMesh:
    """upload_mesh_to_gpu (geometry.jl:50-69): FP32 centres, normals, areas."""
    arrays: torch.Tensor   # [7, n]: cx cy cz nx ny nz area
    n: int

    def view(self) -> N.SurfaceMesh:
        a = self.arrays
        return N.SurfaceMesh(cx=_ptr(a[0]), cy=_ptr(a[1]), cz=_ptr(a[2]), nx=_ptr(a[3]),
                             ny=_ptr(a[4]), nz=_ptr(a[5]), area=_ptr(a[6]), n_triangles=self.n)


def upload_mesh(mesh, device) -> DeviceMesh:
    a = np.stack([mesh.centers[:, 0], mesh.centers[:, 1], mesh.centers[:, 2], mesh.normals[:, 0],
                  mesh.normals[:, 1], mesh.normals[:, 2], mesh.areas]).astype(np.float32)
    return DeviceMesh(torch.from_numpy(np.ascontiguousarray(a)).to(device), mesh.n)


def force_params_for(lv: DeviceLevel, p: DomainParams, cfg: CaseConfig,
                     search_radius: int = 5) -> N.ForceParams:
    vs = p.velocity_scale
    ps = float(np.float32(p.rho_physical * vs * vs))
    h = lv.host
    mc, off = p.moment_center, p.mesh_offset
    return N.ForceParams(dx=float(np.float32(h.dx)), dim_x=h.grid_dim[0], dim_y=h.grid_dim[1],
                         dim_z=h.grid_dim[2], offset_x=off[0], offset_y=off[1], offset_z=off[2],
                         pressure_scale=ps, stress_scale=ps, tau_molecular=h.tau,
                         search_radius=search_radius, c_wale=cfg.c_wale,
                         nu_sgs_bg=cfg.nu_sgs_background, ref_x=mc[0], ref_y=mc[1], ref_z=mc[2])


def compute_aerodynamics(lv: DeviceLevel, dmesh: DeviceMesh, p: DomainParams, cfg: CaseConfig,
                         vel: torch.Tensor | None = None, maps: bool = False,
                         search_radius: int = 5):
    """compute_aerodynamics! (surface.jl:913-920) on a level: returns the raw
    nine sums (and the per-triangle p / shear maps when maps=True).  `vel`
    defaults to the level's `vel` buffer, as the reference reads `level.vel`."""
    fp = force_params_for(lv, p, cfg, search_radius)
    n = dmesh.n
    dev = lv.rho.device
    partials = torch.empty(int(N.lib().ol_surface_forces_scratch_doubles(n)), dtype=torch.float64,
                           device=dev)
    m = torch.empty((4, n), dtype=torch.float32, device=dev) if maps else None
    out = (C.c_double * 9)()
    N.call("ol_surface_forces", C.byref(dmesh.view()), _ptr(lv.rho), _ptr(vel if vel is not None else lv.vel),
           _ptr(lv.obstacle), _ptr(lv.block_ptr), N.i32(lv.n_blocks), C.byref(fp),
           _ptr(m[0]) if maps else None, _ptr(m[1]) if maps else None,
           _ptr(m[2]) if maps else None, _ptr(m[3]) if maps else None, _ptr(partials), out,
           _stream())
    raw = np.array(out[:], dtype=np.float64)
    return (raw, m) if maps else raw


def compute_net_aerodynamics(lv: DeviceLevel, dmesh: DeviceMesh, p: DomainParams,
                             cfg: CaseConfig, search_radius: int = 5, closed_body: bool = True,
                             maps: bool = False):
    """compute_net_aerodynamics! (surface.jl:980-1034): per-triangle net force
    (net_Fx, net_Fy, net_Fz) as float32 numpy arrays.  With maps=True also the
    [8, n] device tensor of plus maps (p, tau x/y/z) and minus maps."""
    fp = force_params_for(lv, p, cfg, search_radius)
    n = dmesh.n
    dev = lv.rho.device
    net = torch.empty((3, n), dtype=torch.float32, device=dev)
    m = torch.empty((8, n), dtype=torch.float32, device=dev) if maps else None
    mp = [_ptr(m[j]) for j in range(8)] if maps else [None] * 8
    out = N.NetForceMaps(*mp, _ptr(net[0]), _ptr(net[1]), _ptr(net[2]))
    N.call("ol_surface_net_forces", C.byref(dmesh.view()), _ptr(lv.rho), _ptr(lv.vel),
           _ptr(lv.obstacle), _ptr(lv.block_ptr), N.i32(lv.n_blocks), C.byref(fp),
           N.i32(1 if closed_body else 0), C.byref(out), _stream())
    h = net.cpu().numpy()
    res = (h[0], h[1], h[2])
    return (res, m) if maps else res


def flow_stats(lv: DeviceLevel) -> dict:
    """compute_flow_stats (diagnostics.jl:43-93) in FP64."""
    partials = torch.empty(int(N.lib().ol_flow_stats_scratch_doubles(lv.n_blocks)),
                           dtype=torch.float64, device=lv.rho.device)
    out = (C.c_double * 7)()
    N.call("ol_flow_stats", _ptr(lv.rho), _ptr(lv.vel), _ptr(lv.obstacle), N.i32(lv.n_blocks),
           _ptr(partials), out, _stream())
    n = out[0]
    return {"n_fluid": int(n), "rho_mean": out[1] / n if n else 1.0, "rho_min": out[2],
            "rho_max": out[3], "v_max": out[4], "kinetic_energy": out[5], "mass": out[6]}


class Simulation:
    """main.jl solve_main() time loop over the device levels: batched cosine
    inlet ramp, diagnostics every diag_freq steps, surface forces on the
    finest level, time averaging after the ramp (ForceAccumulator), and,
    with an output folder, the files the reference writes there.

    `unrotated_mesh` is the body in its STL frame (before the angle-of-attack
    rotation); the surface-pressure and net-force files use it as the
    reference does (main.jl:281-304).  Without it they use `mesh`."""

    def __init__(self, cfg: CaseConfig, mesh, p: DomainParams, hosts, device=None,
                 unrotated_mesh=None):
        from .native import coefficients
        self._coeff = coefficients
        self.cfg, self.mesh, self.p = cfg, mesh, p
        self.unrotated_mesh = unrotated_mesh if unrotated_mesh is not None else mesh
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.levels = [upload_level(h, self.device, ddf=cfg.ddf_enabled, t_init=cfg.ddf_t_initial)
                       for h in hosts]
        self.settings = StepSettings.from_config(cfg, cfg.wall_model_enabled)
        self.dmesh = upload_mesh(mesh, self.device)
        self.dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
        self.t = 0
        self.history: list[dict] = []
        self.acc = np.zeros(9)
        self.n_avg = 0
        self._records = None
        self._out = None

    def forces(self, maps: bool = False):
        got = compute_aerodynamics(self.levels[-1], self.dmesh, self.p, self.cfg, maps=maps)
        raw, m = got if maps else (got, None)
        fr = self._coeff(raw, self.p.rho_physical, self.p.u_physical, self.p.reference_area,
                         self.p.reference_chord, self.cfg.symmetric_analysis)
        return (fr, raw, m) if maps else (fr, raw)

    def _sample(self, step: int, maps: bool):
        """compute_aerodynamics! + accumulate_forces! after the ramp."""
        fr, raw, m = self.forces(maps=True) if maps else (*self.forces(), None)
        if step > self.cfg.ramp_steps:
            self.acc += raw
            self.n_avg += 1
        return fr, m

    def run(self, steps: int, diag_freq: int | None = None,
            output_dir: str | None = None) -> list[dict]:
        """Advance `steps` steps in main.jl's batches (main_loop_batches).
        At a diagnostics step: flow statistics of level 1, forces on the
        finest level (accumulated after the ramp).  At an output step that is
        not a diagnostics multiple the forces are sampled and accumulated as
        well (main.jl:267-275).  With output_dir: convergence.csv and
        forces.csv rows per diagnostics step; per output step the merged
        flow field flow_%06d.vtu (gathered on the device at the batch end,
        copied back while the next batches run, written at the next output
        or at the end), surface_%06d.lbmp and, with net-force export,
        net_forces_%06d.csv; and a final output at the run's last step when
        that is not an output step (main.jl:316-360)."""
        import time as _time
        cfg = self.cfg
        diag = diag_freq or cfg.diag_freq
        last = self.t + steps
        pending = None
        fwd = cfg.forces_enabled
        if output_dir is not None:
            from .output import MergedOutput
            if self._out is None:
                self._out = MergedOutput(self.levels)
            if self._records is None:
                from .records import RunRecords
                self._records = RunRecords(output_dir, fwd)
        cells = cells_total(self.levels)
        last_diag = _time.perf_counter()
        maps = None
        for b in main_loop_batches(self.t + 1, last, cfg.async_depth, diag, cfg.output_freq,
                                   cfg.ramp_steps, cfg.u_target):
            execute_timestep_batch(self.levels, self.settings, b.t, b.actual, b.u, self.dims)
            want_maps = output_dir is not None and b.out_step is not None
            if b.diag_step is not None:
                d = b.diag_step
                rec = {"step": d, "u": b.u, **flow_stats(self.levels[0])}
                fr = None
                if fwd:
                    fr, maps = self._sample(d, want_maps)
                    rec.update(Cd=fr.Cd, Cl=fr.Cl, Cs=fr.Cs, Cmy=fr.Cmy)
                self.history.append(rec)
                if self._records is not None and output_dir is not None:
                    now = _time.perf_counter()
                    mlups = cells * diag / ((now - last_diag) * 1e6)
                    last_diag = now
                    tp = float(d) * self.p.time_scale
                    lx = self.p.domain_size[0]
                    travel = 100.0 * (tp * self.p.u_physical) / lx if lx > 0 else 0.0
                    self._records.append(d, tp, travel, b.u, rec["rho_min"], mlups, fr)
            if b.out_step is not None:
                o = b.out_step
                if fwd and o != (o // diag) * diag:
                    _, maps = self._sample(o, want_maps)
                if output_dir is not None:
                    if pending is not None:
                        self._write(output_dir, pending)
                    pending = self._out.pack(o)
                    if fwd:
                        self._surface_files(output_dir, o, maps)
        self.t = last
        if output_dir is not None:
            of = max(1, cfg.output_freq)
            if (last // of) * of != last or last < of:
                if pending is not None:
                    self._write(output_dir, pending)
                pending = self._out.pack(last)
                if fwd:
                    _, _, maps = self.forces(maps=True)
                    self._surface_files(output_dir, last, maps)
        if pending is not None:
            self._write(output_dir, pending)
        return self.history

    def _surface_files(self, output_dir: str, step: int, maps) -> None:
        """surface_%06d.lbmp from the pressure / shear maps of the last force
        evaluation, in the STL frame without domain offset (main.jl:284-287);
        net_forces_%06d.csv when net-force export is on (main.jl:290-301)."""
        import os
        from .records import write_net_forces_csv, write_surface_pressure_bin
        m = maps.cpu().numpy()
        um = self.unrotated_mesh
        write_surface_pressure_bin(os.path.join(output_dir, "surface_%06d.lbmp" % step),
                                   um.triangles, um.normals, m[0], m[1:4],
                                   self.p.rho_physical, self.p.u_physical)
        if self.cfg.net_force_export:
            net = compute_net_aerodynamics(self.levels[-1], self.dmesh, self.p, self.cfg)
            write_net_forces_csv(os.path.join(output_dir, "net_forces_%06d.csv" % step),
                                 np.stack(net), self.mesh.centers, self.p.mesh_offset,
                                 unrotated_centers=self.unrotated_mesh.centers,
                                 alpha_deg=self.cfg.alpha_deg, beta_deg=self.cfg.beta_deg)

    @staticmethod
    def _write(output_dir: str, snap) -> None:
        import os
        from .output import write_vtu
        os.makedirs(output_dir, exist_ok=True)
        write_vtu(os.path.join(output_dir, "flow_%06d.vtu" % snap.t_step), snap.wait())

    def averaged(self):
        """print_averaged_summary (surface.jl:58-139) coefficients."""
        if self.n_avg == 0:
            return None
        return self._coeff(self.acc / self.n_avg, self.p.rho_physical, self.p.u_physical,
                           self.p.reference_area, self.p.reference_chord,
                           self.cfg.symmetric_analysis)
