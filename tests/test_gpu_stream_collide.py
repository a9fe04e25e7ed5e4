"""GPU parity of the fused stream-collide, Bouzidi and thermal kernels against
the CPU oracle, called through the C ABI.

Tolerances: one FP32 step differs from the oracle only by contraction (FMA)
and evaluation order, a few ulp per operation; the tests allow 2e-6
absolute on populations of O(0.3) and 1e-5 relative in L2.  Multi-step runs
allow 1e-4 relative L2 after 100 steps (growth of those rounding
differences through the dynamics).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import (interior_refined_case, max_abs, perturbed_state, rel_err,
                     small_sphere_case, weights32)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import _native as N  # noqa: E402
from openludwig_b200 import solver as S  # noqa: E402
from oracle import driver as odrv  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def case1():
    orc.build()
    return small_sphere_case(resolution=8)


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


VARIANTS = [
    dict(name="cumulant_factored", op=0, limiter=1),
    dict(name="cumulant_positivity", op=0, limiter=2),
    dict(name="cumulant_none_fixed_w4", op=0, limiter=0, adaptive_omega4=0, omega_4=1.3),
    dict(name="cumulant_wale", op=0, limiter=1, c_wale=0.5),
    dict(name="cumulant_wale_bg_wallmodel", op=0, limiter=1, c_wale=0.5, nu_sgs_bg=1e-4,
         wall_model=1),
    dict(name="cumulant_sponge_blend_turb", op=0, limiter=1, sponge_blend=1, inlet_turbulence=0.05),
    dict(name="cumulant_compressible", op=0, limiter=1, compressible=1),
    dict(name="bgk", op=1, c_wale=0.0),
    dict(name="bgk_wale_wallmodel", op=1, c_wale=0.5, wall_model=1),
    dict(name="bgk_compressible", op=1, c_wale=0.2, compressible=1, sponge_blend=1),
]


@pytest.mark.parametrize("var", VARIANTS, ids=[v["name"] for v in VARIANTS])
def test_single_step_matches_oracle(case1, var):
    c, mesh, p, hosts = case1
    h = hosts[0]
    n = h.n_blocks
    f_in, vel_in = perturbed_state(n, seed=7)
    wd = h.wall_dist.copy()
    if var.get("wall_model"):
        # distances in lattice units so that near-wall cells are active
        wd = np.where(wd < 100.0, wd / np.float32(h.dx_exact), wd).astype(np.float32)
    st = S.StepSettings(**{k: v for k, v in var.items() if k != "name"})
    sp = S.step_params(st, type("L", (), {"tau": 0.52})(), 0.5, True,
                       (p.nx_coarse, p.ny_coarse, p.nz_coarse), 0.05, 37, 0.0, False)
    # GPU
    d_fin, d_fout = _t(f_in), torch.zeros(27 * 512 * n, dtype=torch.float32, device=DEV)
    d_vin, d_vout = _t(vel_in), torch.zeros(3 * 512 * n, dtype=torch.float32, device=DEV)
    d_rho = torch.zeros(512 * n, dtype=torch.float32, device=DEV)
    arrs = {k: _t(getattr(h, k)) for k in ("obstacle", "sponge", "neighbor_table", "map_x",
                                           "map_y", "map_z")}
    d_wd = _t(wd)
    view = N.LevelView(f_out=S._ptr(d_fout), f_in=S._ptr(d_fin), f_post=None, rho=S._ptr(d_rho),
                       vel_out=S._ptr(d_vout), vel_in=S._ptr(d_vin),
                       obstacle=S._ptr(arrs["obstacle"]), sponge=S._ptr(arrs["sponge"]),
                       wall_dist=S._ptr(d_wd), neighbor_table=S._ptr(arrs["neighbor_table"]),
                       map_x=S._ptr(arrs["map_x"]), map_y=S._ptr(arrs["map_y"]),
                       map_z=S._ptr(arrs["map_z"]), n_blocks=n)
    N.call("ol_stream_collide", C.byref(view), C.byref(N.ParentView()), C.byref(sp), S._stream())
    # the same step with the boundary values of absent neighbours from their own pass
    ghost = torch.empty(int(N.lib().ol_ghost_floats(N.i32(n))), dtype=torch.float32, device=DEV)
    d_fout2, d_vout2 = torch.zeros_like(d_fout), torch.zeros_like(d_vout)
    view2 = N.LevelView(**{name: getattr(view, name) for name, _ in N.LevelView._fields_})
    view2.f_out, view2.vel_out, view2.ghost = S._ptr(d_fout2), S._ptr(d_vout2), S._ptr(ghost)
    N.call("ol_stream_collide", C.byref(view2), C.byref(N.ParentView()), C.byref(sp), S._stream())
    torch.cuda.synchronize()
    assert torch.equal(d_fout, d_fout2) and torch.equal(d_vout, d_vout2)
    # oracle
    o_fout = np.zeros(27 * 512 * n, np.float32)
    o_rho = np.zeros(512 * n, np.float32)
    o_vout = np.zeros(3 * 512 * n, np.float32)
    params = {name: getattr(sp, name) for name, _ in N.STEP_FIELDS}
    orc.stream_collide(dict(f_out=o_fout, f_in=f_in, rho=o_rho, vel_out=o_vout, vel_in=vel_in,
                            obstacle=h.obstacle, sponge=h.sponge, wall_dist=wd,
                            neighbor_table=h.neighbor_table, map_x=h.map_x, map_y=h.map_y,
                            map_z=h.map_z, n_blocks=n), None, params)
    g_f = d_fout.cpu().numpy()
    assert max_abs(g_f, o_fout) < 2e-6, var["name"]
    assert rel_err(g_f, o_fout) < 1e-5
    assert max_abs(d_rho.cpu().numpy(), o_rho) < 2e-6
    assert max_abs(d_vout.cpu().numpy(), o_vout) < 2e-6


def _run_gpu(hosts, p, st, steps, u, ddf=False, ghost=None):
    levels = [S.upload_level(h, DEV, ddf=ddf, ghost=ghost) for h in hosts]
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    for t in range(1, steps + 1):
        S.recursive_step(levels, st, 0, t, None, 0.0, u, dims)
    torch.cuda.synchronize()
    return levels


def _run_oracle(hosts, p, st, steps, u, ddf=False):
    levels = odrv.init_levels(hosts, ddf=ddf)
    s = odrv.settings_dict(st)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    for t in range(1, steps + 1):
        odrv.recursive_step(levels, s, 0, t, None, 0.0, u, dims, np.float32)
    return levels


def test_bouzidi_sparse_matches_reference_form(case1):
    """Two-phase in-place Bouzidi == reference form reading a separate f_post."""
    c, mesh, p, hosts = case1
    h = hosts[0]
    n = h.n_blocks
    f_post, _ = perturbed_state(n, seed=3)
    d_out = _t(f_post)
    d_post = _t(f_post)
    arrs = {k: _t(getattr(h, k)) for k in ("cell_block", "cell_x", "cell_y", "cell_z",
                                           "neighbor_table")}
    q = _t(h.q_map.view(np.int16))
    scratch = torch.empty(27 * h.n_boundary, dtype=torch.float32, device=DEV)
    N.call("ol_bouzidi_sparse", S._ptr(d_out), S._ptr(q), S._ptr(arrs["cell_block"]),
           S._ptr(arrs["cell_x"]), S._ptr(arrs["cell_y"]), S._ptr(arrs["cell_z"]),
           N.i32(h.n_boundary), S._ptr(arrs["neighbor_table"]), N.i32(n), N.f32(0.001),
           S._ptr(scratch), S._stream())
    d_ref = _t(f_post)
    N.call("ol_bouzidi", S._ptr(d_ref), S._ptr(d_post), S._ptr(q), S._ptr(arrs["cell_block"]),
           S._ptr(arrs["cell_x"]), S._ptr(arrs["cell_y"]), S._ptr(arrs["cell_z"]),
           N.i32(h.n_boundary), S._ptr(arrs["neighbor_table"]), N.i32(n), N.f32(0.001), S._stream())
    torch.cuda.synchronize()
    o = f_post.copy()
    orc.bouzidi(o, f_post, h.q_map, h.cell_block, h.cell_x, h.cell_y, h.cell_z,
                h.neighbor_table, n, 0.001)
    assert np.array_equal(d_out.cpu().numpy(), d_ref.cpu().numpy())
    assert max_abs(d_out.cpu().numpy(), o) < 1e-6
    assert not np.array_equal(o, f_post)  # the correction did something


def test_100_steps_single_level(case1):
    c, mesh, p, hosts = case1
    st = S.StepSettings.from_config(c, False)
    g = _run_gpu(hosts, p, st, 100, 0.05)
    o = _run_oracle(hosts, p, st, 100, 0.05)
    # after an even number of steps the newest state is in f_temp (t=100 even)
    assert rel_err(g[0].f_temp.cpu().numpy(), o[0].f_temp) < 1e-4
    assert rel_err(g[0].rho.cpu().numpy(), o[0].rho) < 1e-5
    assert rel_err(g[0].vel_temp.cpu().numpy(), o[0].vel_temp) < 1e-3


def test_two_level_recursion():
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5))
    assert len(hosts) == 2 and hosts[1].n_blocks > 0
    st = S.StepSettings.from_config(c, False)
    g = _run_gpu(hosts, p, st, 20, 0.05)
    o = _run_oracle(hosts, p, st, 20, 0.05)
    for lg, lo in zip(g, o):
        assert rel_err(lg.f_temp.cpu().numpy(), lo.f_temp) < 1e-4
        assert rel_err(lg.rho.cpu().numpy(), lo.rho) < 1e-5


@pytest.mark.parametrize("ddf", [False, True], ids=["flow", "flow_thermal"])
def test_ghost_pass_equals_inline_fill(ddf):
    """Interface and domain-boundary values from the separate pass (ghost
    scratch) and from the in-staging fill give the same bits, for the flow
    and for the thermal populations."""
    kw = dict(compressibility_correction=True, ddf_enabled=True,
              u_target=np.float32(0.1)) if ddf else {}
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5), **kw)
    st = S.StepSettings.from_config(c, False)
    u = 0.1 if ddf else 0.05
    a = _run_gpu(hosts, p, st, 6, u, ddf=ddf, ghost=True)
    b = _run_gpu(hosts, p, st, 6, u, ddf=ddf, ghost=False)
    for la, lb in zip(a, b):
        assert la.ghost is not None and lb.ghost is None
        assert torch.equal(la.f_temp, lb.f_temp) and torch.equal(la.f, lb.f)
        assert torch.equal(la.vel_temp, lb.vel_temp) and torch.equal(la.rho, lb.rho)
        if ddf:
            assert la.ghost_g is not None
            assert torch.equal(la.g_temp, lb.g_temp) and torch.equal(la.g, lb.g)
            assert torch.equal(la.temperature, lb.temperature)


@pytest.mark.parametrize("which", ["interior", "edge_ddf"])
def test_ghost_pairing_is_bitwise_neutral(which):
    """The pair's first sub-step filling the second one's coarse-to-fine
    values (OL_GHOST_PAIR_FIRST / _SECOND) gives the bits of evaluating every
    value in every call: on a refined level inside the domain (the second
    pass has nothing left to do) and, with the thermal DDF, on one whose
    blocks also carry domain-boundary values."""
    if which == "interior":
        c, mesh, p, hosts = interior_refined_case()
        st = S.StepSettings.from_config(c, c.wall_model_enabled)
        ddf, u, steps = False, 0.05, 4
    else:
        c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5),
                                              compressibility_correction=True,
                                              ddf_enabled=True, u_target=np.float32(0.1))
        st = S.StepSettings.from_config(c, False)
        ddf, u, steps = True, 0.1, 6
    paired = _run_gpu(hosts, p, st, steps, u, ddf=ddf, ghost=True)
    levels = [S.upload_level(h, DEV, ddf=ddf, ghost=True) for h in hosts]
    for lv in levels:
        lv.ghost2 = lv.ghost_g2 = None          # unpaired: every value in every call
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    for t in range(1, steps + 1):
        S.recursive_step(levels, st, 0, t, None, 0.0, u, dims)
    torch.cuda.synchronize()
    assert paired[1].ghost2 is not None
    for la, lb in zip(paired, levels):
        assert torch.equal(la.f_temp, lb.f_temp) and torch.equal(la.f, lb.f)
        assert torch.equal(la.vel_temp, lb.vel_temp) and torch.equal(la.rho, lb.rho)
        if ddf:
            assert torch.equal(la.g_temp, lb.g_temp) and torch.equal(la.g, lb.g)
            assert torch.equal(la.temperature, lb.temperature)


def test_restriction_matches_oracle():
    """Opt-in fine-to-coarse restriction: one ol_restrict call against the
    oracle on a perturbed state, then 20 coarse steps of a two-level case
    with restriction on against the oracle recursion."""
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5))
    hc, hf = hosts
    rng = np.random.default_rng(4)
    w = weights32()
    f_f = (np.repeat(w, 512 * hf.n_blocks) * rng.uniform(0.95, 1.05, 27 * 512 * hf.n_blocks)
           ).astype(np.float32)
    f_c = (np.repeat(w, 512 * hc.n_blocks) * rng.uniform(0.95, 1.05, 27 * 512 * hc.n_blocks)
           ).astype(np.float32)
    rho_c = np.ones(512 * hc.n_blocks, np.float32)
    vel_c = np.zeros(3 * 512 * hc.n_blocks, np.float32)
    d = {k: _t(v) for k, v in dict(f_f=f_f, f_c=f_c, rho_c=rho_c, vel_c=vel_c,
                                     of=hf.obstacle, oc=hc.obstacle, mx=hf.map_x, my=hf.map_y,
                                     mz=hf.map_z, bp=hc.block_ptr).items()}
    v = N.RestrictView(f_fine=S._ptr(d["f_f"]), obstacle_fine=S._ptr(d["of"]),
                       map_x=S._ptr(d["mx"]), map_y=S._ptr(d["my"]), map_z=S._ptr(d["mz"]),
                       n_fine=hf.n_blocks, f_coarse=S._ptr(d["f_c"]), rho_coarse=S._ptr(d["rho_c"]),
                       vel_coarse=S._ptr(d["vel_c"]), obstacle_coarse=S._ptr(d["oc"]),
                       block_ptr=S._ptr(d["bp"]), dim_x=hc.grid_dim[0], dim_y=hc.grid_dim[1],
                       dim_z=hc.grid_dim[2], n_coarse=hc.n_blocks, tau_fine=hf.tau,
                       tau_coarse=hc.tau, compressible=0)
    N.call("ol_restrict", C.byref(v), S._stream())
    torch.cuda.synchronize()
    orc.restrict(f_f, hf.obstacle, hf.map_x, hf.map_y, hf.map_z, hf.n_blocks, f_c, rho_c, vel_c,
                 hc.obstacle, hc.block_ptr, hc.grid_dim, hc.n_blocks, hf.tau, hc.tau, 0)
    g = d["f_c"].cpu().numpy()
    assert max_abs(g, f_c) < 1e-6
    assert not np.array_equal(g, np.repeat(w, 512 * hc.n_blocks))  # cells were replaced
    assert max_abs(d["rho_c"].cpu().numpy(), rho_c) < 1e-6
    # the recursion with restriction on
    st = S.StepSettings.from_config(c, False)
    st.restriction = 1
    gl = _run_gpu(hosts, p, st, 20, 0.05)
    ol = _run_oracle(hosts, p, st, 20, 0.05)
    for lg, lo in zip(gl, ol):
        assert rel_err(lg.f_temp.cpu().numpy(), lo.f_temp) < 1e-4
        assert rel_err(lg.rho.cpu().numpy(), lo.rho) < 1e-5


def test_two_level_thermal_ddf():
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5),
                                          compressibility_correction=True, ddf_enabled=True,
                                          u_target=np.float32(0.1))
    st = S.StepSettings.from_config(c, False)
    g = _run_gpu(hosts, p, st, 10, 0.1, ddf=True)
    o = _run_oracle(hosts, p, st, 10, 0.1, ddf=True)
    for lg, lo in zip(g, o):
        assert rel_err(lg.f_temp.cpu().numpy(), lo.f_temp) < 1e-4
        assert rel_err(lg.g_temp.cpu().numpy(), lo.g_temp) < 1e-4
        assert rel_err(lg.temperature.cpu().numpy(), lo.T) < 1e-5


def test_bouzidi_links_equal_sparse_form(case1):
    """The link-list correction (ol_bouzidi_build_links + _apply_links) gives
    the bits of ol_bouzidi_sparse, which visits every direction of every
    boundary cell."""
    c, mesh, p, hosts = case1
    h = hosts[0]
    n = h.n_blocks
    rng = np.random.default_rng(8)
    f0 = (np.repeat(weights32(), 512 * n) * rng.uniform(0.9, 1.1, 27 * 512 * n)).astype(np.float32)
    lv = S.upload_level(h, DEV)
    a, b = _t(f0), _t(f0)
    st = S.StepSettings.from_config(c, False)
    N.call("ol_bouzidi_sparse", S._ptr(a), S._ptr(lv.q_map), S._ptr(lv.cell_block),
           S._ptr(lv.cell_x), S._ptr(lv.cell_y), S._ptr(lv.cell_z), N.i32(h.n_boundary),
           S._ptr(lv.neighbor_table), N.i32(n), N.f32(st.q_min), S._ptr(lv.bouzidi_scratch),
           S._stream())
    S.build_bouzidi_links(lv, st.q_min)
    assert 0 < lv.bz_n_links < 27 * h.n_boundary
    N.call("ol_bouzidi_apply_links", S._ptr(b), S._ptr(lv.bz_links), N.i32(lv.bz_n_links),
           N.i32(n), S._ptr(lv.bouzidi_scratch), S._stream())
    torch.cuda.synchronize()
    assert torch.equal(a, b) and not torch.equal(a, _t(f0))
