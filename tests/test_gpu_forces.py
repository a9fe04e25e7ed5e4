"""GPU surface-stress forces against the oracle restatement of
map_stresses_kernel! + integrate_forces_kernel! (surface.jl:350-762).

The per-triangle probe/stress arithmetic is FP32 on both sides (FMA
contraction differs); sums are FP64 on both sides.  Tolerances: per-triangle
pressure within 1e-4 relative to its scale, the nine sums within 1e-4
relative, Cd within 0.5 % of the oracle after a flow develops."""
import numpy as np
import pytest

from helpers import small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import solver as S  # noqa: E402
from openludwig_b200.native import coefficients  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DEV = torch.device("cuda:0")


def test_forces_match_oracle_after_flow_develops():
    orc.build()
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    c.ramp_steps = 0
    sim = S.Simulation(c, mesh, p, hosts, DEV)
    sim.run(60, diag_freq=30)
    lv = sim.levels[-1]
    raw, maps = S.compute_aerodynamics(lv, sim.dmesh, p, c, maps=True)
    torch.cuda.synchronize()
    fp = S.force_params_for(lv, p, c)
    o_raw, o_maps = orc.surface_forces(sim.dmesh.arrays.cpu().numpy(), lv.rho.cpu().numpy(),
                                       lv.vel.cpu().numpy(), lv.obstacle.cpu().numpy(),
                                       lv.block_ptr.cpu().numpy(), lv.n_blocks, fp)
    g_maps = maps.cpu().numpy()
    scale = np.abs(o_maps[0]).max()
    assert scale > 0
    assert np.max(np.abs(g_maps[0] - o_maps[0])) <= 1e-4 * scale
    for j in range(9):
        assert abs(raw[j] - o_raw[j]) <= 1e-4 * max(1e-12, np.abs(o_raw).max())
    cg = coefficients(raw, p.rho_physical, p.u_physical, p.reference_area, p.reference_chord)
    co = coefficients(o_raw, p.rho_physical, p.u_physical, p.reference_area, p.reference_chord)
    assert cg.Cd == pytest.approx(co.Cd, rel=5e-3)
    assert cg.Cd > 0.0   # drag points downstream once the flow is established
    assert len(sim.history) == 2 and "Cd" in sim.history[-1]


def _plate_sim(steps=60):
    from openludwig_b200 import domain, geometry as geo, scaling, workloads
    c, _ = workloads.sphere_1lvl(8)
    c.ramp_steps = 0
    c.alpha_deg = 15.0
    mesh = geo.rotate_mesh(geo.flat_plate(1.0, 8), 15.0, 0.0)
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    sim = S.Simulation(c, mesh, p, hosts, DEV)
    sim.run(steps, diag_freq=steps)
    return sim, c, p


@pytest.mark.parametrize("closed", [False, True])
def test_net_forces_match_oracle_on_open_plate(closed):
    """Two-sided net force (surface.jl:980-1034) on an inclined open plate:
    fluid on both sides, so the minus-side probe finds flow for most
    triangles.  Per-triangle maps and net forces within 1e-4 of their scale."""
    orc.build()
    sim, c, p = _plate_sim()
    lv = sim.levels[-1]
    (fx, fy, fz), maps = S.compute_net_aerodynamics(lv, sim.dmesh, p, c, closed_body=closed,
                                                    maps=True)
    fp = S.force_params_for(lv, p, c)
    o_maps, o_net = orc.surface_net_forces(sim.dmesh.arrays.cpu().numpy(), lv.rho.cpu().numpy(),
                                           lv.vel.cpu().numpy(), lv.obstacle.cpu().numpy(),
                                           lv.block_ptr.cpu().numpy(), lv.n_blocks, fp, closed)
    g_maps = maps.cpu().numpy()
    for j in range(8):
        scale = max(np.abs(o_maps[j]).max(), np.abs(o_maps[0]).max())
        assert np.max(np.abs(g_maps[j] - o_maps[j])) <= 1e-4 * scale
    g_net = np.stack([fx, fy, fz])
    scale = np.abs(o_net).max()
    assert scale > 0
    assert np.max(np.abs(g_net - o_net)) <= 1e-4 * scale
    minus_cover = np.count_nonzero(np.abs(o_maps[4]) > 1e-10)
    if closed:
        assert minus_cover == 0 and not g_maps[4:].any()
        # closed body: the net force sums to the one-sided integrated force
        raw = S.compute_aerodynamics(lv, sim.dmesh, p, c)
        tot = g_net.astype(np.float64).sum(axis=1)
        ref = raw[0:3] + raw[3:6]
        assert np.allclose(tot, ref, rtol=1e-4, atol=1e-4 * np.abs(ref).max())
    else:
        assert minus_cover > 0.8 * sim.dmesh.n


def test_flow_stats_match_numpy_fp64():
    """compute_flow_stats (diagnostics.jl:43-93) in FP64 against numpy on the
    same device state; the asynchronous entry point gives the same bits."""
    import ctypes as C
    from openludwig_b200 import _native as N
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    c.ramp_steps = 0
    sim = S.Simulation(c, mesh, p, hosts, DEV)
    sim.run(20, diag_freq=20)
    lv = sim.levels[0]
    st = S.flow_stats(lv)
    torch.cuda.synchronize()
    rho = lv.rho.cpu().numpy().astype(np.float64)
    vel = lv.vel.cpu().numpy().astype(np.float64).reshape(3, -1)
    fluid = lv.obstacle.cpu().numpy() == 0
    v2 = (vel ** 2).sum(axis=0)
    assert st["n_fluid"] == int(fluid.sum())
    assert st["rho_mean"] == pytest.approx(rho[fluid].mean(), rel=1e-12)
    assert st["rho_min"] == rho[fluid].min() and st["rho_max"] == rho[fluid].max()
    assert st["v_max"] == pytest.approx(np.sqrt(v2[fluid]).max(), rel=1e-15)
    assert st["kinetic_energy"] == pytest.approx((0.5 * rho * v2)[fluid].sum(), rel=1e-12)
    assert st["mass"] == pytest.approx(rho.sum(), rel=1e-12)
    nb = lv.n_blocks
    partials = torch.empty(int(N.lib().ol_flow_stats_scratch_doubles(nb)), dtype=torch.float64,
                           device=DEV)
    out = (C.c_double * 7)()
    N.call("ol_flow_stats", S._ptr(lv.rho), S._ptr(lv.vel), S._ptr(lv.obstacle), N.i32(nb),
           S._ptr(partials), out, S._stream())
    dev7 = torch.empty(7, dtype=torch.float64, device=DEV)
    N.call("ol_flow_stats_device", S._ptr(lv.rho), S._ptr(lv.vel), S._ptr(lv.obstacle), N.i32(nb),
           S._ptr(partials), S._ptr(dev7), S._stream())
    assert dev7.cpu().numpy().tolist() == list(out)
