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
