"""Accuracy against the FP64 oracle (the same algorithm in double precision):
the FP32 time step and FP16-shifted storage after 100 steps of the sphere
case with Bouzidi walls.  Bars: density within 1e-5 and velocity within
1e-3 relative L2 for FP32; drag coefficient from the same surface-force
integration within 0.5 % (FP32) and 1 % (FP16-shifted storage)."""
import numpy as np
import pytest

from helpers import rel_err, small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import native as NT  # noqa: E402
from openludwig_b200 import solver as S  # noqa: E402
from oracle import driver as odrv  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DEV = torch.device("cuda:0")
STEPS = 100


def test_fp32_and_fp16_against_fp64_oracle():
    orc.build()
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    c.ramp_steps = 0
    u = float(c.u_target)
    sim = S.Simulation(c, mesh, p, hosts, DEV)
    sim.run(STEPS, diag_freq=STEPS)
    lv = sim.levels[-1]
    raw32 = S.compute_aerodynamics(lv, sim.dmesh, p, c)
    torch.cuda.synchronize()

    o = odrv.init_levels(hosts, dtype=np.float64)
    s = odrv.settings_dict(sim.settings)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    for t in range(1, STEPS + 1):
        odrv.recursive_step(o, s, 0, t, None, 0.0, u, dims, np.float64)
    o = o[-1]
    assert rel_err(lv.rho.cpu().numpy(), o.rho) < 1e-5
    assert rel_err(lv.vel.cpu().numpy(), o.vel) < 1e-3

    fp = S.force_params_for(lv, p, c)
    raw64, _ = orc.surface_forces(sim.dmesh.arrays.cpu().numpy(), o.rho.astype(np.float32),
                                  o.vel.astype(np.float32), lv.obstacle.cpu().numpy(),
                                  lv.block_ptr.cpu().numpy(), lv.n_blocks, fp)
    ref = (p.rho_physical, p.u_physical, p.reference_area, p.reference_chord)
    c64, c32 = NT.coefficients(raw64, *ref), NT.coefficients(raw32, *ref)
    cd64, cd32 = c64.Cd, c32.Cd
    assert cd64 > 0.0
    assert abs(cd32 - cd64) <= 5e-3 * abs(cd64)
    # mass drift: total density against the FP64 run's
    m32, m64 = float(lv.rho.double().sum()), float(o.rho.sum())
    assert abs(m32 - m64) <= 1e-6 * m64

    case = NT.PreparedCase(c, mesh, p, hosts, sim.settings)
    ctx = NT.Context(budget_bytes=1 << 30, storage="f16")
    cid = ctx.add_case(case)
    ctx.step(STEPS)
    c16 = ctx.forces(cid)
    rho16 = ctx.download(cid, 1)[0]
    ctx.close()
    assert abs(c16.Cd - cd64) <= 1e-2 * abs(cd64)
    m16 = float(np.asarray(rho16, np.float64).sum())
    print(f"\naccuracy vs FP64 after {STEPS} steps: FP32 rho L2 {rel_err(lv.rho.cpu().numpy(), o.rho):.2e}"
          f" u L2 {rel_err(lv.vel.cpu().numpy(), o.vel):.2e} Cd {abs(cd32 / cd64 - 1):.2e}"
          f" Cl {abs(c32.Cl - c64.Cl):.2e} (abs) mass {abs(m32 / m64 - 1):.2e};"
          f" FP16 storage Cd {abs(c16.Cd / cd64 - 1):.2e} Cl {abs(c16.Cl - c64.Cl):.2e} (abs)"
          f" mass {abs(m16 / m64 - 1):.2e}")
