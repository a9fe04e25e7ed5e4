"""The FP64 GPU accuracy oracle (oracle/ol_oracle_gpu.cu: the oracle's
per-cell restatement run one thread per cell) and accuracy at the benchmark
configurations against it.

Pinning the GPU oracle to the CPU oracle (same source, ol_oracle_cell.h):
* FP32, no wall model: bit for bit after 3 coarse steps (both builds round
  every operation as written; sqrt and division are correctly rounded on
  both sides);
* FP32 with the wall model (pow, log from different math libraries) and
  FP64 everywhere: relative L2 below 1e-6 (FP32) / 1e-12 (FP64).

Accuracy against the FP64 GPU oracle, forces time-averaged the way the
reference's main loop samples them (main_loop_batches; surface forces of
the finest level in FP32, as the reference computes them):
* the three-level cube (160x80x80 coarsest, Re 1e5, WALE + wall model):
  500 coarse steps (2000 finest), FP32 drop-in path and FP16-shifted block
  pool;
* the thermal sphere (O(u^4) + DDF, 2 levels): 100 coarse steps, FP32 drop-in
  path: Cd, and rho / T relative L2;
* eight cases of the seeded batch mix in one FP16-shifted pool: 400 steps.
Bars: Cd within 0.5 % (FP32) and 1 % (FP16-shifted storage), Cl and Cs
within the same fractions of Cd.  The measured errors are printed.
"""
import numpy as np
import pytest

from helpers import interior_refined_case, rel_err, small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import domain, native as NT, scaling, solver as S, workloads  # noqa: E402
from oracle import driver as odrv  # noqa: E402
from oracle import gpu as ogpu  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DEV = torch.device("cuda:0")


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()
    ogpu.build()


def _state(levels, ddf):
    out = []
    for lv in levels:
        names = ["f", "f_temp", "rho", "vel", "vel_temp"] + (["g", "g_temp", "T"] if ddf else [])
        for n in names:
            a = getattr(lv, n)
            out.append(a.cpu().numpy() if isinstance(a, torch.Tensor) else a)
    return out


def _run_both(case, steps, dtype, ddf=False):
    c, mesh, p, hosts = case
    st = S.StepSettings.from_config(c, c.wall_model_enabled)
    s = odrv.settings_dict(st)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    u = float(c.u_target)
    npd = np.float32 if dtype == torch.float32 else np.float64
    cpu = odrv.init_levels(hosts, dtype=npd, ddf=ddf, t_init=1.0)
    gpu = ogpu.init_levels(hosts, dtype, ddf=ddf, t_init=1.0, device=DEV)
    for t in range(1, steps + 1):
        odrv.recursive_step(cpu, s, 0, t, None, 0.0, u, dims, npd)
        odrv.recursive_step(gpu, s, 0, t, None, 0.0, u, dims, npd, k=ogpu)
    torch.cuda.synchronize()
    return _state(cpu, ddf), _state(gpu, ddf)


PIN_CASES = {
    "sphere_2lvl": lambda: small_sphere_case(resolution=16, levels=2),
    "sphere_ddf_2lvl": lambda: small_sphere_case(resolution=16, levels=2, ddf_enabled=True,
                                                 compressibility_correction=True),
    "cube_interior_wale": interior_refined_case,
}


@pytest.mark.parametrize("name", list(PIN_CASES))
def test_gpu_oracle_fp32_bit_exact_to_cpu_oracle(name):
    case = PIN_CASES[name]()
    ddf = bool(case[0].ddf_enabled)
    a, b = _run_both(case, 3, torch.float32, ddf)
    for x, y in zip(a, b):
        assert np.array_equal(x, y), name


def test_gpu_oracle_wall_model_and_fp64_match_cpu_oracle():
    case = interior_refined_case()
    case[0].wall_model_enabled = True
    a, b = _run_both(case, 3, torch.float32)
    assert max(rel_err(y, x) for x, y in zip(a, b)) < 1e-6
    a, b = _run_both(case, 3, torch.float64)
    assert max(rel_err(y, x) for x, y in zip(a, b)) < 1e-12
    case = small_sphere_case(resolution=16, levels=2, ddf_enabled=True)
    a, b = _run_both(case, 3, torch.float64, ddf=True)
    assert max(rel_err(y, x) for x, y in zip(a, b)) < 1e-12


# ----------------------------------------------------------------- accuracy

def _sample_steps(cfg, steps, diag):
    """Diagnostics steps of the reference's loop that are averaged."""
    return [b for b in S.main_loop_batches(1, steps, cfg.async_depth, diag, 10 ** 9,
                                           cfg.ramp_steps, cfg.u_target)]


def _fp64_averaged(cfg, p, hosts, steps, diag, fin, ddf=False):
    mesh_arrays, obstacle, block_ptr, fp = fin
    st = S.StepSettings.from_config(cfg, cfg.wall_model_enabled)
    s = odrv.settings_dict(st)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    lv64 = ogpu.init_levels(hosts, torch.float64, ddf=ddf, t_init=cfg.ddf_t_initial, device=DEV)
    acc, n = np.zeros(9), 0
    for b in _sample_steps(cfg, steps, diag):
        for t in range(b.t, b.end + 1):
            odrv.recursive_step(lv64, s, 0, t, None, 0.0, b.u, dims, np.float64, k=ogpu)
        if b.diag_step is not None and b.diag_step > cfg.ramp_steps:
            fl = lv64[-1]
            raw, _ = orc.surface_forces(mesh_arrays, fl.rho.float().cpu().numpy(),
                                        fl.vel.float().cpu().numpy(), obstacle, block_ptr,
                                        fl.host.n_blocks, fp)
            acc += raw
            n += 1
    torch.cuda.synchronize()
    return acc / n, n, lv64


def _pool_averaged(case, cfg, steps, diag, storage):
    ctx = NT.Context(budget_bytes=16 << 30, storage=storage)
    cid = ctx.add_case(case)
    acc, n, done = np.zeros(9), 0, 0
    for b in _sample_steps(cfg, steps, diag):
        if b.diag_step is not None and b.diag_step > cfg.ramp_steps:
            ctx.step(b.end - done)
            done = b.end
            acc += ctx.forces_raw(cid)
            n += 1
    ctx.close()
    return acc / n, n


def _errors(got, ref, p):
    r = (p.rho_physical, p.u_physical, p.reference_area, p.reference_chord)
    a, b = NT.coefficients(got, *r), NT.coefficients(ref, *r)
    return (abs(a.Cd / b.Cd - 1), abs(a.Cl - b.Cl) / abs(b.Cd), abs(a.Cs - b.Cs) / abs(b.Cd),
            b.Cd)


def _fp32_run(cfg, mesh, p, hosts, steps, diag):
    sim = S.Simulation(cfg, mesh, p, hosts, DEV)
    sim.run(steps, diag_freq=diag)
    lv = sim.levels[-1]
    fin = (sim.dmesh.arrays.cpu().numpy(), lv.obstacle.cpu().numpy(), lv.block_ptr.cpu().numpy(),
           S.force_params_for(lv, p, cfg))
    return sim, fin


def test_cube_3lvl_fp32_and_fp16_against_fp64_gpu_oracle():
    cfg, mesh, p, hosts = workloads.build_case("cube_3lvl")
    steps, diag = 500, 100
    sim, fin = _fp32_run(cfg, mesh, p, hosts, steps, diag)
    raw32 = sim.acc / sim.n_avg
    case = NT.PreparedCase(cfg, mesh, p, hosts, sim.settings)
    raw16, n16 = _pool_averaged(case, cfg, steps, diag, "f16")
    raw64, n64, lv64 = _fp64_averaged(cfg, p, hosts, steps, diag, fin)
    assert sim.n_avg == n16 == n64 == steps // diag
    e32, e16 = _errors(raw32, raw64, p), _errors(raw16, raw64, p)
    rho_err = rel_err(sim.levels[-1].rho.double().cpu().numpy(), lv64[-1].rho.cpu().numpy())
    print(f"\ncube_3lvl, {steps} coarse steps, Cd averaged over {n64} samples: FP64 Cd "
          f"{e32[3]:.5f}; FP32 Cd {e32[0]:.2e} Cl {e32[1]:.2e} Cs {e32[2]:.2e}; FP16 storage "
          f"Cd {e16[0]:.2e} Cl {e16[1]:.2e} Cs {e16[2]:.2e}; finest rho (FP32) {rho_err:.2e}")
    assert max(e32[:3]) <= 5e-3
    assert max(e16[:3]) <= 1e-2


def test_sphere_ddf_fp32_against_fp64_gpu_oracle():
    cfg, mesh, p, hosts = workloads.build_case("sphere_ddf")
    steps, diag = 100, 50
    sim, fin = _fp32_run(cfg, mesh, p, hosts, steps, diag)
    raw32 = sim.acc / sim.n_avg
    raw64, n64, lv64 = _fp64_averaged(cfg, p, hosts, steps, diag, fin, ddf=True)
    e32 = _errors(raw32, raw64, p)
    g, o = sim.levels[-1], lv64[-1]
    er = rel_err(g.rho.double().cpu().numpy(), o.rho.cpu().numpy())
    et = rel_err(g.temperature.double().cpu().numpy(), o.T.cpu().numpy())
    print(f"\nsphere_ddf, {steps} coarse steps: FP64 Cd {e32[3]:.5f}; FP32 Cd {e32[0]:.2e} "
          f"Cl {e32[1]:.2e}; finest rho {er:.2e} T {et:.2e}")
    assert max(e32[:3]) <= 5e-3
    assert er < 1e-4 and et < 1e-4


def test_batch_mix_fp16_pool_against_fp64_gpu_oracle():
    mix = workloads.batch_mix(48, seed=1234)[:8]
    steps, diag = 400, 200
    cases = []
    for m in mix:
        cfg, mesh = workloads.mix_case_config(m)
        cfg.ramp_steps = 0
        p = scaling.compute_domain_from_mesh(cfg, mesh.min_bounds, mesh.max_bounds)
        hosts = domain.setup_multilevel_domain(cfg, mesh, p)
        st = S.StepSettings.from_config(cfg, cfg.wall_model_enabled)
        cases.append(NT.PreparedCase(cfg, mesh, p, hosts, st))
    ctx = NT.Context(budget_bytes=32 << 30, storage="f16")
    ids = [ctx.add_case(c) for c in cases]
    acc16 = [np.zeros(9) for _ in cases]
    for k in range(steps // diag):
        ctx.step(diag)
        for i, cid in enumerate(ids):
            acc16[i] += ctx.forces_raw(cid)
    ctx.close()
    worst = []
    for i, cs in enumerate(cases):
        lv = S.upload_level(cs.levels[-1], DEV)
        dmesh = S.upload_mesh(cs.mesh, DEV)
        fin = (dmesh.arrays.cpu().numpy(), lv.obstacle.cpu().numpy(), lv.block_ptr.cpu().numpy(),
               S.force_params_for(lv, cs.params, cs.cfg))
        raw64, n64, _ = _fp64_averaged(cs.cfg, cs.params, cs.levels, steps, diag, fin)
        e = _errors(acc16[i] / (steps // diag), raw64, cs.params)
        worst.append(e)
        print(f"\nmix case {i} ({mix[i].kind} {mix[i].size_cells} cells, {mix[i].levels} levels, "
              f"Re {mix[i].re:.3g}): FP64 Cd {e[3]:.4f}; FP16 pool Cd {e[0]:.2e} Cl {e[1]:.2e} "
              f"Cs {e[2]:.2e}")
    assert max(max(w[:3]) for w in worst) <= 1e-2
