"""The warp-specialised persistent stream-collide kernel (OL_SC_KERNEL_WS:
loader warps stage the next block while consumer warps collide the current
one) against the one-CTA-per-block kernel (OL_SC_KERNEL_BLOCK) and the oracle.

Both kernels stage the same values and run the same cell-update source, so
the pulls, rho and u agree bit for bit.  The post-collision populations of a
few cells may differ in the last bit: the compiler may fuse a product and a
sum into one multiply-add in one kernel and not in the other.  So:

* one level-1 sub-step for every cumulant variant (domain-boundary values
  evaluated by the loader warps), with one CTA per block and with a grid of
  7 CTAs (each walks ~18 blocks through both stages and the descriptor ring):
  rho and u bitwise equal, f within 2.5e-7 absolute (a few ulp of the
  largest population, 8/27) of the block kernel, and within the single-step
  oracle bar (2e-6 absolute, 1e-5 relative L2) of the oracle;
* the two-level recursion with paired ghost rows (coarse-to-fine values),
  4 coarse steps: relative L2 below 1e-6 on f, rho and u of both levels;
* the block pool (batched work items, FP32 and FP16-shifted storage),
  6 coarse steps: the same bar.

Every test also checks that no bounded wait of the kernel ran out.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import (interior_refined_case, max_abs, perturbed_state, rel_err,
                     small_sphere_case)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import _native as N  # noqa: E402
from openludwig_b200 import native as NT  # noqa: E402
from openludwig_b200 import solver as S  # noqa: E402
from oracle import oracle as orc  # noqa: E402

DEV = torch.device("cuda:0")
AUTO, BLOCK, WS = 0, 1, 2


def _kernel(choice, max_ctas=0):
    N.call("ol_set_stream_collide_kernel", N.i32(choice), N.i32(max_ctas))


def _faults():
    v = C.c_int32(-1)
    N.call("ol_pipeline_fault", C.byref(v))
    return v.value


@pytest.fixture(autouse=True)
def _policy():
    _kernel(AUTO)
    _faults()
    yield
    _kernel(AUTO)
    assert _faults() == 0


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.fixture(scope="module")
def sphere():
    return small_sphere_case(resolution=8)


CUMULANT = [
    dict(name="factored", op=0, limiter=1),
    dict(name="positivity", op=0, limiter=2),
    dict(name="none_fixed_w4", op=0, limiter=0, adaptive_omega4=0, omega_4=1.3),
    dict(name="wale", op=0, limiter=1, c_wale=0.5),
    dict(name="wale_bg_wallmodel", op=0, limiter=1, c_wale=0.5, nu_sgs_bg=1e-4, wall_model=1),
    dict(name="sponge_blend_turb", op=0, limiter=1, sponge_blend=1, inlet_turbulence=0.05),
    dict(name="compressible", op=0, limiter=1, compressible=1),
]


def _one_step(sphere, var, choice, max_ctas):
    c, mesh, p, hosts = sphere
    h = hosts[0]
    n = h.n_blocks
    f_in, vel_in = perturbed_state(n, seed=11)
    wd = h.wall_dist.copy()
    if var.get("wall_model"):
        wd = np.where(wd < 100.0, wd / np.float32(h.dx_exact), wd).astype(np.float32)
    st = S.StepSettings(**{k: v for k, v in var.items() if k != "name"})
    sp = S.step_params(st, type("L", (), {"tau": 0.52})(), 0.5, True,
                       (p.nx_coarse, p.ny_coarse, p.nz_coarse), 0.05, 37, 0.0, False)
    d_fin = _t(f_in)
    d_fout = torch.zeros(27 * 512 * n, dtype=torch.float32, device=DEV)
    d_vin = _t(vel_in)
    d_vout = torch.zeros(3 * 512 * n, dtype=torch.float32, device=DEV)
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
    _kernel(choice, max_ctas)
    N.call("ol_stream_collide", C.byref(view), C.byref(N.ParentView()), C.byref(sp), S._stream())
    torch.cuda.synchronize()
    inputs = dict(f_in=f_in, vel_in=vel_in, wd=wd, sp=sp)
    return (d_fout.cpu().numpy(), d_rho.cpu().numpy(), d_vout.cpu().numpy()), inputs


@pytest.mark.parametrize("max_ctas", [0, 7], ids=["cta_per_block", "7_ctas"])
@pytest.mark.parametrize("var", CUMULANT, ids=[v["name"] for v in CUMULANT])
def test_ws_single_step_matches_block_kernel_and_oracle(sphere, var, max_ctas):
    (fa, ra, va), _ = _one_step(sphere, var, BLOCK, 0)
    (fb, rb, vb), inp = _one_step(sphere, var, WS, max_ctas)
    assert np.array_equal(ra, rb) and np.array_equal(va, vb), var["name"]
    assert max_abs(fa, fb) <= 2.5e-7, var["name"]
    assert not np.array_equal(fb, np.zeros_like(fb))
    h = sphere[3][0]
    n = h.n_blocks
    o_f = np.zeros(27 * 512 * n, np.float32)
    o_rho = np.zeros(512 * n, np.float32)
    o_vel = np.zeros(3 * 512 * n, np.float32)
    params = {name: getattr(inp["sp"], name) for name, _ in N.STEP_FIELDS}
    orc.build()
    orc.stream_collide(dict(f_out=o_f, f_in=inp["f_in"], rho=o_rho, vel_out=o_vel,
                            vel_in=inp["vel_in"], obstacle=h.obstacle, sponge=h.sponge,
                            wall_dist=inp["wd"], neighbor_table=h.neighbor_table, map_x=h.map_x,
                            map_y=h.map_y, map_z=h.map_z, n_blocks=n), None, params)
    assert max_abs(fb, o_f) < 2e-6 and rel_err(fb, o_f) < 1e-5, var["name"]
    assert max_abs(rb, o_rho) < 2e-6 and max_abs(vb, o_vel) < 2e-6


def _recursion(hosts, p, st, steps, u, choice, max_ctas):
    _kernel(choice, max_ctas)
    levels = [S.upload_level(h, DEV, ghost=True) for h in hosts]
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)
    for t in range(1, steps + 1):
        S.recursive_step(levels, st, 0, t, None, 0.0, u, dims)
    torch.cuda.synchronize()
    return levels


@pytest.mark.parametrize("max_ctas", [0, 37], ids=["cta_per_sm", "37_ctas"])
def test_ws_recursion_equals_block_kernel(max_ctas):
    """Refined level inside the domain: every absent-neighbour value of the
    fine level is a ghost row written by the paired ghost pass."""
    c, mesh, p, hosts = interior_refined_case()
    st = S.StepSettings.from_config(c, c.wall_model_enabled)
    a = _recursion(hosts, p, st, 4, 0.05, BLOCK, 0)
    b = _recursion(hosts, p, st, 4, 0.05, WS, max_ctas)
    for la, lb in zip(a, b):
        for name in ("f", "f_temp", "rho", "vel", "vel_temp"):
            x, y = getattr(la, name).cpu().numpy(), getattr(lb, name).cpu().numpy()
            assert rel_err(y, x) < 1e-6, name


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_ws_block_pool_equals_block_kernel(storage):
    """Batched work items of a two-level case and a one-level case sharing
    the pool; the warp-specialised kernel at a grid of 11 CTAs."""
    cases = []
    for res, lv in ((16, 2), (8, 1)):
        c, mesh, p, hosts = small_sphere_case(resolution=res, levels=lv,
                                              c_wale=np.float32(0.5))
        c.ramp_steps = 0
        cases.append(NT.PreparedCase(c, mesh, p, hosts,
                                     S.StepSettings.from_config(c, c.wall_model_enabled)))
    out = []
    for choice, max_ctas in ((BLOCK, 0), (WS, 11)):
        _kernel(choice, max_ctas)
        ctx = NT.Context(budget_bytes=2 << 30, storage=storage)
        ids = [ctx.add_case(cs) for cs in cases]
        ctx.step(6)
        ctx.sync()
        got = []
        for cid, cs in zip(ids, cases):
            for lvl in range(1, len(cs.levels) + 1):
                got.extend(ctx.download(cid, lvl, f=True))
        out.append(got)
        ctx.close()
    for x, y in zip(*out):
        assert rel_err(y, x) < 1e-6


@pytest.mark.parametrize("max_ctas", [0, 13, 3], ids=["cta_per_sm", "13_ctas", "3_ctas"])
def test_thermal_ws_equals_block_kernel(max_ctas):
    """The warp-specialised thermal kernel (bulk-copied g planes landing in
    the pull-shifted stage) against the one-CTA-per-block thermal kernel on a
    two-level O(u^4) + DDF sphere (ghost rows on the refined level, domain
    boundaries on level 1, solid cells bouncing their own g), 4 coarse steps:
    f, g, rho, T and u of both levels within 1e-6 relative L2.  With 3 CTAs
    each walks dozens of blocks, so the producer's look-ahead (two stage
    buffers, descriptors of the next block) runs well ahead of the consumers."""
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5),
                                          compressibility_correction=True, ddf_enabled=True,
                                          u_target=np.float32(0.1))
    st = S.StepSettings.from_config(c, False)
    dims = (p.nx_coarse, p.ny_coarse, p.nz_coarse)

    def run(choice, ctas):
        _kernel(choice, ctas)
        levels = [S.upload_level(h, DEV, ddf=True, t_init=c.ddf_t_initial) for h in hosts]
        for t in range(1, 5):
            S.recursive_step(levels, st, 0, t, None, 0.0, 0.1, dims)
        torch.cuda.synchronize()
        return levels

    a = run(BLOCK, 0)
    b = run(WS, max_ctas)
    for la, lb in zip(a, b):
        for name in ("f", "f_temp", "g", "g_temp", "rho", "temperature", "vel", "vel_temp"):
            x, y = getattr(la, name).cpu().numpy(), getattr(lb, name).cpu().numpy()
            assert rel_err(y, x) < 1e-6, name
