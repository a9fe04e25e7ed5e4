"""Native multi-case context on the GPU.

* FP32 pool storage reproduces the drop-in path (same kernels, the schedule
  and A/B bookkeeping done on the device) to FP32 rounding.
* A case's result is bitwise the same alone and in a mix of other cases.
* FP16-shifted storage stays within 2e-3 relative L2 of FP32 populations
  and within 1 % in Cd over the test horizon.
* Admission is refused beyond the HBM budget; a NaN planted in one case's
  host-uploaded state raises that case's watchdog bit and leaves the other
  case bitwise unchanged.
"""
import numpy as np
import pytest

from helpers import interior_refined_case, rel_err, small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import _native as N  # noqa: E402
from openludwig_b200 import native as NT  # noqa: E402
from openludwig_b200 import solver as S  # noqa: E402
from openludwig_b200 import workloads  # noqa: E402

DEV = torch.device("cuda:0")


def _case(resolution=8, levels=1, **kw):
    c, mesh, p, hosts = small_sphere_case(resolution=resolution, levels=levels, **kw)
    c.ramp_steps = 0
    return NT.PreparedCase(c, mesh, p, hosts, S.StepSettings.from_config(c, c.wall_model_enabled))


@pytest.fixture(scope="module")
def one_level():
    return _case(8)


@pytest.fixture(scope="module")
def two_level():
    return _case(16, 2, c_wale=np.float32(0.5))


def _dropin(case, steps):
    levels = [S.upload_level(h, DEV) for h in case.levels]
    dims = (case.params.nx_coarse, case.params.ny_coarse, case.params.nz_coarse)
    for t in range(1, steps + 1):
        S.recursive_step(levels, case.settings, 0, t, None, 0.0, float(case.cfg.u_target), dims)
    torch.cuda.synchronize()
    return levels


@pytest.fixture(scope="module")
def interior_two_level():
    c, mesh, p, hosts = interior_refined_case()
    return NT.PreparedCase(c, mesh, p, hosts, S.StepSettings.from_config(c, c.wall_model_enabled))


@pytest.mark.parametrize("which", ["one_level", "two_level", "interior_two_level"])
def test_native_f32_matches_dropin(which, request):
    """interior_two_level: no refined block has a domain-boundary value, so
    the second sub-step of each pair launches no ghost pass at all."""
    case = request.getfixturevalue(which)
    steps = 10
    ctx = NT.Context(budget_bytes=2 << 30, storage="f32")
    cid = ctx.add_case(case)
    ctx.step(steps)
    ctx.sync()
    ref = _dropin(case, steps)
    for lvl, lv in enumerate(ref, start=1):
        rho, vel, f = ctx.download(cid, lvl, f=True)
        sub = 1 << (lvl - 1)
        last = steps * sub + sub - 1          # t_sub of the level's last sub-step
        newest = lv.f_temp if last % 2 == 0 else lv.f
        assert rel_err(f, newest.cpu().numpy()) < 1e-6
        assert rel_err(rho, lv.rho.cpu().numpy()) < 1e-6
    steps_done, status = ctx.info(cid)
    assert steps_done == steps and status == 0
    ctx.close()


def test_native_ddf_matches_dropin():
    """Thermal DDF in the pool (refined-level ghost rows for f and g filled in
    the coarse-step graph) against the drop-in path, both FP32."""
    case = _case(16, 2, c_wale=np.float32(0.5), compressibility_correction=True,
                 ddf_enabled=True, u_target=np.float32(0.1))
    steps = 6
    ctx = NT.Context(budget_bytes=2 << 30, storage="f32", ddf=True)
    cid = ctx.add_case(case)
    ctx.step(steps)
    ctx.sync()
    levels = [S.upload_level(h, DEV, ddf=True) for h in case.levels]
    dims = (case.params.nx_coarse, case.params.ny_coarse, case.params.nz_coarse)
    for t in range(1, steps + 1):
        S.recursive_step(levels, case.settings, 0, t, None, 0.0, float(case.cfg.u_target), dims)
    torch.cuda.synchronize()
    for lvl, lv in enumerate(levels, start=1):
        sub = 1 << (lvl - 1)
        last = steps * sub + sub - 1
        newest_g = lv.g_temp if last % 2 == 0 else lv.g
        T, g = ctx.download_thermal(cid, lvl, g=True)
        assert rel_err(g, newest_g.cpu().numpy()) < 1e-6
        assert rel_err(T, lv.temperature.cpu().numpy()) < 1e-6
    ctx.close()


def test_alone_equals_in_mix(one_level, two_level):
    steps = 8
    a = NT.Context(budget_bytes=2 << 30, storage="f16")
    ca = a.add_case(one_level)
    a.step(steps)
    fa = a.download(ca, 1, f=True)[2]
    a.close()
    b = NT.Context(budget_bytes=2 << 30, storage="f16")
    b.add_case(two_level)
    cb = b.add_case(one_level)
    b.step(steps)
    fb = b.download(cb, 1, f=True)[2]
    b.close()
    assert np.array_equal(fa, fb)


def test_f16_storage_close_to_f32(one_level):
    steps = 40
    out = {}
    for st in ("f32", "f16"):
        ctx = NT.Context(budget_bytes=2 << 30, storage=st)
        cid = ctx.add_case(one_level)
        ctx.step(steps)
        out[st] = (ctx.download(cid, 1, f=True), ctx.forces(cid))
        ctx.close()
    (r32, v32, f32), F32 = out["f32"]
    (r16, v16, f16), F16 = out["f16"]
    assert rel_err(f16, f32) < 2e-3
    assert rel_err(r16, r32) < 1e-4
    assert abs(F16.Cd - F32.Cd) <= 0.01 * abs(F32.Cd) + 1e-6


def test_budget_admission_and_removal(one_level):
    ctx = NT.Context(budget_bytes=256 << 20, storage="f16")
    need = ctx.footprint(one_level)
    n = 0
    ids = []
    while True:
        try:
            ids.append(ctx.add_case(one_level))
            n += 1
        except N.OLError as e:
            assert e.code == 3  # OL_ERR_NOMEM
            break
        assert n < 100
    # the pool holds 15/16 of the budget; the rest is per-case metadata
    assert int(0.85 * (256 << 20) / need) <= n <= (256 << 20) // need
    ctx.remove_case(ids[0])
    ids[0] = ctx.add_case(one_level)   # space is reusable
    ctx.step(2)
    ctx.sync()
    assert ctx.stats()["cases"] == len(ids)
    ctx.close()


def test_nan_watchdog_isolated_to_its_case(one_level):
    bad = NT.PreparedCase(**{k: getattr(one_level, k) for k in ("cfg", "mesh", "params", "levels",
                                                                  "settings", "name")})
    import copy
    bad.levels = copy.deepcopy(one_level.levels)
    bad.levels[0].sponge = bad.levels[0].sponge.copy()
    # fault planted on the host: an infinite sponge weight turns the blended
    # density into inf - inf = NaN on the first step
    bad.levels[0].sponge[1000] = np.float32(np.inf)
    steps = 6
    ref = NT.Context(budget_bytes=2 << 30, storage="f32")
    cr = ref.add_case(one_level)
    ref.step(steps)
    f_ref = ref.download(cr, 1, f=True)[2]
    ref.close()
    ctx = NT.Context(budget_bytes=2 << 30, storage="f32")
    good = ctx.add_case(one_level)
    badid = ctx.add_case(bad)
    ctx.step(steps)
    ctx.sync()
    assert ctx.info(badid)[1] & 1
    assert ctx.info(good)[1] == 0
    assert np.array_equal(ctx.download(good, 1, f=True)[2], f_ref)
    ctx.remove_case(badid)   # retire the faulted case, keep the other running
    ctx.step(2)
    assert ctx.info(good)[1] == 0
    ctx.close()


SHAPES = {"ws": -2, "pipelined": -1, "per_item": 0, "grid_1x": 1, "grid_2x": 2}


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_every_launch_shape_gives_the_same_state(storage, two_level):
    """Every launch shape the autotuner chooses among, against one CTA per
    item: the persistent grids run the same kernel (same bits); the
    pipelined and warp-specialised kernels stage the same values and run the
    same cell update, and may differ only where the compiler fused a
    multiply-add differently (relative L2 below 1e-6 after 6 steps)."""
    out = {}
    for name, shape in SHAPES.items():
        ctx = NT.Context(budget_bytes=2 << 30, storage=storage)
        cid = ctx.add_case(two_level)
        ctx.set_launch(shape)
        assert ctx.launch() == shape
        ctx.step(6)
        out[name] = [ctx.download(cid, lvl, f=True) for lvl in (1, 2)]
        assert ctx.info(cid) == (6, 0)
        ctx.close()
    ref = out["per_item"]
    for name, got in out.items():
        for (r0, v0, f0), (r1, v1, f1) in zip(ref, got):
            if name.startswith("grid"):
                assert np.array_equal(f0, f1) and np.array_equal(r0, r1), name
            else:
                assert rel_err(f1, f0) < 1e-6 and rel_err(r1, r0) < 1e-6, name


def test_autotune_keeps_results_valid(one_level):
    """The tuner keeps one of the shapes, and the state it leaves behind is
    the state of the same number of steps under one CTA per item."""
    ctx = NT.Context(budget_bytes=2 << 30, storage="f32")
    cid = ctx.add_case(one_level)
    ctx.autotune(1)
    assert ctx.launch() in SHAPES.values()
    steps, status = ctx.info(cid)
    assert steps == 5 * 2 and status == 0
    f_tuned = ctx.download(cid, 1, f=True)[2]
    ctx.close()
    ref = NT.Context(budget_bytes=2 << 30, storage="f32")
    rid = ref.add_case(one_level)
    ref.set_launch(0)
    ref.step(steps)
    f_ref = ref.download(rid, 1, f=True)[2]
    ref.close()
    assert rel_err(f_tuned, f_ref) < 1e-6


def test_autotune_per_variant_on_a_two_variant_mix(one_level, two_level):
    """A mix of a case without WALE and one with it holds two collision
    variants: the tuner times the whole mix, then each variant's shape with
    the other held, and every case steps 5 * 2 + 2 * 5 * 2 = 30 coarse steps
    (trials = 1).  The state it leaves is that of the same steps under one
    CTA per item."""
    ctx = NT.Context(budget_bytes=2 << 30, storage="f32")
    ids = [ctx.add_case(c) for c in (one_level, two_level)]
    ctx.autotune(1)
    shapes = {w: ctx.variant_launch(0, w) for w in (False, True)}
    assert all(v in SHAPES.values() for v in shapes.values())
    assert [ctx.info(i) for i in ids] == [(30, 0), (30, 0)]
    got = [ctx.download(i, lvl, f=True)[2] for i, c in zip(ids, (one_level, two_level))
           for lvl in range(1, len(c.levels) + 1)]
    ctx.close()
    ref = NT.Context(budget_bytes=2 << 30, storage="f32")
    rids = [ref.add_case(c) for c in (one_level, two_level)]
    ref.set_launch(0)
    assert ref.variant_launch(0, True) == 0
    ref.step(30)
    want = [ref.download(i, lvl, f=True)[2] for i, c in zip(rids, (one_level, two_level))
            for lvl in range(1, len(c.levels) + 1)]
    ref.close()
    for g, w in zip(got, want):
        assert rel_err(g, w) < 1e-6
