"""Continuous-batching service through the library's serving layer
(ol_server_* / ol_serve_*, driven by serving.Server): requests that arrive
while others run are admitted as memory frees up, and every result equals
the same request run alone (bitwise: each case's kernels only read its own
state, and its force sums are fixed-order FP64).  Per-case control through
the C ABI: ol_ctx_case_step and the coefficient record."""
import numpy as np
import pytest

from helpers import small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import native as NT  # noqa: E402
from openludwig_b200 import serving as SV  # noqa: E402
from openludwig_b200 import solver as S  # noqa: E402


def _case(res, levels=1, **kw):
    c, mesh, p, hosts = small_sphere_case(resolution=res, levels=levels, **kw)
    c.ramp_steps = 0
    return NT.PreparedCase(c, mesh, p, hosts, S.StepSettings.from_config(c, c.wall_model_enabled))


def test_served_results_equal_alone_results():
    a = _case(8)
    b = _case(16, 2)
    kw = dict(check_every=20, window=40, tol=1e-9, max_steps=80)
    reqs = [SV.Request(0, 0.0, a), SV.Request(1, 0.0, b), SV.Request(2, 0.05, a)]
    ctx = NT.Context(budget_bytes=1 << 30, storage="f16")
    mixed = SV.Server(ctx, **kw).run(reqs)
    ctx.close()
    assert mixed["n"] == 3
    alone = {}
    for rid, case in ((0, a), (1, b)):
        ctx = NT.Context(budget_bytes=1 << 30, storage="f16")
        r = SV.Server(ctx, **kw).run([SV.Request(rid, 0.0, case)])
        ctx.close()
        alone[rid] = r["results"][0]
    by = {r.rid: r for r in mixed["results"]}
    assert by[0].cd_history == alone[0].cd_history
    assert by[2].cd_history == alone[0].cd_history
    assert by[1].cd_history == alone[1].cd_history
    assert mixed["p99_s"] >= mixed["p50_s"] > 0.0


def test_admission_waits_for_memory():
    a = _case(8)
    ctx = NT.Context(budget_bytes=1 << 30, storage="f16")
    need = ctx.footprint(a)
    ctx.close()
    budget = int(need * 1.5) + (need // 8)  # room for one case at a time
    ctx = NT.Context(budget_bytes=max(budget, 64 << 20), storage="f16")
    cap = ctx.stats()["budget"] // need
    reqs = [SV.Request(i, 0.0, a) for i in range(int(cap) + 2)]
    out = SV.Server(ctx, check_every=10, window=20, tol=1e-9, max_steps=20).run(reqs)
    ctx.close()
    assert out["n"] == len(reqs)
    admits = sorted(r.admit_s for r in out["results"])
    assert admits[-1] > admits[0]      # later requests waited for a retirement
    assert all(np.isfinite(r.cd) for r in out["results"])


def test_lazy_requests_count_their_preparation():
    """A request given as a preparation function is prepared on arrival, and
    its latency includes that preparation."""
    a = _case(8)

    def make():
        import time
        time.sleep(0.2)
        return a

    ctx = NT.Context(budget_bytes=1 << 30, storage="f16")
    out = SV.Server(ctx, check_every=10, window=20, tol=1e-9, max_steps=20).run(
        [SV.Request(0, 0.0, make)])
    ctx.close()
    r = out["results"][0]
    assert r.prep_s >= 0.2 and r.latency_s >= r.prep_s and r.steps == 20


def test_case_step_moves_one_case_and_matches_alone():
    """ol_ctx_case_step advances one resident case only; its state is the
    state of the case stepped alone, and u_in fixes its inlet speed the same
    way in a mix as alone."""
    a = _case(8)
    b = _case(16, 2)
    ctx = NT.Context(budget_bytes=1 << 30, storage="f32")
    ca, cb = ctx.add_case(a), ctx.add_case(b)
    ctx.case_step(ca, 5)
    assert ctx.info(ca)[0] == 5 and ctx.info(cb)[0] == 0
    fa = ctx.download(ca, 1, f=True)[2]
    ctx.step(2)                                   # the full plan again: both move
    assert ctx.info(ca)[0] == 7 and ctx.info(cb)[0] == 2
    ctx.case_step(cb, 3, u_in=0.03)
    assert ctx.info(cb)[0] == 5 and ctx.info(ca)[0] == 7
    fb = ctx.download(cb, 2, f=True)[2]
    ctx.close()
    alone = NT.Context(budget_bytes=1 << 30, storage="f32")
    ia = alone.add_case(a)
    alone.step(5)
    assert np.array_equal(alone.download(ia, 1, f=True)[2], fa)
    alone.close()
    ref = NT.Context(budget_bytes=1 << 30, storage="f32")
    ib = ref.add_case(b)
    ref.step(2)
    ref.case_step(ib, 3, u_in=0.03)
    assert np.array_equal(ref.download(ib, 2, f=True)[2], fb)
    ref.close()


def test_coefficient_record_matches_the_raw_sums():
    a = _case(8)
    ctx = NT.Context(budget_bytes=1 << 30, storage="f32")
    cid = ctx.add_case(a)
    ctx.step(20)
    rec = ctx.coefficient_record(cid)
    raw = ctx.forces_raw(cid)
    fr = ctx.forces(cid)
    ctx.close()
    assert rec["Cd"] == fr.Cd and rec["Cl"] == fr.Cl and rec["Cs"] == fr.Cs
    assert rec["Cmy"] == fr.Cmy
    assert rec["Fx"] == raw[0] + raw[3] and rec["Mz"] == raw[8]
    assert rec["Cd"] != 0.0
