"""Main-loop policy (main.jl:208-315) and the run records: CPU tests.

* main_loop_batches against a transcription of the reference's while loop,
  written out here statement by statement (batch ends, per-batch inlet
  velocity, diagnostics and output steps), over batch sizes that do and do
  not divide the diagnostics and output intervals, runs that end mid-batch
  and runs that start after an earlier one.
* ramp_velocity: Float32 arithmetic (every intermediate a Float32), constant
  within a batch, 0 -> u_target monotone over the ramp, exactly u_target
  after it and with no ramp, and the value Julia's Float32 expression gives
  wherever cos is not within 2^-33 of a Float32 rounding midpoint.
* convergence.csv / forces.csv rows against the C library's printf with
  the reference's format strings; the LBMP surface file against a byte-level
  reading of forces/io.jl:236-351's layout; the net-force table's inverse
  rotation in Float32.
"""
import ctypes as C
import ctypes.util
import math
import struct

import numpy as np
import pytest

from openludwig_b200 import records as R
from openludwig_b200.native import coefficients
from openludwig_b200.solver import main_loop_batches, ramp_velocity

F32 = np.float32


def reference_loop(first, last, batch, diag, out_freq, ramp, u_target):
    """main.jl:212-313 as written (Julia's ÷ is floor division on positives)."""
    got = []
    t = first
    while t <= last:
        batch_end = min(t + batch - 1, last)
        actual = batch_end - t + 1
        if batch_end <= ramp:
            prog = F32(0.5) * (F32(1.0) - F32(math.cos(float(F32(F32(math.pi) * F32(batch_end))
                                                              / F32(ramp)))))
        else:
            prog = F32(1.0)
        u_curr = F32(u_target) * prog
        d_step = o_step = None
        if batch_end % diag < actual or batch_end == last:
            diag_step = (batch_end // diag) * diag
            if diag_step >= t and diag_step <= batch_end:
                d_step = diag_step
        if batch_end % out_freq < actual:
            out_step = (batch_end // out_freq) * out_freq
            if out_step >= t and out_step <= batch_end:
                o_step = out_step
        got.append((t, batch_end, actual, float(u_curr), d_step, o_step))
        t = batch_end + 1
    return got


SCHEDULES = [
    (1, 2000, 8, 100, 100, 0),       # benchmark defaults: batch divides both
    (1, 2000, 8, 500, 100, 1500),    # reference defaults: ramp 1500
    (1, 1003, 7, 100, 250, 300),     # batch divides neither; run ends mid-batch
    (1, 95, 8, 100, 40, 50),         # run shorter than one diagnostics interval
    (201, 600, 12, 200, 200, 1000),  # a continuation run, still inside the ramp
    (1, 64, 1, 5, 3, 10),            # unbatched
    (1, 333, 50, 30, 70, 120),       # batch longer than both intervals
]


@pytest.mark.parametrize("first,last,batch,diag,of,ramp", SCHEDULES)
def test_schedule_matches_reference_loop(first, last, batch, diag, of, ramp):
    u = float(F32(0.05))
    mine = [(b.t, b.end, b.actual, b.u, b.diag_step, b.out_step)
            for b in main_loop_batches(first, last, batch, diag, of, ramp, u)]
    ref = reference_loop(first, last, batch, diag, of, ramp, u)
    assert mine == ref


def test_schedule_last_batch_and_every_crossing():
    # batch 7, diag 100: every multiple of 100 is reported once, at the batch
    # that contains it; the run's final batch is always checked
    got = list(main_loop_batches(1, 1003, 7, 100, 100, 0, 0.05))
    diags = [b.diag_step for b in got if b.diag_step is not None]
    assert diags == list(range(100, 1001, 100))
    assert got[-1].end == 1003 and sum(b.actual for b in got) == 1003
    for b in got:
        if b.diag_step is not None:
            assert b.t <= b.diag_step <= b.end


def test_ramp_velocity_float32_and_shape():
    u = float(F32(0.08))
    ramp = 1500
    vals = [ramp_velocity(u, be, ramp) for be in list(range(8, ramp, 8)) + [ramp]]
    assert all(float(F32(v)) == v for v in vals)          # Float32 values
    assert all(a <= b for a, b in zip(vals, vals[1:]))     # monotone
    assert vals[0] > 0.0 and vals[-1] == u
    assert ramp_velocity(u, ramp + 1, ramp) == u
    assert ramp_velocity(u, 1, 0) == u                     # no ramp
    # the half-way value: cos(pi/2) rounds to a tiny negative, so prog = 0.5f0 * (1 - c)
    half = ramp_velocity(u, 750, ramp)
    x = F32(F32(math.pi) * F32(750)) / F32(ramp)
    assert half == float(F32(u) * (F32(0.5) * (F32(1.0) - F32(math.cos(float(x))))))
    assert abs(half - u / 2) < 1e-8


def test_ramp_matches_julia_where_rounding_is_unambiguous():
    """Julia's cos(::Float32) evaluates a Float64 kernel and rounds once; it
    returns the correctly rounded Float32 of cos(x) unless cos(x) is closer
    to a Float32 rounding midpoint than the kernel error (about 2^-34).
    Where the midpoint is further than 2^-33 away the Float32 result is
    determined, and ramp_velocity must give exactly that value."""
    u = float(F32(0.05))
    checked = 0
    for ramp in (100, 500, 1500, 4000):
        for be in range(1, ramp + 1):
            x = F32(F32(math.pi) * F32(be)) / F32(ramp)
            c = math.cos(float(x))
            f = F32(c)
            up, dn = np.nextafter(f, F32(np.inf)), np.nextafter(f, F32(-np.inf))
            gap = min(abs(c - (float(f) + float(up)) / 2), abs(c - (float(f) + float(dn)) / 2))
            if gap < 2.0 ** -33:
                continue
            want = float(F32(u) * (F32(0.5) * (F32(1.0) - f)))
            assert ramp_velocity(u, be, ramp) == want
            checked += 1
    assert checked > 5000


def _libc():
    return C.CDLL(ctypes.util.find_library("c"))


def _c_format(fmt: str, *args) -> str:
    buf = C.create_string_buffer(4096)
    cargs = [C.c_int(a) if isinstance(a, int) else
             C.c_char_p(a.encode()) if isinstance(a, str) else C.c_double(a) for a in args]
    _libc().snprintf(buf, 4096, fmt.encode(), *cargs)
    return buf.value.decode()


def _force_result(seed=3):
    rng = np.random.default_rng(seed)
    raw = rng.normal(size=9) * 10.0 ** rng.integers(-3, 3, size=9)
    return coefficients(raw, 1.225, 30.0, 0.785, 1.0)


def test_convergence_and_force_rows_match_printf():
    fr = _force_result()
    row = R.convergence_row(1200, 0.0123456789, 41.5, 0.0512, 0.99876, 9677.43, fr)
    ref = _c_format("%d,%.6e,%.6e,%.4f,%.6f,%.1f,%s,%s,%s", 1200, 0.0123456789, 41.5, 0.0512,
                    0.99876, 9677.43, _c_format("%.4f", fr.Cd), _c_format("%.4f", fr.Cl),
                    _c_format("%.4f", fr.Cs))
    assert row == ref
    assert R.convergence_row(100, 1.0, 2.0, 0.05, 1.0, 3.0).endswith(",N/A,N/A,N/A")
    u = float(F32(0.05))
    row = R.force_row(1200, 0.0123456789, fr, u)
    vals = [fr.Fx_p + fr.Fx_v, fr.Fy_p + fr.Fy_v, fr.Fz_p + fr.Fz_v, fr.Fx_p, fr.Fy_p, fr.Fz_p,
            fr.Fx_v, fr.Fy_v, fr.Fz_v, fr.Mx, fr.My, fr.Mz]
    ref = _c_format("%d,%.6e,%.6f," + ",".join(["%.6e"] * 12) + "," + ",".join(["%.6f"] * 6),
                    1200, 0.0123456789, u, *vals, fr.Cd, fr.Cl, fr.Cs, fr.Cmx, fr.Cmy, fr.Cmz)
    assert row == ref
    assert R.FORCE_HEADER.count(",") == row.count(",")
    assert R.CONVERGENCE_HEADER.count(",") == 8


def test_run_records_files(tmp_path):
    rr = R.RunRecords(str(tmp_path), forces=True)
    fr = _force_result(5)
    rr.append(100, 0.1, 1.0, 0.05, 0.999, 1234.5, fr)
    rr.append(200, 0.2, 2.0, 0.05, 0.998, 1234.6, fr)
    conv = (tmp_path / "convergence.csv").read_text().splitlines()
    forces = (tmp_path / "forces.csv").read_text().splitlines()
    assert conv[0] == R.CONVERGENCE_HEADER and len(conv) == 3
    assert forces[0] == R.FORCE_HEADER and len(forces) == 3
    assert forces[2].startswith("200,")


def test_lbmp_layout(tmp_path):
    rng = np.random.default_rng(7)
    n = 5
    tris = rng.normal(size=(n, 3, 3))
    normals = rng.normal(size=(n, 3)).astype(np.float32)
    p = rng.normal(size=n).astype(np.float32)
    shear = rng.normal(size=(3, n)).astype(np.float32)
    names = ["wing", "wing", "flap", "wing", "flap"]
    path = tmp_path / "surface_000100.lbmp"
    R.write_surface_pressure_bin(str(path), tris, normals, p, shear, 1.225, 30.0,
                                 offset=(0.5, 0.25, 0.125), object_names=names)
    raw = path.read_bytes()
    # byte-level reading of the documented layout
    assert raw[:4] == b"LBMP"
    version, nt, nobj = struct.unpack_from("<III", raw, 4)
    assert (version, nt, nobj) == (1, n, 2)
    pos = 16
    got_names = []
    for _ in range(nobj):
        (ln,) = struct.unpack_from("<I", raw, pos)
        got_names.append(raw[pos + 4:pos + 4 + ln].decode())
        pos += 4 + ln
    assert got_names == ["wing", "flap"]
    verts = np.frombuffer(raw, "<f4", 9 * n, pos).reshape(n, 9)
    pos += 36 * n
    want = tris.astype(np.float32) + np.array([0.5, 0.25, 0.125], np.float32)
    assert np.array_equal(verts, want.reshape(n, 9))
    nrm = np.frombuffer(raw, "<f4", 3 * n, pos).reshape(n, 3)
    pos += 12 * n
    assert np.array_equal(nrm, normals)
    pp = np.frombuffer(raw, "<f4", n, pos)
    pos += 4 * n
    sm = np.frombuffer(raw, "<f4", n, pos)
    pos += 4 * n
    cp = np.frombuffer(raw, "<f4", n, pos)
    pos += 4 * n
    ids = np.frombuffer(raw, "<i4", n, pos)
    pos += 4 * n
    assert pos == len(raw)
    assert np.array_equal(pp, p)
    sx, sy, sz = shear
    assert np.array_equal(sm, np.sqrt(sx * sx + sy * sy + sz * sz))
    q = F32(0.5 * 1.225 * 30.0 ** 2)
    assert np.array_equal(cp, p / q)
    assert ids.tolist() == [1, 1, 2, 1, 2]
    back = R.read_surface_pressure_bin(str(path))
    assert back["names"] == ["wing", "flap"] and np.array_equal(back["cp"], cp)


def test_net_forces_csv_inverse_rotation(tmp_path):
    rng = np.random.default_rng(9)
    n = 4
    net = rng.normal(size=(3, n)).astype(np.float32)
    cen = rng.normal(size=(n, 3))
    ucen = rng.normal(size=(n, 3))
    path = tmp_path / "net.csv"
    R.write_net_forces_csv(str(path), net, cen, (1.0, 2.0, 3.0), unrotated_centers=ucen,
                           alpha_deg=10.0, beta_deg=-3.0)
    lines = path.read_text().splitlines()
    assert lines[0] == R.NET_FORCE_HEADER and len(lines) == n + 1
    a, b = math.radians(10.0), math.radians(-3.0)
    # R = Rz(beta) Ry(alpha) applied to a vector, then R^T undoes it
    ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
    rot = np.array([[ca * cb, sb, -sa * cb], [-ca * sb, cb, sa * sb], [sa, 0.0, ca]])
    inv = R.inverse_rotation_f32(10.0, -3.0).astype(np.float64)
    assert np.allclose(inv @ rot, np.eye(3), atol=1e-6)
    for i, line in enumerate(lines[1:]):
        parts = line.split(",")
        assert parts[0] == str(i + 1) and parts[1] == "default"
        f = np.array([float(v) for v in parts[5:8]])
        assert np.allclose(f, inv @ net[:, i].astype(np.float64), rtol=1e-5, atol=1e-6)
        c = np.array([float(v) for v in parts[2:5]])
        assert np.allclose(c, ucen[i].astype(np.float32), rtol=1e-6)
    # without unrotated centres: solver-frame centres + Float32 offset, forces as given
    R.write_net_forces_csv(str(path), net, cen, (1.0, 2.0, 3.0))
    parts = path.read_text().splitlines()[1].split(",")
    assert float(parts[2]) == pytest.approx(float(F32(cen[0, 0]) + F32(1.0)), rel=1e-6)
    assert float(parts[5]) == pytest.approx(float(net[0, 0]), rel=1e-6)
