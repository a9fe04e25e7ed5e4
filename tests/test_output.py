"""Merged flow output (io_vtk.jl:6-129): exported-block selection, the
device gather against the oracle restatement (bit-exact: copies, NaN / Inf
to 0, Float32 magnitude and point coordinates), and the .vtu writer."""
import re

import numpy as np
import pytest

from helpers import small_sphere_case
from oracle import oracle as orc
from openludwig_b200 import output as OUT


def _host_levels(hosts, t_step, rng=None):
    """Host stand-ins of the device levels, with seeded fields."""
    rng = rng or np.random.default_rng(3)
    out = []
    for h in hosts:
        S = 512 * h.n_blocks
        out.append(dict(coords=h.coords, rho=rng.uniform(0.9, 1.1, S).astype(np.float32),
                        vel=rng.normal(0, 0.05, 3 * S).astype(np.float32),
                        vel_temp=rng.normal(0, 0.05, 3 * S).astype(np.float32),
                        obstacle=h.obstacle, temperature=None, dx=h.dx, level_id=h.level_id))
    return out


def test_export_lists_match_the_oracle_selection():
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2)
    lists = OUT.export_block_lists(hosts)
    ref = orc.merged_output(_host_levels(hosts, 1), 1)
    for lvl, lst in enumerate(lists, start=1):
        assert np.count_nonzero(ref["level"] == lvl) == 512 * len(lst)
    assert len(lists[-1]) == hosts[-1].n_blocks        # the finest level exports everything
    assert len(lists[0]) < hosts[0].n_blocks            # covered coarse blocks are skipped


def test_vtu_writer_round_trip(tmp_path):
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    arrays = orc.merged_output(_host_levels(hosts, 2), 2)
    path = tmp_path / "flow_000002.vtu"
    OUT.write_vtu(str(path), arrays)
    raw = path.read_bytes()
    head, _, body = raw.partition(b'<AppendedData encoding="raw">\n_')
    xml = head.decode()
    n_blocks = hosts[0].n_blocks
    assert f'NumberOfPoints="{729 * n_blocks}"' in xml and f'NumberOfCells="{512 * n_blocks}"' in xml
    offs = {m.group(1): int(m.group(2))
            for m in re.finditer(r'Name="(\w+)"[^>]*offset="(\d+)"', xml)}
    pts_off = int(re.search(r'<Points>\s*<DataArray[^>]*offset="(\d+)"', xml).group(1))

    def block(off, dtype):
        n = int(np.frombuffer(body[off:off + 8], dtype="<u8")[0])
        return np.frombuffer(body[off + 8:off + 8 + n], dtype=dtype)
    assert np.array_equal(block(pts_off, np.float32).reshape(-1, 3), arrays["points"])
    assert np.array_equal(block(offs["Density"], np.float32), arrays["rho"])
    assert np.array_equal(block(offs["Velocity"], np.float32).reshape(-1, 3), arrays["vel"])
    assert np.array_equal(block(offs["Level"], np.int32), arrays["level"])
    conn = block(offs["connectivity"], np.int64).reshape(-1, 8)
    assert conn.max() == 729 * n_blocks - 1
    # cell 0 of block 0 spans points 0, 1, 9, 10, 81, 82, 90, 91
    assert conn[0].tolist() == [0, 1, 9, 10, 81, 82, 90, 91]
    assert set(block(offs["types"], np.uint8).tolist()) == {11}


@pytest.mark.gpu
def test_device_pack_matches_oracle():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():  # pragma: no cover
        pytest.skip("needs a CUDA device")
    from openludwig_b200 import solver as S
    c, mesh, p, hosts = small_sphere_case(resolution=16, levels=2, c_wale=np.float32(0.5))
    c.ramp_steps = 0
    dev = torch.device("cuda:0")
    sim = S.Simulation(c, mesh, p, hosts, dev)
    sim.run(6, diag_freq=6)
    lv = sim.levels
    # planted non-finite values, which the output replaces by 0
    lv[0].rho[5] = float("nan")
    lv[1].vel_temp[7] = float("inf")
    torch.cuda.synchronize()
    mo = OUT.MergedOutput(lv)
    for t_step in (6, 7):
        got = mo.pack(t_step).wait()
        ref = orc.merged_output([dict(coords=h.coords, rho=L.rho.cpu().numpy(),
                                      vel=L.vel.cpu().numpy(), vel_temp=L.vel_temp.cpu().numpy(),
                                      obstacle=L.obstacle.cpu().numpy(), temperature=None,
                                      dx=h.dx, level_id=h.level_id)
                                 for h, L in zip(hosts, lv)], t_step)
        for k in ("points", "rho", "vel", "vel_mag", "obstacle", "level"):
            assert np.array_equal(got[k].reshape(ref[k].shape), ref[k]), k
        assert all(np.isfinite(got[k]).all() for k in ("rho", "vel", "vel_mag"))


@pytest.mark.gpu
def test_simulation_writes_merged_output(tmp_path):
    """Simulation.run(output_dir=...) writes flow_%06d.vtu at every
    output_freq step (main.jl:259-263); the file holds the packed state."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():  # pragma: no cover
        pytest.skip("needs a CUDA device")
    from openludwig_b200 import solver as S
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    c.ramp_steps = 0
    c.output_freq = 4
    c.async_depth = 4
    sim = S.Simulation(c, mesh, p, hosts, torch.device("cuda:0"))
    sim.run(8, diag_freq=8, output_dir=str(tmp_path))
    names = sorted(f.name for f in tmp_path.iterdir())
    assert names == ["convergence.csv", "flow_000004.vtu", "flow_000008.vtu", "forces.csv",
                     "surface_000004.lbmp", "surface_000008.lbmp"]
    raw = (tmp_path / "flow_000008.vtu").read_bytes()
    assert f'NumberOfCells="{512 * hosts[0].n_blocks}"'.encode() in raw
    # output step 4 is not a diagnostics multiple: its force sample is
    # accumulated too (main.jl:267-275); step 8 is the diagnostics sample
    assert sim.n_avg == 2 and len(sim.history) == 1
    from openludwig_b200 import records as R
    conv = (tmp_path / "convergence.csv").read_text().splitlines()
    forces = (tmp_path / "forces.csv").read_text().splitlines()
    assert conv[0] == R.CONVERGENCE_HEADER and len(conv) == 2 and conv[1].startswith("8,")
    assert forces[0] == R.FORCE_HEADER and len(forces) == 2
    fr, _, maps = sim.forces(maps=True)
    assert forces[1] == R.force_row(8, 8 * p.time_scale, fr, sim.history[0]["u"])
    got = R.read_surface_pressure_bin(str(tmp_path / "surface_000008.lbmp"))
    m = maps.cpu().numpy()
    assert got["pressure"].shape == (mesh.n,) and np.array_equal(got["pressure"], m[0])
    assert np.array_equal(got["shear"], np.sqrt(m[1] * m[1] + m[2] * m[2] + m[3] * m[3]))
