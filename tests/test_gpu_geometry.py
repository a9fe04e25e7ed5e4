"""Device voxelisation and Bouzidi q-map (ol_voxelize / ol_bouzidi_qmap) give
the same bits as the host build (openludwig_b200/domain.py), which itself
matches the C++ oracle bit for bit (test_domain_parity.py)."""
import numpy as np
import pytest
import torch

from openludwig_b200 import domain as D
from openludwig_b200 import geometry as G
from openludwig_b200 import scaling, workloads

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)


def _level_inputs(cfg, mesh, level=1):
    p = scaling.compute_domain_from_mesh(cfg, mesh.min_bounds, mesh.max_bounds)
    hosts = D.setup_multilevel_domain(cfg, mesh, p, with_bouzidi=False)
    h = hosts[level - 1]
    return mesh.triangles, h.coords, p.dx_coarse / 2 ** (level - 1), p.mesh_offset


CASES = {
    "sphere": lambda: workloads.sphere_1lvl(8),
    "rotated_cube_l3": lambda: workloads.cube_3lvl(),
    "wing": lambda: _small_wing(),
}


def _small_wing():
    """A coarse, rotated NACA0012 wing (thin trailing edge, tip caps)."""
    cfg, _ = workloads.mix_case_config(workloads.MixCase("wing", 16, 1, 1e4, 6.0, 2.0))
    mesh = G.rotate_mesh(G.naca0012_wing(chord=1.0, span=1.0, n_chord=40, n_span=6), 6.0, 2.0)
    return cfg, mesh


@pytest.mark.parametrize("name", list(CASES))
def test_device_voxelize_and_qmap_bit_exact(name):
    cfg, mesh = CASES[name]()
    level = 3 if name == "rotated_cube_l3" else 1
    tris, coords, dx, offset = _level_inputs(cfg, mesh, level)
    dg = D.DeviceGeometry(tris, 0)
    # voxelisation (margin 2 dx)
    bm = D.block_triangle_map(tris, coords, dx, offset, dx * 2)
    host = D.voxelize_blocks(coords, tris, dx, offset)
    dev = dg.voxelize(coords, dx, offset, bm)
    assert host.sum() > 0
    assert np.array_equal(host, dev)
    # Bouzidi q-map (margin 2.5 dx)
    bm = D.block_triangle_map(tris, coords, dx, offset, dx * 2.5)
    q_h, t_h, c_h = D.compute_bouzidi_qmap(coords, tris, dx, offset)
    q_d, t_d, c_d = dg.qmap(coords, dx, offset, bm)
    assert c_h.shape[0] > 0
    assert np.array_equal(q_h, q_d)
    assert np.array_equal(t_h, t_d)
    assert np.array_equal(c_h, c_d)


def test_device_domain_build_equals_host():
    cfg, mesh = workloads.sphere_1lvl(8)
    p = scaling.compute_domain_from_mesh(cfg, mesh.min_bounds, mesh.max_bounds)
    a = D.setup_multilevel_domain(cfg, mesh, p)
    b = D.setup_multilevel_domain(cfg, mesh, p, device=0)
    for la, lb in zip(a, b):
        for k in ("obstacle", "sponge", "wall_dist", "q_map", "tri_map", "cell_block", "cell_x"):
            va, vb = getattr(la, k), getattr(lb, k)
            assert (va is None and vb is None) or np.array_equal(va, vb), k


def test_empty_level_and_no_triangles():
    mesh = G.cube(1.0)
    tris = mesh.triangles
    dg = D.DeviceGeometry(tris, 0)
    coords = np.array([[1, 1, 1], [2, 1, 1]], dtype=np.int32)
    # no triangle near these blocks: nothing solid, no Bouzidi cell
    bm = [[], []]
    assert dg.voxelize(coords, 0.1, (50.0, 50.0, 50.0), bm).sum() == 0
    q, t, c = dg.qmap(coords, 0.1, (50.0, 50.0, 50.0), bm)
    assert q.sum() == 0 and t.sum() == 0 and c.shape == (0, 4)
