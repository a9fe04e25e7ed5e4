"""Host preprocessing parity: the product's numpy domain build against the
CPU oracle, bit for bit (block sets and order, neighbour tables, block
pointers, SAT voxels, flood fill, sponge, wall distance, Float16 q-map,
triangle ids, boundary-cell set compared as sorted sets because the
reference's cell-list order is thread-dependent, bouzidi_setup.jl:95-143)."""
import numpy as np
import pytest

from openludwig_b200 import domain, geometry as geo, scaling, workloads
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build_oracle():
    orc.build()


def _compare_level(h, tris, dx, offset, dims, prev=None, prev_bs=0.0, margin=2, sponge_args=None):
    oc = orc.level_blocks(h.level_id, tris, dx, offset, dims, prev, prev_bs, None, margin)
    assert np.array_equal(oc, h.coords)
    assert np.array_equal(orc.neighbor_table(oc, dims), h.neighbor_table)
    ov = orc.voxelize(oc, tris, dx, offset)
    assert np.array_equal(ov, domain.voxelize_blocks(h.coords, tris, dx, offset))
    of = orc.flood_fill(oc, dims, ov)
    assert np.array_equal(of, h.obstacle)
    if sponge_args is not None:
        assert np.array_equal(orc.sponge(oc, dx, *sponge_args), h.sponge)
    ow = orc.wall_dist(oc, of, dx)
    assert np.array_equal(ow, domain.compute_wall_distances(h.coords, h.neighbor_table, h.obstacle, dx))
    if h.bouzidi:
        q, tri, cells = orc.bouzidi_qmap(oc, tris, dx, offset)
        assert np.array_equal(q, h.q_map)
        assert np.array_equal(tri, h.tri_map)
        pc = np.stack([h.cell_block, h.cell_x, h.cell_y, h.cell_z], 1).astype(np.int32)
        assert np.array_equal(np.unique(pc, axis=0), np.unique(cells, axis=0))
    return oc


def test_sphere_single_level_matches_oracle():
    c, mesh = workloads.sphere_1lvl(8)
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    assert (p.nx_coarse, p.ny_coarse, p.nz_coarse) == (64, 32, 32)
    h = hosts[0]
    assert h.n_blocks == 128 and h.bouzidi and h.n_boundary > 0
    _compare_level(h, mesh.triangles, p.dx_coarse, p.mesh_offset, (p.bx_max, p.by_max, p.bz_max),
                   sponge_args=(p.domain_size, c.sponge_thickness, False))


def test_rotated_cube_three_levels_matches_oracle():
    """Rotated cube (alpha = 10 deg) with three 2:1 levels, wall model on."""
    c, mesh = workloads.cube_3lvl()
    c.surface_resolution = 16          # smaller copy of the 3-level workload
    c.domain_upstream, c.domain_downstream = 1.5, 2.5
    c.domain_lateral = c.domain_height = 1.5
    c.min_coarse_blocks = 1
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    assert p.num_levels == 3
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    prev = None
    for i, h in enumerate(hosts):
        scale = 2 ** i
        dims = (p.bx_max * scale, p.by_max * scale, p.bz_max * scale)
        prev_bs = 8 * (p.dx_coarse / 2 ** (i - 1)) if i > 0 else 0.0
        prev = _compare_level(h, mesh.triangles, p.dx_coarse / scale, p.mesh_offset, dims, prev,
                              prev_bs, sponge_args=(p.domain_size, c.sponge_thickness, False))
        assert (h.wall_dist < 100).any()
    # every fine block has its parent (domain.jl:229-243)
    for a, b in zip(hosts[:-1], hosts[1:]):
        par = set(map(tuple, a.coords.tolist()))
        assert all(((x + 1) // 2, (y + 1) // 2, (z + 1) // 2) in par for x, y, z in b.coords.tolist())


def test_cube_3lvl_full_size_matches_oracle():
    """The benchmark workload's own domain (cube side 64 finest cells, three
    levels of 2000 / 1728 / 4608 blocks): every level's block set and order,
    neighbour table, voxels, flood fill, sponge, wall distance and the finest
    level's Bouzidi q-map, triangle ids and boundary cells, bit for bit."""
    c, mesh = workloads.cube_3lvl()
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    assert [h.n_blocks for h in hosts] == [2000, 1728, 4608]
    assert (p.nx_coarse, p.ny_coarse, p.nz_coarse) == (160, 80, 80)
    prev = None
    for i, h in enumerate(hosts):
        scale = 2 ** i
        dims = (p.bx_max * scale, p.by_max * scale, p.bz_max * scale)
        prev_bs = 8 * (p.dx_coarse / 2 ** (i - 1)) if i > 0 else 0.0
        prev = _compare_level(h, mesh.triangles, p.dx_coarse / scale, p.mesh_offset, dims, prev,
                              prev_bs, sponge_args=(p.domain_size, c.sponge_thickness, False))
    assert hosts[-1].bouzidi and hosts[-1].n_boundary > 0


def test_wing_voxelization_and_qmap_match_oracle():
    """Thin closed NACA0012 wing (coarse panels) on one level."""
    mesh = geo.rotate_mesh(geo.naca0012_wing(1.0, 1.0, n_chord=24, n_span=4), 6.0, -3.0)
    c = workloads.base_config(surface_resolution=12, num_levels_config=1, domain_upstream=1.0,
                              domain_downstream=1.5, domain_lateral=0.6, domain_height=0.6)
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    hosts = domain.setup_multilevel_domain(c, mesh, p)
    _compare_level(hosts[0], mesh.triangles, p.dx_coarse, p.mesh_offset,
                   (p.bx_max, p.by_max, p.bz_max))


def test_flood_fill_closes_body_interior():
    c, mesh = workloads.sphere_1lvl(8)
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    h = domain.setup_multilevel_domain(c, mesh, p, with_bouzidi=False)[0]
    shell = domain.voxelize_blocks(h.coords, mesh.triangles, p.dx_coarse, p.mesh_offset)
    assert h.obstacle.sum() > shell.sum()       # interior filled
    # the sphere centre cell (40/2, 32/2, 32/2 at resolution 8) is solid
    gx, gy, gz = 20, 16, 16
    b = np.nonzero((h.coords == [(gx - 1) // 8 + 1, (gy - 1) // 8 + 1, (gz - 1) // 8 + 1]).all(1))[0][0]
    cell = (gx - 1) % 8 + 8 * ((gy - 1) % 8) + 64 * ((gz - 1) % 8)
    assert h.obstacle[b * 512 + cell] == 1


def test_empty_and_edge_inputs():
    # a triangle outside the domain activates no block on a fine level
    tris = np.array([[[100.0, 100, 100], [101, 100, 100], [100, 101, 100]]])
    assert domain.active_blocks_for_level(tris, 0.1, (0, 0, 0), (4, 4, 4)) == set()
    # neighbour table of a single block has only itself
    t = domain.build_neighbor_table(np.array([[1, 1, 1]], dtype=np.int32), (1, 1, 1))
    assert t.tolist() == [0] * 13 + [1] + [0] * 13
    assert np.array_equal(orc.neighbor_table(np.array([[1, 1, 1]], np.int32), (1, 1, 1)), t)
    # empty voxelization / q-map
    c = np.array([[1, 1, 1]], dtype=np.int32)
    assert domain.voxelize_blocks(c, tris, 0.1, (0, 0, 0)).sum() == 0
    q, tri, cells = domain.compute_bouzidi_qmap(c, tris, 0.1, (0, 0, 0))
    assert cells.shape == (0, 4) and q.sum() == 0
