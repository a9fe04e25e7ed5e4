"""FE load mapping (PREPOST/map_forces_to_nodes.jl), CPU part: the oracle's
restatement against known answers, and the host side of
openludwig_b200.fe_map (CSV reading and writing, grouping by object, the
reference's rules for objects without nodes or forces and for repeated
nodes, the summary) driven by the oracle in place of the device mapper.

Known answers: a force at the centroid of three nodes placed symmetrically
about it splits into three equal thirds; one node takes the whole force;
three nodes in general position keep force and moment equilibrium about the
centroid exactly (to rounding); two nodes give the least-squares minimum-norm
solution (numpy lstsq of the same system)."""
import math

import numpy as np
import pytest

from oracle import femap as ofm
from openludwig_b200 import fe_map as FM


def oracle_mapper(g):
    return ofm.map_grouped(g.node_xyz, g.tri_xyz, g.tri_force, g.node_begin, g.tri_begin)


def test_symmetric_nodes_take_equal_thirds():
    c = np.array([0.3, -0.2, 1.0])
    P = np.array([[math.cos(a), math.sin(a), 0.0] for a in (0.0, 2 * math.pi / 3, 4 * math.pi / 3)])
    F = np.array([1.0, -2.0, 0.5])
    f = ofm.distribute_force(F, c, P + c)
    assert np.allclose(f, np.tile(F / 3, (3, 1)), atol=1e-14)


def test_one_node_takes_everything_and_three_keep_equilibrium():
    F = np.array([0.4, 0.1, -3.0])
    assert np.array_equal(ofm.distribute_force(F, np.zeros(3), [[1.0, 2.0, 3.0]]), F.reshape(1, 3))
    rng = np.random.default_rng(4)
    for _ in range(20):
        c = rng.normal(size=3)
        P = c + rng.normal(size=(3, 3))
        F = rng.normal(size=3)
        f = ofm.distribute_force(F, c, P)
        assert np.allclose(f.sum(axis=0), F, atol=1e-12)
        assert np.allclose(np.cross(P - c, f).sum(axis=0), 0.0, atol=1e-12)


def test_two_nodes_give_the_least_squares_minimum_norm():
    rng = np.random.default_rng(5)
    c = rng.normal(size=3)
    P = c + rng.normal(size=(2, 3))
    F = rng.normal(size=3)
    A = np.zeros((6, 6))
    for i in range(2):
        A[0, 3 * i] = A[1, 3 * i + 1] = A[2, 3 * i + 2] = 1.0
        A[3:, 3 * i:3 * i + 3] = ofm.skew(P[i] - c)
    want = np.linalg.lstsq(A, np.concatenate([F, np.zeros(3)]), rcond=None)[0]
    assert np.allclose(ofm.distribute_force(F, c, P).reshape(-1), want, atol=1e-12)


def _write(tmp_path, nodes, forces):
    npth, fpth = tmp_path / "nodes.csv", tmp_path / "net_forces.csv"
    with open(npth, "w") as f:
        f.write("node_id,object_name,cx,cy,cz\n")
        for n in nodes:
            f.write("%d, %s ,%r,%r,%r\n" % n)
        f.write("\n99,broken\n")                       # malformed: skipped with a warning
    with open(fpth, "w") as f:
        f.write("triangle_id,object_name,cx,cy,cz,Fx,Fy,Fz\n")
        for t in forces:
            f.write("%d,%s,%r,%r,%r,%r,%r,%r\n" % t)
    return npth, fpth


def _case(seed=0):
    rng = np.random.default_rng(seed)
    nodes, forces = [], []
    nid = 1
    for name, nn in (("wing", 40), ("flap", 2), ("tab", 1), ("spar", 5), ("body", 30)):
        for _ in range(nn):
            nodes.append((nid, name, *rng.normal(size=3).tolist()))
            nid += 1
    nodes.append((3, "wing", *nodes[2][2:]))            # repeated (id, object): loads go to the first
    tid = 1
    for name, nt in (("wing", 60), ("flap", 7), ("tab", 3), ("ghost", 4), ("body", 50)):
        # "ghost" has forces but no nodes
        for _ in range(nt):
            forces.append((tid, name, *rng.normal(size=3).tolist(), *rng.normal(size=3).tolist()))
            tid += 1
    return nodes, forces


def test_host_pipeline_with_oracle_mapper(tmp_path):
    nodes, forces = _case()
    npth, fpth = _write(tmp_path, nodes, forces)
    with pytest.warns(UserWarning):
        rc = FM.main([str(npth), str(fpth), str(tmp_path / "out")], mapper=oracle_mapper)
    assert rc == 0
    N = FM.parse_nodes_csv(str(npth))
    assert len(N) == len(nodes) and N[0].object_name == "wing"
    lines = (tmp_path / "out" / "nodal_loads.csv").read_text().splitlines()
    assert lines[0] == FM.NODES_HEADER and len(lines) == len(nodes) + 1
    res = FM.map_forces_to_nodes(N, FM.parse_forces_csv(str(fpth)), oracle_mapper)
    # objects: spar has nodes but no forces (zero), ghost has forces but no nodes (skipped)
    assert set(res.objects) == {"wing", "flap", "tab", "body"}
    spar = [i for i, n in enumerate(N) if n.object_name == "spar"]
    assert not res.has_load[spar].any() and np.all(res.nodal[spar] == 0.0)
    # the repeated node's own row stays zero, its loads sit on the first occurrence
    assert np.all(res.nodal[-1] == 0.0) and res.has_load[2]
    # equilibrium: body (>= 3 nodes in general position) keeps force and
    # moment; tab (one node: the moment of the offset is lost) keeps the
    # force; flap (two nodes) and wing (whose repeated node sits where its
    # first copy is, so some triangles see two distinct positions only) are
    # least-squares compromises between the six equations
    r = res.objects["body"]
    assert np.allclose(r["F_nod"], r["F_tri"], atol=1e-10)
    assert np.allclose(r["M_nod"], r["M_tri"], atol=1e-10)
    assert np.allclose(res.objects["tab"]["F_nod"], res.objects["tab"]["F_tri"], atol=1e-10)
    md = (tmp_path / "out" / "Nodal_loads_summary.md").read_text()
    assert "### Object: `wing`" in md and "## Global Validation (All Objects)" in md
    # the nodal file carries the mapped loads in file order
    row = lines[1].split(",")
    assert [float(v) for v in row[5:8]] == pytest.approx(res.nodal[0].tolist(), rel=1e-6, abs=1e-12)
