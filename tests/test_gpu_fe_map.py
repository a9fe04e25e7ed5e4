"""FE load mapping on the GPU (ol_fe_map_forces) against the oracle's
restatement of map_forces_to_nodes.jl (oracle/femap.py).

* a seeded multi-object case: objects with one node, two nodes, three
  collinear nodes (rank-deficient systems: the pseudo-inverse cut-off
  decides), hundreds of nodes, and none: the chosen nodes equal, the
  per-triangle forces and the nodal sums within 1e-9 of the force scale, no
  SVD at its sweep limit, and two runs bitwise equal (fixed-point sums);
* the whole chain on a flow: net per-triangle forces of a sphere after 40
  steps, written as the reference's net_forces CSV, mapped onto 200 nodes
  by `python -m openludwig_b200.fe_map`'s main(): global force and moment
  kept to 1e-6 of their size (the summary's PASS line).
"""
import numpy as np
import pytest

from helpers import small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import fe_map as FM  # noqa: E402
from openludwig_b200 import records as R  # noqa: E402
from openludwig_b200 import solver as S  # noqa: E402
from oracle import femap as ofm  # noqa: E402


def _grouped(seed=1):
    rng = np.random.default_rng(seed)
    nodes, forces = [], []
    specs = [("many", rng.normal(size=(300, 3)), 1500), ("one", rng.normal(size=(1, 3)), 40),
             ("two", rng.normal(size=(2, 3)), 40),
             ("line", np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [3.0, 0.0, 0.0]]), 40),
             ("none", np.zeros((0, 3)), 20), ("idle", rng.normal(size=(5, 3)), 0)]
    nid = tid = 1
    for name, P, nt in specs:
        for p in P:
            nodes.append(FM.Node(nid, name, *p.tolist()))
            nid += 1
        for _ in range(nt):
            c = rng.normal(size=3) * 1.5
            forces.append(FM.TriForce(tid, name, *c.tolist(), *(rng.normal(size=3) * 10).tolist()))
            tid += 1
    with pytest.warns(UserWarning):
        g = FM.group(nodes, forces)
    return nodes, forces, g


def test_device_mapping_matches_oracle():
    nodes, forces, g = _grouped()
    tn, tf, nod, unconv = FM.device_map(g)
    otn, otf, onod, _ = ofm.map_grouped(g.node_xyz, g.tri_xyz, g.tri_force, g.node_begin,
                                        g.tri_begin)
    assert unconv == 0
    assert np.array_equal(tn, otn)
    scale = float(np.abs(g.tri_force).max())
    assert np.abs(tf - otf).max() <= 1e-9 * scale
    assert np.abs(nod - onod).max() <= 1e-9 * scale
    print(f"\nFE map vs oracle: per-triangle {np.abs(tf - otf).max() / scale:.2e}, "
          f"nodal {np.abs(nod - onod).max() / scale:.2e} of the force scale")
    again = FM.device_map(g)
    assert np.array_equal(again[2], nod) and np.array_equal(again[1], tf)


def test_net_forces_of_a_flow_to_nodes(tmp_path):
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    c.ramp_steps = 0
    c.net_force_export = True
    sim = S.Simulation(c, mesh, p, hosts, torch.device("cuda:0"))
    sim.run(40, diag_freq=40)
    net = S.compute_net_aerodynamics(sim.levels[-1], sim.dmesh, p, c)
    fpth = tmp_path / "net_forces_000040.csv"
    R.write_net_forces_csv(str(fpth), np.stack(net), mesh.centers, p.mesh_offset)
    rng = np.random.default_rng(2)
    d = rng.normal(size=(200, 3))
    d = 0.45 * d / np.linalg.norm(d, axis=1, keepdims=True)
    ctr = np.asarray(mesh.centers).mean(axis=0) + np.asarray(p.mesh_offset)
    npth = tmp_path / "nodes.csv"
    with open(npth, "w") as f:
        f.write("node_id,object_name,cx,cy,cz\n")
        for i, q in enumerate(d + ctr):
            f.write("%d,default,%.9e,%.9e,%.9e\n" % (i + 1, *q))
    assert FM.main([str(npth), str(fpth), str(tmp_path / "fe")]) == 0
    nodes, forces = FM.parse_nodes_csv(str(npth)), FM.parse_forces_csv(str(fpth))
    res = FM.map_forces_to_nodes(nodes, forces)
    r = res.global_result
    fs, ms = np.abs(r["F_tri"]).max(), np.abs(r["M_tri"]).max()
    assert fs > 0 and np.abs(r["F_nod"] - r["F_tri"]).max() <= 1e-6 * fs
    assert np.abs(r["M_nod"] - r["M_tri"]).max() <= 1e-6 * ms
    md = (tmp_path / "fe" / "Nodal_loads_summary.md").read_text()
    assert "Global Validation" in md
    lines = (tmp_path / "fe" / "nodal_loads.csv").read_text().splitlines()
    assert len(lines) == 201
