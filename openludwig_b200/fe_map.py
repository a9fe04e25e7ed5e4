"""Net triangle forces to structural FE nodes (PREPOST/map_forces_to_nodes.jl).

Same inputs, outputs and rules as the reference script:

    python -m openludwig_b200.fe_map nodes.csv net_forces.csv [output_dir]

  nodes.csv       node_id, object_name, cx, cy, cz
  net_forces.csv  triangle_id, object_name, cx, cy, cz, Fx, Fy, Fz
                  (written by records.write_net_forces_csv)
  output_dir      default: the folder of net_forces.csv; receives
                  nodal_loads.csv and Nodal_loads_summary.md

Every triangle force goes to the 3 nearest nodes of its object (fewer when
the object has fewer) as the minimum-norm solution of force and moment
equilibrium about the triangle centroid; the per-triangle work (search and
pseudo-inverse) runs on the GPU (ol_fe_map_forces), one thread per
triangle.  Objects with forces but no nodes are skipped with a warning, nodes
of objects without forces get zero load, and a node that appears twice with
the same id and object receives its copies' loads at its first occurrence,
as in the reference (map_forces_to_nodes.jl:462-470).
"""
from __future__ import annotations

import ctypes as C
import dataclasses as dc
import os
import sys
import time
import warnings

import numpy as np

NODES_HEADER = "node_id,object_name,cx,cy,cz,Fx,Fy,Fz"


@dc.dataclass
class Node:
    node_id: int
    object_name: str
    cx: float
    cy: float
    cz: float


@dc.dataclass
class TriForce:
    triangle_id: int
    object_name: str
    cx: float
    cy: float
    cz: float
    Fx: float
    Fy: float
    Fz: float


def _parse(path: str, ncols: int, kind: str, make):
    """map_forces_to_nodes.jl:41-109: header skipped, blank lines skipped,
    lines with too few columns skipped with a warning, fields stripped."""
    out = []
    with open(path) as f:
        f.readline()
        for line_num, line in enumerate(f, start=2):
            s = line.strip()
            if not s:
                continue
            parts = [p.strip() for p in s.split(",")]
            if len(parts) < ncols:
                warnings.warn(f"[MapForces] Skipping malformed line {line_num} in {kind} file "
                              f"({len(parts)} columns)")
                continue
            out.append(make(parts))
    return out


def parse_nodes_csv(path: str) -> list[Node]:
    return _parse(path, 5, "nodes", lambda p: Node(int(p[0]), p[1], float(p[2]), float(p[3]),
                                                   float(p[4])))


def parse_forces_csv(path: str) -> list[TriForce]:
    return _parse(path, 8, "forces", lambda p: TriForce(int(p[0]), p[1], *(float(v) for v in p[2:8])))


def group_by_object(items) -> dict:
    groups: dict = {}
    for it in items:
        groups.setdefault(it.object_name, []).append(it)
    return groups


def compute_resultant(positions: np.ndarray, forces: np.ndarray):
    """map_forces_to_nodes.jl:244-264: total force and moment about the origin,
    summed in order."""
    F = [0.0, 0.0, 0.0]
    M = [0.0, 0.0, 0.0]
    for (px, py, pz), (fx, fy, fz) in zip(positions.tolist(), forces.tolist()):
        F[0] += fx
        F[1] += fy
        F[2] += fz
        M[0] += py * fz - pz * fy
        M[1] += pz * fx - px * fz
        M[2] += px * fy - py * fx
    return np.array(F), np.array(M)


@dc.dataclass
class Grouped:
    """Nodes and triangles regrouped by object (objects in sorted order, items
    in file order within an object), the layout ol_fe_map_forces takes."""
    objects: list
    node_xyz: np.ndarray      # [N, 3]
    tri_xyz: np.ndarray       # [T, 3]
    tri_force: np.ndarray     # [T, 3]
    node_begin: np.ndarray    # [n_obj + 1] int32
    tri_begin: np.ndarray     # [n_obj + 1] int32
    node_global: np.ndarray   # [N] index into the file's node list (first (id, object) match)


def group(nodes: list[Node], forces: list[TriForce]) -> Grouped:
    ng, fg = group_by_object(nodes), group_by_object(forces)
    objects = sorted(set(ng) | set(fg))
    first = {}
    for gi, nd in enumerate(nodes):
        first.setdefault((nd.node_id, nd.object_name), gi)
    nx, nglob, tx, tf = [], [], [], []
    nb, tb = [0], [0]
    for o in objects:
        on = ng.get(o, [])
        of = fg.get(o, [])
        if of and not on:
            warnings.warn(f"[MapForces] Object '{o}' has {len(of)} forces but NO nodes — skipping")
        for nd in on:
            nx.append((nd.cx, nd.cy, nd.cz))
            nglob.append(first[(nd.node_id, nd.object_name)])
        for t in of:
            tx.append((t.cx, t.cy, t.cz))
            tf.append((t.Fx, t.Fy, t.Fz))
        nb.append(len(nx))
        tb.append(len(tx))
    return Grouped(objects, np.array(nx, np.float64).reshape(-1, 3),
                   np.array(tx, np.float64).reshape(-1, 3), np.array(tf, np.float64).reshape(-1, 3),
                   np.array(nb, np.int32), np.array(tb, np.int32), np.array(nglob, np.int64))


def device_map(g: Grouped, device=None):
    """ol_fe_map_forces on the GPU: returns (tri_nodes [T, 3] int32, -1 unused;
    tri_node_force [T, 3, 3]; nodal [N, 3]; unconverged count)."""
    import torch

    from . import _native as NV
    dev = device or torch.device("cuda", torch.cuda.current_device())
    N, T = g.node_xyz.shape[0], g.tri_xyz.shape[0]

    def planes(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).to(dev)

    nxyz, txyz, tfor = planes(g.node_xyz), planes(g.tri_xyz), planes(g.tri_force)
    nb = torch.from_numpy(g.node_begin).to(dev)
    tb = torch.from_numpy(g.tri_begin).to(dev)
    tri_nodes = torch.empty(3 * max(T, 1), dtype=torch.int32, device=dev)
    tri_f = torch.empty(9 * max(T, 1), dtype=torch.float64, device=dev)
    nodal = torch.empty(3 * max(N, 1), dtype=torch.float64, device=dev)
    scratch = torch.empty(int(NV.lib().ol_fe_map_scratch_bytes(NV.i32(N))), dtype=torch.uint8,
                          device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    v = NV.FeMapView(p(nxyz), p(txyz), p(tfor), p(nb), p(tb), N, T, len(g.objects), p(tri_nodes),
                     p(tri_f), p(nodal), p(scratch))
    unconv = NV.i32(0)
    NV.call("ol_fe_map_forces", C.byref(v), C.byref(unconv),
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    tn = tri_nodes.cpu().numpy()[:3 * T].reshape(3, T).T.copy()
    tfv = tri_f.cpu().numpy()[:9 * T].reshape(3, 3, T).transpose(2, 0, 1).copy()
    nod = nodal.cpu().numpy()[:3 * N].reshape(3, N).T.copy()
    return tn, tfv, nod, int(unconv.value)


@dc.dataclass
class MapResult:
    nodal: np.ndarray          # [n_nodes, 3] in file order (zero where no load)
    has_load: np.ndarray       # [n_nodes] bool: the node received a contribution
    objects: dict              # name -> dict(n_nodes, n_forces, F_tri, M_tri, F_nod, M_nod)
    global_result: dict        # F_tri, M_tri, F_nod, M_nod
    unconverged: int


def map_forces_to_nodes(nodes: list[Node], forces: list[TriForce], mapper=None) -> MapResult:
    """map_forces_to_nodes.jl:381-560 without the file handling.  `mapper`
    maps a Grouped layout (default: device_map on the GPU)."""
    if not nodes or not forces:
        raise ValueError("[MapForces] Empty input data. Cannot proceed.")
    g = group(nodes, forces)
    tn, _, nod, unconv = (mapper or device_map)(g)
    n = len(nodes)
    nodal = np.zeros((n, 3))
    has = np.zeros(n, bool)
    used = np.zeros(g.node_xyz.shape[0], bool)
    used[tn[tn >= 0]] = True
    for li in range(g.node_xyz.shape[0]):       # grouped -> file order (duplicates add up)
        if used[li]:
            gi = g.node_global[li]
            nodal[gi] += nod[li]
            has[gi] = True
    ng, fg = group_by_object(nodes), group_by_object(forces)
    first = {}
    for gi, nd in enumerate(nodes):
        first.setdefault((nd.node_id, nd.object_name), gi)
    objects = {}
    for o in g.objects:
        of, on = fg.get(o), ng.get(o)
        if not of or not on:
            continue
        tp = np.array([(t.cx, t.cy, t.cz) for t in of])
        tf = np.array([(t.Fx, t.Fy, t.Fz) for t in of])
        F_tri, M_tri = compute_resultant(tp, tf)
        npos = np.array([(nd.cx, nd.cy, nd.cz) for nd in on])
        nfor = np.array([nodal[first[(nd.node_id, nd.object_name)]] for nd in on])
        F_nod, M_nod = compute_resultant(npos, nfor)
        objects[o] = dict(n_nodes=len(on), n_forces=len(of), F_tri=F_tri, M_tri=M_tri,
                          F_nod=F_nod, M_nod=M_nod)
    allp = np.array([(t.cx, t.cy, t.cz) for t in forces])
    allf = np.array([(t.Fx, t.Fy, t.Fz) for t in forces])
    F_tri, M_tri = compute_resultant(allp, allf)
    idx = np.nonzero(has)[0]
    npos = np.array([(nodes[i].cx, nodes[i].cy, nodes[i].cz) for i in idx]).reshape(-1, 3)
    F_nod, M_nod = compute_resultant(npos, nodal[idx].reshape(-1, 3))
    return MapResult(nodal, has, objects, dict(F_tri=F_tri, M_tri=M_tri, F_nod=F_nod, M_nod=M_nod),
                     unconv)


def write_nodal_loads_csv(path: str, nodes: list[Node], nodal: np.ndarray) -> None:
    """map_forces_to_nodes.jl:276-287."""
    with open(path, "w") as f:
        f.write(NODES_HEADER + "\n")
        for nd, F in zip(nodes, nodal.tolist()):
            f.write("%d,%s,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e\n" % (
                nd.node_id, nd.object_name, nd.cx, nd.cy, nd.cz, F[0], F[1], F[2]))


def _table(f, r) -> None:
    f.write("| Quantity | Triangle Forces | Nodal Loads | Difference |\n")
    f.write("|----------|---------------:|------------:|-----------:|\n")
    for name, key, i in (("Fx [N]  ", "F", 0), ("Fy [N]  ", "F", 1), ("Fz [N]  ", "F", 2),
                         ("Mx [N.m]", "M", 0), ("My [N.m]", "M", 1), ("Mz [N.m]", "M", 2)):
        a, b = r[key + "_tri"][i], r[key + "_nod"][i]
        f.write("| %s | %+.6e | %+.6e | %+.6e |\n" % (name, a, b, a - b))


def write_summary_md(path: str, res: MapResult, n_nodes: int, n_forces: int,
                     elapsed: float) -> None:
    """map_forces_to_nodes.jl:297-370."""
    with open(path, "w") as f:
        f.write("# Nodal Loads Mapping Summary\n\n")
        f.write("**Generated:** %s\n" % time.strftime("%Y-%m-%d %H:%M:%S"))
        f.write("**Elapsed time:** %.3f s\n" % elapsed)
        f.write("**Total nodes:** %d\n" % n_nodes)
        f.write("**Total triangle forces:** %d\n\n" % n_forces)
        f.write("## Per-Object Validation\n\n")
        for o in sorted(res.objects):
            r = res.objects[o]
            f.write("### Object: `%s`\n\n" % o)
            f.write("- **Nodes:** %d\n" % r["n_nodes"])
            f.write("- **Triangle forces:** %d\n\n" % r["n_forces"])
            _table(f, r)
            f.write("\n")
        f.write("## Global Validation (All Objects)\n\n")
        r = res.global_result
        _table(f, r)
        f.write("\n")
        dF = float(np.max(np.abs(r["F_tri"] - r["F_nod"])))
        dM = float(np.max(np.abs(r["M_tri"] - r["M_nod"])))
        f.write("**Max force difference:**  %.2e N\n" % dF)
        f.write("**Max moment difference:** %.2e N.m\n\n" % dM)
        if dF < 1e-6 and dM < 1e-6:
            f.write("> **PASS** - Force and moment equilibrium preserved within machine precision.\n")
        else:
            f.write("> **WARNING** - Differences exceed expected machine precision. Check input data.\n")


def main(argv: list[str] | None = None, mapper=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 2:
        print(__doc__)
        return 2
    t0 = time.time()
    nodes_path, forces_path = argv[0], argv[1]
    out = argv[2] if len(argv) >= 3 else (os.path.dirname(forces_path) or ".")
    for pth, kind in ((nodes_path, "Nodes"), (forces_path, "Forces")):
        if not os.path.isfile(pth):
            raise FileNotFoundError(f"[MapForces] {kind} file not found: {pth}")
    nodes, forces = parse_nodes_csv(nodes_path), parse_forces_csv(forces_path)
    res = map_forces_to_nodes(nodes, forces, mapper)
    os.makedirs(out, exist_ok=True)
    write_nodal_loads_csv(os.path.join(out, "nodal_loads.csv"), nodes, res.nodal)
    write_summary_md(os.path.join(out, "Nodal_loads_summary.md"), res, len(nodes), len(forces),
                     time.time() - t0)
    dF = float(np.max(np.abs(res.global_result["F_tri"] - res.global_result["F_nod"])))
    dM = float(np.max(np.abs(res.global_result["M_tri"] - res.global_result["M_nod"])))
    print("[MapForces] %d nodes, %d triangle forces -> %s (max |dF| %.2e, max |dM| %.2e%s)" % (
        len(nodes), len(forces), out, dF, dM,
        "" if not res.unconverged else f", {res.unconverged} SVDs at the sweep limit"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
