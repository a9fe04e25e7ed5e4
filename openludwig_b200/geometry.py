"""Surface meshes: STL loading with winding repair, longest-edge subdivision,
rotation (alpha about Y, then beta about Z), merging, and the synthetic
bodies of the benchmark workloads (icosphere, cube, NACA0012 wing).

Mirrors geometry/geometry.jl: ``SolverMesh`` (triangles as float64
[n, 3 vertices, xyz], per-triangle normals, areas, centres, bounds).
"""
from __future__ import annotations

import dataclasses as dc
import math
import struct
from pathlib import Path

import numpy as np


@dc.dataclass
class SolverMesh:
    triangles: np.ndarray           # [n, 3, 3] float64
    normals: np.ndarray             # [n, 3]
    areas: np.ndarray               # [n]
    centers: np.ndarray             # [n, 3]

    @property
    def n(self) -> int:
        return int(self.triangles.shape[0])

    @property
    def min_bounds(self) -> tuple:
        return tuple(float(v) for v in self.triangles.reshape(-1, 3).min(axis=0))

    @property
    def max_bounds(self) -> tuple:
        return tuple(float(v) for v in self.triangles.reshape(-1, 3).max(axis=0))


def _cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _norm(v: np.ndarray) -> np.ndarray:
    return np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])


def geometry_properties(tris: np.ndarray):
    """geometry.jl:71-98: unit normal of cross(v2-v1, v3-v1), area, centroid."""
    v1, v2, v3 = tris[:, 0], tris[:, 1], tris[:, 2]
    cp = _cross(v2 - v1, v3 - v1)
    area = 0.5 * _norm(cp)
    with np.errstate(invalid="ignore", divide="ignore"):
        normals = np.where((area > 1e-12)[:, None], cp / (2.0 * area)[:, None], 0.0)
    centers = (v1 + v2 + v3) / 3.0
    return normals, area, centers


def make_mesh(tris: np.ndarray) -> SolverMesh:
    tris = np.ascontiguousarray(tris, dtype=np.float64)
    n, a, c = geometry_properties(tris)
    return SolverMesh(tris, n, a, c)


# ----------------------------------------------------------------------------- STL

def parse_binary_stl(data: bytes, scale: float) -> np.ndarray:
    """geometry.jl:385-429: float32 records; swap v2/v3 where the vertex
    winding disagrees with the stored facet normal."""
    count = struct.unpack_from("<I", data, 80)[0]
    rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]),
                        count=count, offset=84)
    fn = rec["n"].astype(np.float64)
    v = rec["v"].astype(np.float64) * scale
    e1 = v[:, 1] - v[:, 0]
    e2 = v[:, 2] - v[:, 0]
    cp = _cross(e1, e2)
    flip = (cp[:, 0] * fn[:, 0] + cp[:, 1] * fn[:, 1] + cp[:, 2] * fn[:, 2]) < 0.0
    out = v.copy()
    out[flip, 1], out[flip, 2] = v[flip, 2], v[flip, 1]
    return out


def parse_ascii_stl(text: str, scale: float) -> np.ndarray:
    """geometry.jl:431-450: vertex lines grouped per loop (no winding repair)."""
    tris, cur = [], []
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("vertex"):
            p = s.split()
            if len(p) >= 4:
                cur.append([float(p[1]) * scale, float(p[2]) * scale, float(p[3]) * scale])
        elif s.startswith("endloop"):
            if len(cur) == 3:
                tris.append(cur)
            cur = []
    return np.array(tris, dtype=np.float64).reshape(-1, 3, 3)


def load_mesh(filename: str | Path, scale: float = 1.0, min_facet_size: float = 0.0) -> SolverMesh:
    """geometry.jl:458-520."""
    p = Path(filename)
    if not p.is_file():
        raise FileNotFoundError(f"STL file not found: {p}")
    data = p.read_bytes()
    is_binary = True
    if len(data) < 84:
        is_binary = False
    elif data[:5].lower().startswith(b"solid"):
        count = struct.unpack_from("<I", data, 80)[0]
        if len(data) != 84 + count * 50:
            is_binary = False
    tris = parse_binary_stl(data, scale) if is_binary else parse_ascii_stl(data.decode(errors="replace"), scale)
    if tris.shape[0] == 0:
        raise ValueError("No triangles loaded.")
    mesh = make_mesh(tris)
    if min_facet_size > 0.0:
        mesh = subdivide_mesh(mesh, min_facet_size)
    return mesh


def write_stl_binary(filename: str | Path, mesh: SolverMesh, header: bytes = b"openludwig_b200") -> None:
    rec = np.zeros(mesh.n, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]))
    rec["n"] = mesh.normals
    rec["v"] = mesh.triangles
    with open(filename, "wb") as fh:
        fh.write(header[:80].ljust(80, b"\0"))
        fh.write(struct.pack("<I", mesh.n))
        fh.write(rec.tobytes())


# ------------------------------------------------------------------ transforms

def subdivide_mesh(mesh: SolverMesh, min_size: float) -> SolverMesh:
    """geometry.jl:109-258: bisect the longest edge until every edge <= min_size;
    children inherit the parent's normal."""
    if min_size <= 0.0:
        return mesh
    out_t, out_n = [], []
    for tri, nrm in zip(mesh.triangles, mesh.normals):
        work = [tuple(map(tuple, tri))]
        res = []
        while work:
            t = work.pop()
            v1, v2, v3 = (np.array(x) for x in t)
            e1, e2, e3 = np.linalg.norm(v2 - v1), np.linalg.norm(v3 - v2), np.linalg.norm(v1 - v3)
            if max(e1, e2, e3) <= min_size:
                res.append(t)
            elif e1 >= e2 and e1 >= e3:
                m = tuple((v1 + v2) / 2.0)
                work.append((t[0], m, t[2])); work.append((m, t[1], t[2]))
            elif e2 >= e1 and e2 >= e3:
                m = tuple((v2 + v3) / 2.0)
                work.append((t[1], m, t[0])); work.append((m, t[2], t[0]))
            else:
                m = tuple((v3 + v1) / 2.0)
                work.append((t[2], m, t[1])); work.append((m, t[0], t[1]))
        out_t.extend(res)
        out_n.extend([nrm] * len(res))
    tris = np.array(out_t, dtype=np.float64)
    _, area, centers = geometry_properties(tris)
    return SolverMesh(tris, np.array(out_n, dtype=np.float64), area, centers)


def rotation_matrix(alpha_deg: float, beta_deg: float) -> np.ndarray:
    """geometry.jl:279-304: R = Rz(beta) * Ry(alpha)."""
    a, b = math.radians(alpha_deg), math.radians(beta_deg)
    ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
    Ry = np.array([[ca, 0.0, -sa], [0.0, 1.0, 0.0], [sa, 0.0, ca]])
    Rz = np.array([[cb, sb, 0.0], [-sb, cb, 0.0], [0.0, 0.0, 1.0]])
    R = np.empty((3, 3))
    for i in range(3):
        for j in range(3):
            R[i, j] = Rz[i, 0] * Ry[0, j] + Rz[i, 1] * Ry[1, j] + Rz[i, 2] * Ry[2, j]
    return R


def _matvec(R: np.ndarray, v: np.ndarray) -> np.ndarray:
    return np.stack([R[i, 0] * v[..., 0] + R[i, 1] * v[..., 1] + R[i, 2] * v[..., 2]
                     for i in range(3)], axis=-1)


def rotate_mesh(mesh: SolverMesh, alpha_deg: float, beta_deg: float) -> SolverMesh:
    """geometry.jl:267-340: rotate about the bounding-box centre; normals rotate,
    areas and centres are recomputed."""
    if alpha_deg == 0.0 and beta_deg == 0.0:
        return mesh
    R = rotation_matrix(alpha_deg, beta_deg)
    mn, mx = np.array(mesh.min_bounds), np.array(mesh.max_bounds)
    origin = (mn + mx) / 2.0
    tris = _matvec(R, mesh.triangles - origin) + origin
    _, area, centers = geometry_properties(tris)
    return SolverMesh(tris, _matvec(R, mesh.normals), area, centers)


def merge_meshes(meshes: list[SolverMesh]) -> SolverMesh:
    if len(meshes) == 1:
        return meshes[0]
    return SolverMesh(np.concatenate([m.triangles for m in meshes]),
                      np.concatenate([m.normals for m in meshes]),
                      np.concatenate([m.areas for m in meshes]),
                      np.concatenate([m.centers for m in meshes]))


# ------------------------------------------------------------- synthetic bodies

def icosphere(subdivisions: int, radius: float = 1.0, center=(0.0, 0.0, 0.0)) -> SolverMesh:
    """Icosahedron refined `subdivisions` times (20 * 4^s triangles), vertices
    projected to the sphere, outward winding."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    cache: dict = {}

    def mid(i, j):
        key = (min(i, j), max(i, j))
        if key not in cache:
            m = verts[i] + verts[j]
            verts.append(m / np.linalg.norm(m))
            cache[key] = len(verts) - 1
        return cache[key]

    for _ in range(subdivisions):
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    tris = V[np.array(faces)]
    # orient outward
    cp = _cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    cen = tris.mean(axis=1) - np.asarray(center)
    inward = (cp * cen).sum(axis=1) < 0
    tris[inward, 1], tris[inward, 2] = tris[inward, 2].copy(), tris[inward, 1].copy()
    return make_mesh(tris)


def cube(side: float = 1.0, center=(0.0, 0.0, 0.0)) -> SolverMesh:
    """Axis-aligned cube, 12 outward triangles."""
    h = side / 2.0
    c = np.asarray(center, dtype=np.float64)
    P = np.array([[x, y, z] for z in (-h, h) for y in (-h, h) for x in (-h, h)]) + c
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    tris = []
    for a, b, cc, d in quads:
        tris.append([P[a], P[b], P[cc]])
        tris.append([P[a], P[cc], P[d]])
    tris = np.array(tris)
    cp = _cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    cen = tris.mean(axis=1) - c
    inward = (cp * cen).sum(axis=1) < 0
    tris[inward, 1], tris[inward, 2] = tris[inward, 2].copy(), tris[inward, 1].copy()
    return make_mesh(tris)


def flat_plate(side: float = 1.0, n: int = 8, center=(0.0, 0.0, 0.0)) -> SolverMesh:
    """Open square plate of zero thickness in the x-y plane, normal +z,
    n x n panels of 2 triangles: a thin surface with fluid on both sides."""
    s = np.linspace(-side / 2.0, side / 2.0, n + 1)
    tris = []
    for j in range(n):
        for i in range(n):
            a, b = (s[i], s[j], 0.0), (s[i + 1], s[j], 0.0)
            c, d = (s[i + 1], s[j + 1], 0.0), (s[i], s[j + 1], 0.0)
            tris.append([a, b, c]); tris.append([a, c, d])
    return make_mesh(np.array(tris, dtype=np.float64) + np.asarray(center, dtype=np.float64))


def naca0012_wing(chord: float = 1.0, span: float = 3.0, n_chord: int = 200, n_span: int = 40,
                  center=(0.0, 0.0, 0.0)) -> SolverMesh:
    """Closed rectangular NACA0012 wing: chord along x, span along y, thickness
    along z; n_chord x n_span panels per side (2 triangles each) plus tip caps."""
    beta = np.linspace(0.0, math.pi, n_chord + 1)
    xc = 0.5 * (1.0 - np.cos(beta))
    t = 5.0 * 0.12 * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc ** 2 + 0.2843 * xc ** 3
                      - 0.1036 * xc ** 4)
    x = xc * chord - chord / 2.0
    zu, zl = t * chord, -t * chord
    ys = np.linspace(-span / 2.0, span / 2.0, n_span + 1)
    tris = []
    for j in range(n_span):
        y0, y1 = ys[j], ys[j + 1]
        for i in range(n_chord):
            for z in (zu, zl):
                a = (x[i], y0, z[i]); b = (x[i + 1], y0, z[i + 1])
                c = (x[i + 1], y1, z[i + 1]); d = (x[i], y1, z[i])
                tris.append([a, b, c]); tris.append([a, c, d])
    for y in (ys[0], ys[-1]):
        for i in range(n_chord):
            if t[i] == 0.0 and t[i + 1] == 0.0:
                continue
            a = (x[i], y, zu[i]); b = (x[i + 1], y, zu[i + 1])
            c = (x[i + 1], y, zl[i + 1]); d = (x[i], y, zl[i])
            if t[i + 1] > 0.0:
                tris.append([a, b, c])
            if t[i] > 0.0:
                tris.append([a, c, d])
    tris = np.array(tris, dtype=np.float64) + np.asarray(center, dtype=np.float64)
    # orient outward (convex per section: compare with the local section centre)
    cp = _cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    cen = tris.mean(axis=1)
    ref = np.zeros_like(cen)
    ref[:, 0] = cen[:, 0]
    ref[:, 1] = np.where(np.abs(cp[:, 1]) > np.abs(cp[:, 2]), center[1], cen[:, 1])
    ref[:, 2] = center[2]
    inward = (cp * (cen - ref)).sum(axis=1) < 0
    tris[inward, 1], tris[inward, 2] = tris[inward, 2].copy(), tris[inward, 1].copy()
    return make_mesh(tris)
