"""Multi-level sparse block domain (geometry/domain.jl, domain_topology.jl,
domain_generation.jl, bouzidi_setup.jl, bouzidi_math.jl), vectorised with
numpy on the host.

Each level is a sorted list of active 8^3 blocks (lexicographic (bx, by, bz),
block id = rank + 1) with its 27-neighbour table, dense block pointer grid,
obstacle / sponge / wall-distance masks and, on Bouzidi levels, the Float16
q-map with its sparse boundary-cell list.  All arrays use the reference's
column-major layout (see include/openludwig_b200.h) so they can be uploaded
unchanged.  FP64 geometry is evaluated in the reference's expression order;
the tests compare every integer output with the oracle bit for bit.
"""
from __future__ import annotations

import dataclasses as dc
import math

import numpy as np

from .config import CaseConfig
from .geometry import SolverMesh
from .scaling import DomainParams

BS = 8


@dc.dataclass
class HostLevel:
    level_id: int
    dx: float                     # Float64(Float32(dx)) as BlockLevel stores it
    dx_exact: float               # the Float64 dx the geometry used
    tau: float
    tau_g: float
    coords: np.ndarray            # [n, 3] int32, 1-based
    neighbor_table: np.ndarray    # [27 * n] int32 (b + n*dir), 1-based ids
    block_ptr: np.ndarray         # [dx*dy*dz] int32, bx fastest
    grid_dim: tuple               # size(block_ptr) = max active coords
    obstacle: np.ndarray          # [512 n] uint8
    sponge: np.ndarray            # [512 n] float32
    wall_dist: np.ndarray         # [512 n] float32 (100 = far)
    bouzidi: bool = False
    q_map: np.ndarray | None = None      # [512 n 27] uint16 (binary16 bits)
    tri_map: np.ndarray | None = None    # [512 n 27] int32 (1-based triangle ids)
    cell_block: np.ndarray | None = None  # [nb] int32 1-based
    cell_x: np.ndarray | None = None     # [nb] int8 1-based
    cell_y: np.ndarray | None = None
    cell_z: np.ndarray | None = None

    @property
    def n_blocks(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_boundary(self) -> int:
        return 0 if self.cell_block is None else int(self.cell_block.shape[0])

    @property
    def map_x(self) -> np.ndarray:
        return np.ascontiguousarray(self.coords[:, 0])

    @property
    def map_y(self) -> np.ndarray:
        return np.ascontiguousarray(self.coords[:, 1])

    @property
    def map_z(self) -> np.ndarray:
        return np.ascontiguousarray(self.coords[:, 2])


# ------------------------------------------------------------------ topology

def _floor_int(v: np.ndarray) -> np.ndarray:
    return np.floor(v).astype(np.int64)


def active_blocks_for_level(tris: np.ndarray, dx: float, offset, dims) -> set:
    """domain_topology.jl:9-52: blocks overlapped by each triangle's AABB
    (+0.01 dx), clamped to the level dims."""
    off = np.asarray(offset, dtype=np.float64)
    p = tris + off
    mn = p.min(axis=1)
    mx = p.max(axis=1)
    margin = dx * 0.01
    inv = 1.0 / (BS * dx)
    lo = _floor_int((mn - margin) * inv) + 1
    hi = _floor_int((mx + margin) * inv) + 1
    lo = np.maximum(lo, 1)
    hi = np.minimum(hi, np.asarray(dims))
    out = set()
    for (x0, y0, z0), (x1, y1, z1) in zip(lo.tolist(), hi.tolist()):
        for bz in range(z0, z1 + 1):
            for by in range(y0, y1 + 1):
                for bx in range(x0, x1 + 1):
                    out.add((bx, by, bz))
    return out


def _in(b, dims) -> bool:
    return 1 <= b[0] <= dims[0] and 1 <= b[1] <= dims[1] and 1 <= b[2] <= dims[2]


_OFFS26 = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
           if (dx, dy, dz) != (0, 0, 0)]
_SIB = [(dx, dy, dz) for dz in (0, 1) for dy in (0, 1) for dx in (0, 1)]


def add_halo_blocks_with_siblings(s: set, layers: int, dims) -> None:
    """domain_topology.jl:54-99."""
    for _ in range(layers):
        new = set()
        for (bx, by, bz) in s:
            for dx, dy, dz in _OFFS26:
                n = (bx + dx, by + dy, bz + dz)
                if _in(n, dims) and n not in s:
                    new.add(n)
        sib = set()
        for (bx, by, bz) in new:
            px, py, pz = (bx + 1) // 2, (by + 1) // 2, (bz + 1) // 2
            for dx, dy, dz in _SIB:
                c = (2 * px - 1 + dx, 2 * py - 1 + dy, 2 * pz - 1 + dz)
                if _in(c, dims) and c not in s and c not in new:
                    sib.add(c)
        s |= new
        s |= sib


def ensure_complete_parent_coverage(s: set, dims) -> None:
    """domain_topology.jl:101-133."""
    added, it = True, 0
    while added and it < 10:
        added = False
        it += 1
        add = set()
        for (bx, by, bz) in s:
            px, py, pz = (bx + 1) // 2, (by + 1) // 2, (bz + 1) // 2
            for dx, dy, dz in _SIB:
                c = (2 * px - 1 + dx, 2 * py - 1 + dy, 2 * pz - 1 + dz)
                if _in(c, dims) and c not in s:
                    add.add(c)
                    added = True
        s |= add


def build_neighbor_table(coords: np.ndarray, dims) -> np.ndarray:
    """domain_topology.jl:135-159 -> flat [b + n*dir], 1-based ids, 0 = none."""
    n = coords.shape[0]
    ptr = np.zeros((dims[2] + 2, dims[1] + 2, dims[0] + 2), dtype=np.int32)
    ptr[coords[:, 2], coords[:, 1], coords[:, 0]] = np.arange(1, n + 1, dtype=np.int32)
    table = np.zeros((27, n), dtype=np.int32)
    d = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                table[d] = ptr[coords[:, 2] + dz, coords[:, 1] + dy, coords[:, 0] + dx]
                d += 1
    return table.reshape(-1)


def block_pointer(coords: np.ndarray) -> tuple[np.ndarray, tuple]:
    """blocks.jl:239-250: dense grid sized by the max active coordinates."""
    if coords.shape[0] == 0:
        return np.zeros(0, dtype=np.int32), (0, 0, 0)
    dims = tuple(int(v) for v in coords.max(axis=0))
    ptr = np.zeros((dims[2], dims[1], dims[0]), dtype=np.int32)
    ptr[coords[:, 2] - 1, coords[:, 1] - 1, coords[:, 0] - 1] = np.arange(1, coords.shape[0] + 1)
    return ptr.reshape(-1), dims


def _cell_centers(coords: np.ndarray, dx: float) -> np.ndarray:
    """((b-1)*8 + l - 0.5) * dx per cell, [n, 512, 3] (x fastest)."""
    l = np.arange(1, BS + 1)
    lz, ly, lx = np.meshgrid(l, l, l, indexing="ij")
    loc = np.stack([lx.reshape(-1), ly.reshape(-1), lz.reshape(-1)], axis=-1)  # [512, 3]
    g = (coords[:, None, :].astype(np.int64) - 1) * BS + loc[None]
    return (g.astype(np.float64) - 0.5) * dx


def block_triangle_map(tris: np.ndarray, coords: np.ndarray, dx: float, offset,
                       margin: float) -> list:
    """Triangles whose AABB (+margin) overlaps each block, in triangle order
    (domain_generation.jl:34-72, bouzidi_setup.jl:12-54)."""
    n = coords.shape[0]
    out = [[] for _ in range(n)]
    if n == 0:
        return out
    off = np.asarray(offset, dtype=np.float64)
    p = tris + off
    mn, mx = p.min(axis=1), p.max(axis=1)
    bsd = BS * dx
    lo = _floor_int((mn - margin) / bsd) + 1
    hi = _floor_int((mx + margin) / bsd) + 1
    dims = coords.max(axis=0)
    lut = np.full((dims[2] + 1, dims[1] + 1, dims[0] + 1), -1, dtype=np.int64)
    lut[coords[:, 2], coords[:, 1], coords[:, 0]] = np.arange(n)
    for t, ((x0, y0, z0), (x1, y1, z1)) in enumerate(zip(lo.tolist(), hi.tolist())):
        x0, y0, z0 = max(1, x0), max(1, y0), max(1, z0)
        x1, y1, z1 = min(x1, int(dims[0])), min(y1, int(dims[1])), min(z1, int(dims[2]))
        if x0 > x1 or y0 > y1 or z0 > z1:
            continue
        ids = lut[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1].reshape(-1)
        for i in ids[ids >= 0].tolist():
            out[i].append(t)
    return out


# -------------------------------------------------------------- voxelization

def _tri_box_any(c: np.ndarray, h0: float, v1, v2, v3) -> np.ndarray:
    """domain_generation.jl:10-32 vectorised over cells [m,3] x triangles [T,3];
    returns [m] bool (some triangle overlaps the cell box)."""
    h = h0 * 1.001
    t1 = v1[None] - c[:, None]
    t2 = v2[None] - c[:, None]
    t3 = v3[None] - c[:, None]
    ok = np.ones(t1.shape[:2], dtype=bool)
    for a in range(3):
        mn = np.minimum(np.minimum(t1[..., a], t2[..., a]), t3[..., a])
        mx = np.maximum(np.maximum(t1[..., a], t2[..., a]), t3[..., a])
        ok &= ~((mn > h) | (mx < -h))
    f = (t2 - t1, t3 - t2, t1 - t3)
    units = ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0))
    for u in units:
        for fj in f:
            ax = u[1] * fj[..., 2] - u[2] * fj[..., 1]
            ay = u[2] * fj[..., 0] - u[0] * fj[..., 2]
            az = u[0] * fj[..., 1] - u[1] * fj[..., 0]
            skip = (ax * ax + ay * ay + az * az) < 1e-10
            p1 = t1[..., 0] * ax + t1[..., 1] * ay + t1[..., 2] * az
            p2 = t2[..., 0] * ax + t2[..., 1] * ay + t2[..., 2] * az
            p3 = t3[..., 0] * ax + t3[..., 1] * ay + t3[..., 2] * az
            r = h * np.abs(ax) + h * np.abs(ay) + h * np.abs(az)
            sep = (np.minimum(p1, np.minimum(p2, p3)) > r) | (np.maximum(p1, np.maximum(p2, p3)) < -r)
            ok &= skip | ~sep
    return ok.any(axis=1)


def voxelize_blocks(coords: np.ndarray, tris: np.ndarray, dx: float, offset) -> np.ndarray:
    """domain_generation.jl:74-112: cells whose 1.5 dx box a triangle touches."""
    n = coords.shape[0]
    obst = np.zeros(n * 512, dtype=np.uint8)
    bmap = block_triangle_map(tris, coords, dx, offset, dx * 2)
    off = np.asarray(offset, dtype=np.float64)
    cent = _cell_centers(coords, dx)
    for i, tl in enumerate(bmap):
        if not tl:
            continue
        T = tris[tl] + off
        hit = _tri_box_any(cent[i], 0.75 * dx, T[:, 0], T[:, 1], T[:, 2])
        obst[i * 512:(i + 1) * 512] = hit.astype(np.uint8)
    return obst


def flood_fill(coords: np.ndarray, obstacle: np.ndarray) -> np.ndarray:
    """domain_generation.jl:114-203: cells not 6-connected (through active
    blocks) to a fluid cell of the min-x block layer become solid."""
    from scipy import ndimage
    n = coords.shape[0]
    if n == 0:
        return obstacle
    lo = coords.min(axis=0)
    hi = coords.max(axis=0)
    ext = (hi - lo + 1) * BS
    fluid = np.zeros((ext[2], ext[1], ext[0]), dtype=bool)
    ob = obstacle.reshape(n, BS, BS, BS)  # [b, z, y, x]
    o = (coords - lo) * BS
    for i in range(n):
        fluid[o[i, 2]:o[i, 2] + BS, o[i, 1]:o[i, 1] + BS, o[i, 0]:o[i, 0] + BS] = ob[i] == 0
    lab, _ = ndimage.label(fluid)  # default structure = 6-connectivity
    minx = coords[:, 0].min()
    seeds = set()
    for i in np.nonzero(coords[:, 0] == minx)[0]:
        blk = lab[o[i, 2]:o[i, 2] + BS, o[i, 1]:o[i, 1] + BS, o[i, 0]:o[i, 0] + BS]
        seeds.update(np.unique(blk[blk > 0]).tolist())
    keep = np.isin(lab, np.array(sorted(seeds), dtype=lab.dtype)) if seeds else np.zeros_like(fluid)
    out = obstacle.copy().reshape(n, BS, BS, BS)
    for i in range(n):
        k = keep[o[i, 2]:o[i, 2] + BS, o[i, 1]:o[i, 1] + BS, o[i, 0]:o[i, 0] + BS]
        out[i][(out[i] == 0) & ~k] = 1
    return out.reshape(-1)


def _sponge_profile(x: np.ndarray, thk: float) -> np.ndarray:
    import math as _m
    out = np.where(x <= 0.0, 1.0, 0.0)
    mid = (x > 0.0) & (x < thk)
    if mid.any():
        arg = (np.pi * x[mid]) / thk
        out[mid] = 0.5 * (1.0 + np.array([_m.cos(a) for a in arg.tolist()]))
    return out


def apply_sponge(coords: np.ndarray, dx: float, domain_size, sponge_thickness: float,
                 symmetric: bool) -> np.ndarray:
    """domain_generation.jl:215-289."""
    Lx, Ly, Lz = domain_size
    st = float(sponge_thickness)
    out_thk = Lx * max(st, 0.08)
    in_thk = Lx * 0.02
    y_thk = Ly * st * 0.5
    z_thk = Lz * st * 0.5
    out_start, y_top, z_back = Lx - out_thk, Ly - y_thk, Lz - z_thk
    c = _cell_centers(coords, dx).reshape(-1, 3)
    px, py, pz = c[:, 0], c[:, 1], c[:, 2]
    s = np.zeros(px.shape[0])
    m = px > out_start
    if m.any():
        s[m] = np.maximum(s[m], _sponge_profile(out_thk - (px[m] - out_start), out_thk) * 1.0)
    m = px < in_thk
    if m.any():
        s[m] = np.maximum(s[m], _sponge_profile(px[m], in_thk) * 0.05)
    if not symmetric:
        m = py < y_thk
        if m.any():
            s[m] = np.maximum(s[m], _sponge_profile(py[m], y_thk) * 0.1)
    m = py > y_top
    if m.any():
        s[m] = np.maximum(s[m], _sponge_profile(y_thk - (py[m] - y_top), y_thk) * 0.1)
    m = pz < z_thk
    if m.any():
        s[m] = np.maximum(s[m], _sponge_profile(pz[m], z_thk) * 0.1)
    m = pz > z_back
    if m.any():
        s[m] = np.maximum(s[m], _sponge_profile(z_thk - (pz[m] - z_back), z_thk) * 0.1)
    return s.astype(np.float32)


def gather_halo(values: np.ndarray, table: np.ndarray, n: int, fill) -> np.ndarray:
    """Per block, its 8^3 values plus a one-cell halo from the 26 neighbours
    -> [n, 10, 10, 10] ([b, z, y, x]); absent neighbours give `fill`."""
    v = values.reshape(n, BS, BS, BS)
    ext = np.concatenate([v, np.full((1, BS, BS, BS), fill, dtype=values.dtype)], axis=0)
    tab = table.reshape(27, n)
    out = np.empty((n, BS + 2, BS + 2, BS + 2), dtype=values.dtype)
    sl = {-1: (slice(0, 1), slice(BS - 1, BS)), 0: (slice(1, BS + 1), slice(0, BS)),
          1: (slice(BS + 1, BS + 2), slice(0, 1))}
    d = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                nb = tab[d].astype(np.int64) - 1
                nb[nb < 0] = n
                out[:, sl[dz][0], sl[dy][0], sl[dx][0]] = ext[nb][:, sl[dz][1], sl[dy][1], sl[dx][1]]
                d += 1
    return out


def compute_wall_distances(coords: np.ndarray, table: np.ndarray, obstacle: np.ndarray,
                           dx: float) -> np.ndarray:
    """domain_generation.jl:371-434: for fluid cells next to a solid cell,
    the smallest link length to it (Float32 sqrt(|c|^2) * Float32(dx))."""
    n = coords.shape[0]
    wd = np.full(n * 512, 100.0, dtype=np.float32)
    if n == 0:
        return wd
    halo = gather_halo(obstacle, table, n, np.uint8(0))
    md = np.full((n, BS, BS, BS), np.float32(100.0), dtype=np.float32)
    near = np.zeros((n, BS, BS, BS), dtype=bool)
    fdx = np.float32(dx)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dxo in (-1, 0, 1):
                if (dxo, dy, dz) == (0, 0, 0):
                    continue
                nbv = halo[:, 1 + dz:1 + dz + BS, 1 + dy:1 + dy + BS, 1 + dxo:1 + dxo + BS] != 0
                d = np.sqrt(np.float32(dxo * dxo + dy * dy + dz * dz)) * fdx
                md = np.where(nbv, np.minimum(md, d), md)
                near |= nbv
    own = obstacle.reshape(n, BS, BS, BS) != 0
    sel = near & ~own
    wd = wd.reshape(n, BS, BS, BS)
    wd[sel] = md[sel]
    return wd.reshape(-1)


# ------------------------------------------------------------------- Bouzidi

def _dirs():
    out = []
    for cz in (-1, 0, 1):
        for cy in (-1, 0, 1):
            for cx in (-1, 0, 1):
                out.append((cx, cy, cz))
    return out


DIRS = _dirs()


def compute_bouzidi_qmap(coords: np.ndarray, tris: np.ndarray, dx: float, offset):
    """bouzidi_setup.jl:64-166 + bouzidi_math.jl: per cell and link, the
    nearest Moller-Trumbore hit along the unit link direction, q = t/(dx|c|)
    in (0, 1] stored as binary16, plus the hit triangle (1-based)."""
    n = coords.shape[0]
    S = n * 512
    q16 = np.zeros(S * 27, dtype=np.uint16)
    trim = np.zeros(S * 27, dtype=np.int32)
    bmap = block_triangle_map(tris, coords, dx, offset, dx * 2.5)
    off = np.asarray(offset, dtype=np.float64)
    cent = _cell_centers(coords, dx)
    cells = []
    eps = 1e-9
    for i, tl in enumerate(bmap):
        if not tl:
            continue
        T = tris[tl] + off
        v1, v2, v3 = T[:, 0], T[:, 1], T[:, 2]
        e1 = v2 - v1
        e2 = v3 - v1
        c = cent[i]                        # [512, 3]
        s = c[:, None, :] - v1[None]       # [512, T, 3]
        qv_ = np.stack([s[..., 1] * e1[None, :, 2] - s[..., 2] * e1[None, :, 1],
                        s[..., 2] * e1[None, :, 0] - s[..., 0] * e1[None, :, 2],
                        s[..., 0] * e1[None, :, 1] - s[..., 1] * e1[None, :, 0]], axis=-1)
        has = np.zeros(512, dtype=bool)
        tl_arr = np.asarray(tl, dtype=np.int32)
        for k, (cx, cy, cz) in enumerate(DIRS):
            if cx == 0 and cy == 0 and cz == 0:
                continue
            nrm = math.sqrt(float(cx * cx) + float(cy * cy) + float(cz * cz))
            d = (cx / nrm, cy / nrm, cz / nrm)
            hx = d[1] * e2[:, 2] - d[2] * e2[:, 1]
            hy = d[2] * e2[:, 0] - d[0] * e2[:, 2]
            hz = d[0] * e2[:, 1] - d[1] * e2[:, 0]
            a = e1[:, 0] * hx + e1[:, 1] * hy + e1[:, 2] * hz
            valid_t = ~(np.abs(a) < eps)
            with np.errstate(divide="ignore", invalid="ignore"):
                f = 1.0 / a
                u = f[None] * (s[..., 0] * hx[None] + s[..., 1] * hy[None] + s[..., 2] * hz[None])
                v = f[None] * (d[0] * qv_[..., 0] + d[1] * qv_[..., 1] + d[2] * qv_[..., 2])
                t = f[None] * (e2[None, :, 0] * qv_[..., 0] + e2[None, :, 1] * qv_[..., 1]
                               + e2[None, :, 2] * qv_[..., 2])
                hit = valid_t[None] & ~((u < 0.0) | (u > 1.0)) & ~((v < 0.0) | (u + v > 1.0)) & (t > eps)
            tt = np.where(hit, t, np.inf)
            j = np.argmin(tt, axis=1)
            mt = tt[np.arange(512), j]
            found = mt < np.inf
            q = np.where(found, mt / (dx * nrm), 0.0)
            ok = found & (q > 0.0) & (q <= 1.0)
            if ok.any():
                idx = i * 512 + np.nonzero(ok)[0] + k * S
                q16[idx] = q[ok].astype(np.float16).view(np.uint16)
                trim[idx] = tl_arr[j[ok]] + 1
                has |= ok
        for cidx in np.nonzero(has)[0].tolist():
            cells.append((i + 1, cidx % 8 + 1, (cidx // 8) % 8 + 1, cidx // 64 + 1))
    cells = np.array(cells, dtype=np.int32).reshape(-1, 4)
    return q16, trim, cells


# ------------------------------------------------- the same two steps on a GPU

def _tri_csr(bmap: list) -> tuple[np.ndarray, np.ndarray]:
    off = np.zeros(len(bmap) + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(t) for t in bmap])
    lst = np.fromiter((t for tl in bmap for t in tl), dtype=np.int32, count=int(off[-1]))
    return off, lst


class DeviceGeometry:
    """Triangles of one mesh resident on a CUDA device, for ol_voxelize and
    ol_bouzidi_qmap (same bits as voxelize_blocks / compute_bouzidi_qmap)."""

    def __init__(self, tris: np.ndarray, device: int = 0):
        import torch
        from . import _native as N
        self.torch, self.N = torch, N
        self.dev = torch.device("cuda", device)
        self.n_tris = int(tris.shape[0])
        self.tris = torch.from_numpy(np.ascontiguousarray(tris, dtype=np.float64)).to(self.dev)

    def _common(self, coords, bmap, dx, offset):
        t = self.torch
        off_arr, lst = _tri_csr(bmap)
        d_coords = t.from_numpy(np.ascontiguousarray(coords, dtype=np.int32)).to(self.dev)
        d_off = t.from_numpy(off_arr).to(self.dev)
        d_lst = t.from_numpy(lst if lst.size else np.zeros(1, np.int32)).to(self.dev)
        o3 = (self.N.C.c_double * 3)(*[float(v) for v in offset])
        return d_coords, d_off, d_lst, o3

    def _p(self, a):
        return self.N.C.c_void_p(a.data_ptr())

    def voxelize(self, coords: np.ndarray, dx: float, offset, bmap: list) -> np.ndarray:
        n = coords.shape[0]
        d_coords, d_off, d_lst, o3 = self._common(coords, bmap, dx, offset)
        out = self.torch.empty(n * 512, dtype=self.torch.uint8, device=self.dev)
        s = self.N.C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)
        self.N.call("ol_voxelize", self._p(d_coords), self.N.i32(n), self._p(self.tris),
                    self.N.i32(self.n_tris), self._p(d_off), self._p(d_lst), float(dx), o3,
                    self._p(out), s)
        return out.cpu().numpy()

    def qmap(self, coords: np.ndarray, dx: float, offset, bmap: list):
        t = self.torch
        n = coords.shape[0]
        S = n * 512
        d_coords, d_off, d_lst, o3 = self._common(coords, bmap, dx, offset)
        q = t.empty(S * 27, dtype=t.int16, device=self.dev)
        tri = t.empty(S * 27, dtype=t.int32, device=self.dev)
        has = t.empty(S, dtype=t.uint8, device=self.dev)
        s = self.N.C.c_void_p(t.cuda.current_stream(self.dev).cuda_stream)
        self.N.call("ol_bouzidi_qmap", self._p(d_coords), self.N.i32(n), self._p(self.tris),
                    self.N.i32(self.n_tris), self._p(d_off), self._p(d_lst), float(dx), o3,
                    self._p(q), self._p(tri), self._p(has), s)
        q16 = q.cpu().numpy().view(np.uint16)
        trim = tri.cpu().numpy()
        idx = np.nonzero(has.cpu().numpy())[0]
        cells = np.stack([idx // 512 + 1, idx % 8 + 1, (idx // 8) % 8 + 1, (idx // 64) % 8 + 1],
                         axis=1).astype(np.int32).reshape(-1, 4)
        return q16, trim, cells


def should_use_bouzidi(level_id: int, num_levels: int, method: str, bouzidi_levels: int) -> bool:
    """bouzidi_common.jl:28-33."""
    return method == "bouzidi" and level_id > num_levels - bouzidi_levels


# -------------------------------------------------------------- orchestration

def level_block_set(lvl: int, tris: np.ndarray, dx: float, offset, dims, prev_coords,
                    prev_bs_phys: float, wake_box, cfg: CaseConfig) -> np.ndarray:
    """domain.jl:39-152 for one level -> sorted [n, 3] int32 coordinates."""
    s: set = set()
    if lvl == 1:
        for bz in range(1, dims[2] + 1):
            for by in range(1, dims[1] + 1):
                for bx in range(1, dims[0] + 1):
                    s.add((bx, by, bz))
    elif cfg.refinement_strategy == "geometry_first":
        s = active_blocks_for_level(tris, dx, offset, dims)
        if cfg.wake_enabled and wake_box is not None:
            x0, x1, y0, y1, z0, z1 = wake_box
            for (cbx, cby, cbz) in prev_coords.tolist():
                ox = (cbx - 1) * prev_bs_phys <= x1 and cbx * prev_bs_phys >= x0
                oy = (cby - 1) * prev_bs_phys <= y1 and cby * prev_bs_phys >= y0
                oz = (cbz - 1) * prev_bs_phys <= z1 and cbz * prev_bs_phys >= z0
                if ox and oy and oz:
                    for dx_, dy_, dz_ in _SIB:
                        c = (2 * cbx - 1 + dx_, 2 * cby - 1 + dy_, 2 * cbz - 1 + dz_)
                        if _in(c, dims):
                            s.add(c)
        prev = set(map(tuple, prev_coords.tolist()))
        s = {b for b in s if ((b[0] + 1) // 2, (b[1] + 1) // 2, (b[2] + 1) // 2) in prev}
    else:
        raise NotImplementedError("only refinement.strategy = geometry_first is supported")
    add_halo_blocks_with_siblings(s, cfg.refinement_margin, dims)
    ensure_complete_parent_coverage(s, dims)
    return np.array(sorted(s), dtype=np.int32).reshape(-1, 3)


def setup_multilevel_domain(cfg: CaseConfig, mesh: SolverMesh, p: DomainParams,
                            with_bouzidi: bool = True,
                            device: int | None = None) -> list[HostLevel]:
    """domain.jl:1-246.  device: CUDA device for the voxelisation and the
    Bouzidi q-map (ol_voxelize / ol_bouzidi_qmap, same bits), None = host."""
    tris = mesh.triangles
    offset = p.mesh_offset
    dg = DeviceGeometry(tris, device) if device is not None else None
    pmin = np.asarray(p.mesh_min) + np.asarray(offset)
    pmax = np.asarray(p.mesh_max) + np.asarray(offset)
    wake_box = None
    if cfg.wake_enabled:
        wx0 = pmax[0] - p.reference_length * 0.1
        wx1 = pmax[0] + p.reference_length * cfg.wake_length
        cy, cz = (pmin[1] + pmax[1]) / 2.0, (pmin[2] + pmax[2]) / 2.0
        ww = (pmax[1] - pmin[1]) * cfg.wake_width_factor
        wh = (pmax[2] - pmin[2]) * cfg.wake_height_factor
        wake_box = (wx0, wx1, cy - ww / 2.0, cy + ww / 2.0, cz - wh / 2.0, cz + wh / 2.0)
    levels: list[HostLevel] = []
    for lvl in range(1, p.num_levels + 1):
        scale = 2 ** (lvl - 1)
        dx = p.dx_coarse / scale
        dims = (p.bx_max * scale, p.by_max * scale, p.bz_max * scale)
        prev_coords = levels[-1].coords if levels else None
        prev_bs_phys = BS * (p.dx_coarse / 2 ** (lvl - 2)) if lvl > 1 else 0.0
        coords = level_block_set(lvl, tris, dx, offset, dims, prev_coords, prev_bs_phys,
                                 wake_box, cfg)
        table = build_neighbor_table(coords, dims)
        ptr, gdim = block_pointer(coords)
        if dg is not None:
            obst = dg.voxelize(coords, dx, offset,
                               block_triangle_map(tris, coords, dx, offset, dx * 2))
        else:
            obst = voxelize_blocks(coords, tris, dx, offset)
        obst = flood_fill(coords, obst)
        sponge = apply_sponge(coords, dx, p.domain_size, cfg.sponge_thickness, cfg.symmetric_analysis)
        wd = (compute_wall_distances(coords, table, obst, dx) if cfg.wall_model_enabled
              else np.full(coords.shape[0] * 512, 100.0, dtype=np.float32))
        tau_g = p.tau_g_levels[lvl - 1] if p.tau_g_levels else 0.0
        lv = HostLevel(level_id=lvl, dx=float(np.float32(dx)), dx_exact=dx,
                       tau=p.tau_levels[lvl - 1], tau_g=tau_g, coords=coords,
                       neighbor_table=table, block_ptr=ptr, grid_dim=gdim, obstacle=obst,
                       sponge=sponge, wall_dist=wd)
        if with_bouzidi and should_use_bouzidi(lvl, p.num_levels, cfg.boundary_method,
                                               cfg.bouzidi_levels):
            if dg is not None:
                q16, trim, cells = dg.qmap(coords, dx, offset,
                                           block_triangle_map(tris, coords, dx, offset, dx * 2.5))
            else:
                q16, trim, cells = compute_bouzidi_qmap(coords, tris, dx, offset)
            if cells.shape[0] > 0:
                lv.bouzidi = True
                lv.q_map, lv.tri_map = q16, trim
                lv.cell_block = np.ascontiguousarray(cells[:, 0]).astype(np.int32)
                lv.cell_x = cells[:, 1].astype(np.int8)
                lv.cell_y = cells[:, 2].astype(np.int8)
                lv.cell_z = cells[:, 3].astype(np.int8)
        levels.append(lv)
    return levels
