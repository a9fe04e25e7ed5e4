"""Run records the reference writes beside the flow field: the per-diagnostic
convergence and force tables, the binary surface-pressure file and the
two-sided per-triangle force table.

  CONVERGENCE_HEADER / convergence_row   convergence.csv (main.jl:56-57, :250-257)
  FORCE_HEADER / force_row               forces.csv (forces/io.jl:5-23)
  write_surface_pressure_bin             surface_%06d.lbmp (forces/io.jl:236-351)
  write_net_forces_csv                   net_forces_%06d.csv (forces/io.jl:141-234)

The numbers come from the device (force sums, per-triangle pressure and shear
maps, net forces); these functions only format them.  Text rows use the
reference's printf formats, which Python's %-formatting renders identically
(both round correctly).  Binary output is little-endian, as the reference
writes on x86.
"""
from __future__ import annotations

import math
import os

import numpy as np

CONVERGENCE_HEADER = "Step,Time_phys_s,Domain_travel_pct,U_inlet_lat,Rho_min,MLUPS,Cd,Cl,Cs"
FORCE_HEADER = ("Step,Time_phys_s,U_inlet_lat,Fx_N,Fy_N,Fz_N,Fx_p,Fy_p,Fz_p,Fx_v,Fy_v,Fz_v,"
                "Mx,My,Mz,Cd,Cl,Cs,Cmx,Cmy,Cmz")
NET_FORCE_HEADER = "triangle_id,object_name,cx,cy,cz,Fx,Fy,Fz"
LBMP_MAGIC = b"LBMP"
LBMP_VERSION = 1


def convergence_row(step: int, time_phys: float, travel_pct: float, u_inlet: float,
                    rho_min: float, mlups: float, fr=None) -> str:
    """One line of convergence.csv (main.jl:255-256); Cd/Cl/Cs as "%.4f"
    strings, or "N/A" without forces."""
    if fr is None:
        cd = cl = cs = "N/A"
    else:
        cd, cl, cs = ("%.4f" % fr.Cd), ("%.4f" % fr.Cl), ("%.4f" % fr.Cs)
    return "%d,%.6e,%.6e,%.4f,%.6f,%.1f,%s,%s,%s" % (step, time_phys, travel_pct, u_inlet,
                                                     rho_min, mlups, cd, cl, cs)


def force_row(step: int, time_phys: float, fr, u_inlet: float) -> str:
    """append_force_csv (forces/io.jl:11-23): totals, pressure and viscous
    parts, moments (N, N m) and the six coefficients of a ForceResult."""
    fx, fy, fz = fr.Fx_p + fr.Fx_v, fr.Fy_p + fr.Fy_v, fr.Fz_p + fr.Fz_v
    return ("%d,%.6e,%.6f,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,"
            "%.6f,%.6f,%.6f,%.6f,%.6f,%.6f" % (
                step, time_phys, float(np.float32(u_inlet)), fx, fy, fz, fr.Fx_p, fr.Fy_p,
                fr.Fz_p, fr.Fx_v, fr.Fy_v, fr.Fz_v, fr.Mx, fr.My, fr.Mz, fr.Cd, fr.Cl, fr.Cs,
                fr.Cmx, fr.Cmy, fr.Cmz))


class RunRecords:
    """convergence.csv and (with forces) forces.csv in one output folder,
    created with their headers like main.jl:52-60 and appended per
    diagnostics step."""

    def __init__(self, output_dir: str, forces: bool):
        os.makedirs(output_dir, exist_ok=True)
        self.conv = os.path.join(output_dir, "convergence.csv")
        self.force = os.path.join(output_dir, "forces.csv") if forces else None
        with open(self.conv, "w") as f:
            f.write(CONVERGENCE_HEADER + "\n")
        if self.force:
            with open(self.force, "w") as f:
                f.write(FORCE_HEADER + "\n")

    def append(self, step: int, time_phys: float, travel_pct: float, u_inlet: float,
               rho_min: float, mlups: float, fr=None) -> None:
        if self.force and fr is not None:
            with open(self.force, "a") as f:
                f.write(force_row(step, time_phys, fr, u_inlet) + "\n")
        with open(self.conv, "a") as f:
            f.write(convergence_row(step, time_phys, travel_pct, u_inlet, rho_min, mlups, fr) + "\n")


def _names_table(object_names, n):
    if object_names is None:
        return ["default"], np.ones(n, np.int32)
    uniq = list(dict.fromkeys(object_names))           # first-seen order, like unique()
    ids = {s: i + 1 for i, s in enumerate(uniq)}
    return uniq, np.array([ids[s] for s in object_names], np.int32)


def write_surface_pressure_bin(path: str, triangles: np.ndarray, normals: np.ndarray,
                               pressure: np.ndarray, shear: np.ndarray, rho_ref: float,
                               u_ref: float, offset=(0.0, 0.0, 0.0), object_names=None) -> None:
    """export_surface_pressure_bin (forces/io.jl:260-351): header "LBMP",
    version 1, triangle and object counts; the object-name table; then
    vertices [n, 9] (Float32(v) + Float32(offset)), normals [n, 3], gauge
    pressure, shear magnitude sqrt(sx^2 + sy^2 + sz^2) and Cp = p / q_inf
    (Float32(q_inf), zero when q_inf <= 1e-10) as Float32, object ids as
    Int32.  `shear` is the [3, n] Float32 shear map."""
    tri = np.asarray(triangles, np.float64)
    n = tri.shape[0]
    off = np.asarray([np.float32(v) for v in offset], np.float32)
    verts = (tri.reshape(n, 3, 3).astype(np.float32) + off).reshape(n, 9)
    p = np.asarray(pressure, np.float32)
    sx, sy, sz = (np.asarray(shear[i], np.float32) for i in range(3))
    smag = np.sqrt(sx * sx + sy * sy + sz * sz).astype(np.float32)
    q_inf = np.float32(0.5 * rho_ref * u_ref ** 2)
    cp = (p / q_inf).astype(np.float32) if q_inf > np.float32(1e-10) else np.zeros(n, np.float32)
    names, ids = _names_table(object_names, n)
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "wb") as f:
        f.write(LBMP_MAGIC)
        f.write(np.array([LBMP_VERSION, n, len(names)], "<u4").tobytes())
        for s in names:
            b = s.encode("utf-8")
            f.write(np.array([len(b)], "<u4").tobytes())
            f.write(b)
        f.write(verts.astype("<f4").tobytes())
        f.write(np.asarray(normals, np.float32).reshape(n, 3).astype("<f4").tobytes())
        f.write(p.astype("<f4").tobytes())
        f.write(smag.astype("<f4").tobytes())
        f.write(cp.astype("<f4").tobytes())
        f.write(ids.astype("<i4").tobytes())


def read_surface_pressure_bin(path: str) -> dict:
    """Parse a file written by write_surface_pressure_bin."""
    raw = open(path, "rb").read()
    if raw[:4] != LBMP_MAGIC:
        raise ValueError("not an LBMP file")
    version, n, n_obj = np.frombuffer(raw, "<u4", 3, 4)
    pos = 16
    names = []
    for _ in range(int(n_obj)):
        (ln,) = np.frombuffer(raw, "<u4", 1, pos)
        pos += 4
        names.append(raw[pos:pos + int(ln)].decode("utf-8"))
        pos += int(ln)
    n = int(n)

    def take(dt, count):
        nonlocal pos
        a = np.frombuffer(raw, dt, count, pos)
        pos += a.nbytes
        return a

    out = dict(version=int(version), names=names, vertices=take("<f4", 9 * n).reshape(n, 9),
               normals=take("<f4", 3 * n).reshape(n, 3), pressure=take("<f4", n),
               shear=take("<f4", n), cp=take("<f4", n), object_id=take("<i4", n))
    if pos != len(raw):
        raise ValueError("trailing bytes in LBMP file")
    return out


def inverse_rotation_f32(alpha_deg: float, beta_deg: float) -> np.ndarray:
    """R^T of the mesh rotation R = Rz(beta) Ry(alpha) as the Float32 entries
    forces/io.jl:186-195 builds (row-major)."""
    a, b = math.radians(alpha_deg), math.radians(beta_deg)
    ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
    return np.array([[ca * cb, -ca * sb, sa], [sb, cb, 0.0], [-sa * cb, sa * sb, ca]], np.float32)


def write_net_forces_csv(path: str, net: np.ndarray, centers: np.ndarray, offset=(0.0, 0.0, 0.0),
                         unrotated_centers: np.ndarray | None = None, alpha_deg: float = 0.0,
                         beta_deg: float = 0.0, object_names=None) -> None:
    """export_net_triangle_forces_csv (forces/io.jl:141-234).  `net` is the
    [3, n] Float32 net force per triangle, `centers` the solver-frame
    centroids [n, 3].  With unrotated_centers the positions are those
    (no offset) and the forces are rotated back by R^T in Float32 when a
    rotation angle is non-zero; otherwise centers + Float32(offset)."""
    fx, fy, fz = (np.asarray(net[i], np.float32) for i in range(3))
    n = fx.shape[0]
    if unrotated_centers is not None:
        c = np.asarray(unrotated_centers, np.float64).astype(np.float32)
        off = np.zeros(3, np.float32)
        if alpha_deg != 0.0 or beta_deg != 0.0:
            r = inverse_rotation_f32(alpha_deg, beta_deg)
            # Float32 r11*fx + r12*fy + r13*fz, summed left to right
            rx = (r[0, 0] * fx + r[0, 1] * fy) + r[0, 2] * fz
            ry = (r[1, 0] * fx + r[1, 1] * fy) + r[1, 2] * fz
            rz = (r[2, 0] * fx + r[2, 1] * fy) + r[2, 2] * fz
            fx, fy, fz = rx, ry, rz
    else:
        c = np.asarray(centers, np.float32)
        off = np.asarray([np.float32(v) for v in offset], np.float32)
    px, py, pz = c[:, 0] + off[0], c[:, 1] + off[1], c[:, 2] + off[2]
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w") as f:
        f.write(NET_FORCE_HEADER + "\n")
        for i in range(n):
            name = object_names[i] if object_names is not None else "default"
            f.write("%d,%s,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e\n" % (
                i + 1, name, px[i], py[i], pz[i], fx[i], fy[i], fz[i]))
