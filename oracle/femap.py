"""Restatement of the FE load mapper's per-triangle algorithm
(PREPOST/map_forces_to_nodes.jl:143-231 and the accumulation loop :486-509)
over the grouped layout of openludwig_b200.fe_map.Grouped, in numpy FP64.

TEST INFRASTRUCTURE (see oracle.py).  Nearest nodes by a stable sort of the
squared distances (dx*dx + dy*dy + dz*dz, summed left to right); the
distribution f = pinv(A) b with numpy's SVD pseudo-inverse at the cut-off
LinearAlgebra.pinv uses by default (min(size(A)) * eps * sigma_max); nodal
sums in triangle order, as the reference's loop adds them.
"""
from __future__ import annotations

import numpy as np


def skew(r) -> np.ndarray:
    return np.array([[0.0, -r[2], r[1]], [r[2], 0.0, -r[0]], [-r[1], r[0], 0.0]])


def distribute_force(F, centroid, node_positions) -> np.ndarray:
    """map_forces_to_nodes.jl:190-231: k x 3 nodal forces."""
    P = np.asarray(node_positions, np.float64)
    k = P.shape[0]
    F = np.asarray(F, np.float64)
    if k == 1:
        return F.reshape(1, 3).copy()
    A = np.zeros((6, 3 * k))
    b = np.zeros(6)
    b[:3] = F
    for i in range(k):
        A[0, 3 * i] = A[1, 3 * i + 1] = A[2, 3 * i + 2] = 1.0
        A[3:6, 3 * i:3 * i + 3] = skew(P[i] - np.asarray(centroid, np.float64))
    f = np.linalg.pinv(A, rcond=min(A.shape) * np.finfo(np.float64).eps) @ b
    return f.reshape(k, 3)


def nearest(c, node_xyz, k) -> np.ndarray:
    d = node_xyz - np.asarray(c, np.float64)
    dist = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    return np.argsort(dist, kind="stable")[:k]


def map_grouped(node_xyz, tri_xyz, tri_force, node_begin, tri_begin):
    """Returns (tri_nodes [T, 3] with -1 unused, tri_node_force [T, 3, 3],
    nodal [N, 3], 0) -- the shape of fe_map.device_map's result."""
    N, T = node_xyz.shape[0], tri_xyz.shape[0]
    tn = np.full((T, 3), -1, np.int32)
    tf = np.zeros((T, 3, 3))
    nodal = np.zeros((N, 3))
    for o in range(len(node_begin) - 1):
        n0, n1 = int(node_begin[o]), int(node_begin[o + 1])
        if n1 == n0:
            continue
        k = min(3, n1 - n0)
        for t in range(int(tri_begin[o]), int(tri_begin[o + 1])):
            loc = nearest(tri_xyz[t], node_xyz[n0:n1], k)
            f = distribute_force(tri_force[t], tri_xyz[t], node_xyz[n0:n1][loc])
            for j, li in enumerate(loc):
                i = n0 + int(li)
                tn[t, j] = i
                tf[t, j] = f[j]
                nodal[i] += f[j]
    return tn, tf, nodal, 0
