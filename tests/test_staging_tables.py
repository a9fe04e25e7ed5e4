"""The static staging tables of the stream-collide kernels, checked on the
CPU against their definition (no GPU needed):

* every out-of-block pull (cell d, direction k whose source d - c_k leaves the
  8^3 block) appears exactly once in the loader table of the warp-specialised
  kernel, with the neighbour direction and the source cell the pull wraps to;
* the FP32 compute stage: each population plane k lands 32-byte aligned at
  k * P + pad + 8 c_y + 64 c_z inside its plane of P slots, each
  out-of-block value is written at its table slot k * P + pad + d - c_x, and
  every cell's pull k reads slot k * P + pad + t - c_x -- emulated for all
  27 x 512 pulls, each must read its own source value or its own
  out-of-block value;
* the face-halo velocity entries cover each of the 6 x 64 face cells once;
* the ghost pass's staging table (halo entries, ring positions, ring index
  of each entry) is consistent with the same pulls.
"""
import ctypes as C

import numpy as np
import pytest

from openludwig_b200 import _native as N

HALO = 3176


def _tables():
    sizes = (C.c_int32 * 4)()
    N.call("ol_staging_tables", None, 0, None, 0, sizes)
    nh, nw, plane, pad = sizes[:4]
    h = (C.c_uint32 * nh)()
    w = (C.c_uint32 * nw)()
    N.call("ol_staging_tables", h, nh, w, nw, sizes)
    return np.array(h, np.int64), np.array(w, np.int64), plane, pad


def _c(k):
    return k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1


@pytest.fixture(scope="module")
def tables():
    try:
        return _tables()
    except Exception as ex:  # pragma: no cover - library not built
        pytest.fail(f"staging tables unavailable: {ex}")


def test_loader_table_lists_every_out_of_block_pull_once(tables):
    _, w, plane, pad = tables
    seen = {}
    for i in range(HALO):
        e = int(w[i])
        k, dr, src, d = e & 31, (e >> 5) & 31, (e >> 10) & 511, e >> 19
        cx, cy, cz = _c(k)
        x, y, z = d % 8, (d // 8) % 8, d // 64
        sx, sy, sz = x - cx, y - cy, z - cz
        assert not (0 <= sx < 8 and 0 <= sy < 8 and 0 <= sz < 8)
        ox = -1 if sx < 0 else (1 if sx > 7 else 0)
        oy = -1 if sy < 0 else (1 if sy > 7 else 0)
        oz = -1 if sz < 0 else (1 if sz > 7 else 0)
        assert dr == (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)
        assert src == (sx % 8) + 8 * (sy % 8) + 64 * (sz % 8)
        assert (k, d) not in seen
        seen[(k, d)] = i
    want = sum(1 for k in range(27) for d in range(512)
               if not (0 <= d % 8 - _c(k)[0] < 8 and 0 <= (d // 8) % 8 - _c(k)[1] < 8
                       and 0 <= d // 64 - _c(k)[2] < 8))
    assert len(seen) == want == HALO


def test_fp32_stage_layout_delivers_every_pull(tables):
    _, w, plane, pad = tables
    assert (plane * 4) % 32 == 0 and (pad * 4) % 32 == 0
    rng = np.random.default_rng(0)
    land = rng.normal(size=(27, 512))
    S = np.full(27 * plane, np.nan)
    for k in range(27):
        cx, cy, cz = _c(k)
        start = k * plane + pad + 8 * cy + 64 * cz
        assert start >= k * plane and start + 512 <= (k + 1) * plane
        assert (start * 4) % 16 == 0                  # bulk-copy destination alignment
        S[start:start + 512] = land[k]
    marker = {}
    for i in range(HALO):
        e = int(w[i])
        k, d = e & 31, e >> 19
        slot = int(w[3176 + 384 + i])
        assert slot == k * plane + pad + d - _c(k)[0]
        assert k * plane <= slot < (k + 1) * plane
        marker[(k, d)] = 1e6 + i
        S[slot] = marker[(k, d)]
    for k in range(27):
        cx, cy, cz = _c(k)
        for t in range(512):
            v = S[k * plane + pad + t - cx]
            x, y, z = t % 8, (t // 8) % 8, t // 64
            if (k, t) in marker:
                assert v == marker[(k, t)]
            else:
                assert v == land[k][(x - cx) + 8 * (y - cy) + 64 * (z - cz)]


def test_face_halo_velocity_entries(tables):
    _, w, _, _ = tables
    faces = {}
    for j in range(384):
        e = int(w[HALO + j])
        dr, oc = e & 31, e >> 5
        dx, dy, dz = dr % 3 - 1, (dr // 3) % 3 - 1, dr // 9 - 1
        assert abs(dx) + abs(dy) + abs(dz) == 1
        x, y, z = oc % 8, (oc // 8) % 8, oc // 64
        on = {(-1, 0, 0): x == 0, (1, 0, 0): x == 7, (0, -1, 0): y == 0,
              (0, 1, 0): y == 7, (0, 0, -1): z == 0, (0, 0, 1): z == 7}[(dx, dy, dz)]
        assert on
        faces.setdefault(dr, set()).add(oc)
    assert len(faces) == 6 and all(len(v) == 64 for v in faces.values())


def test_ghost_staging_table_is_consistent(tables):
    h, _, _, _ = tables
    ring = [int(p) for p in h[HALO:HALO + 488]]
    assert len(set(ring)) == 488
    for p in ring:
        x, y, z = p % 10 - 1, (p // 10) % 10 - 1, p // 100 - 1
        assert not (0 <= x < 8 and 0 <= y < 8 and 0 <= z < 8)
    for i in range(HALO):
        e = int(h[i])
        k, dst = e & 31, e >> 19
        q = int(h[HALO + 488 + i])
        assert ring[q] == dst
        x, y, z = dst % 10 - 1, (dst // 10) % 10 - 1, dst // 100 - 1
        cx, cy, cz = _c(k)
        # the slot is the source of a pull of an in-block cell
        assert 0 <= x + cx < 8 and 0 <= y + cy < 8 and 0 <= z + cz < 8


def test_ghost_visit_order_weights_count_the_loader_table(tables):
    """The ghost pass visits blocks by their number of absent-neighbour pulls
    (solver.ghost_block_lists; native.cu orders the block pool's lists the
    same way): the per-direction weights are the loader table's counts of
    pulls from each neighbour, and a list is ordered largest first, ties by
    block id."""
    from openludwig_b200 import solver as S
    _, w, _, _ = tables
    counts = np.bincount((w[:HALO] >> 5) & 31, minlength=27)
    assert counts.tolist() == S._PULLS_FROM_NEIGHBOUR.tolist()

    class Lvl:  # four blocks in a row along x; the middle ones see more
        n_blocks = 4
        map_x, map_y, map_z = [1, 2, 3, 4], [1, 1, 1, 1], [1, 1, 1, 1]
    nbr = np.zeros((27, 4), np.int32)
    for b in range(4):
        nbr[13, b] = b + 1
        if b > 0:
            nbr[12, b] = b       # -x neighbour present
        if b < 3:
            nbr[14, b] = b + 2   # +x neighbour present
    Lvl.neighbor_table = nbr.reshape(-1)
    ghost, edge = S.ghost_block_lists(Lvl, (64, 8, 8))
    # every block misses 24 neighbours; the end blocks also miss the x face
    assert ghost.tolist() == [0, 3, 1, 2]
    # in a 64 x 8 x 8 domain the y / z neighbours are outside, and so is block
    # 0's -x neighbour (block 3's absent +x neighbour is inside)
    assert edge.tolist() == [0, 1, 2, 3]
