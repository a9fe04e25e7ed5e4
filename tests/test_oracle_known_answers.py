"""Known-answer checks that pin the oracle independently of itself.

The reference ships no tests, golden vectors or fixtures for this path (its
Julia toolchain is also absent here), so these come from the mathematics of
the method and from exact integer / IEEE arithmetic:
  * the inlet-noise hash against a hand-written uint32 evaluation,
  * binary16 rounding of q against numpy's IEEE conversion,
  * collision invariants: mass and momentum conservation of the cumulant and
    regularized-BGK collisions, rest state as a fixed point,
  * Bouzidi at q = 1/2 equals half-way bounce-back and at q = 1 the average,
  * restriction keeps equilibrium, mass and momentum,
  * two-sided net force on an open plate at rest vanishes; closed-body mode
    leaves -p n A.
"""
import numpy as np
import pytest

from helpers import lattice, perturbed_state, weights32
from oracle import oracle as orc


@pytest.fixture(scope="module", autouse=True)
def _build():
    orc.build()


def _hash(x):
    h = x & 0xFFFFFFFF
    h = ((h ^ (h >> 16)) * 0x85EBCA6B) & 0xFFFFFFFF
    h = ((h ^ (h >> 13)) * 0xC2B2AE35) & 0xFFFFFFFF
    return h ^ (h >> 16)


def test_noise_hash_matches_uint32_arithmetic():
    """physics_utils.jl:5-17 with Int32 wrap-around products."""
    for gy, gz, seed in [(1, 1, 1), (33, 17, 999999), (64, 64, 123456), (-5, 7, 0)]:
        comb = (gy * 374761393 + gz * 668265263 + seed * 1274126177 + 1234) & 0xFFFFFFFF
        expect = np.float32(np.float32(_hash(comb) & 0xFFFF) / np.float32(32768.0)) - np.float32(1.0)
        assert orc.gradient_noise(gy, gz, seed, 1234) == float(expect)


def test_half_rounding_matches_ieee():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(0, 1, 2000), [1e-8, 6e-8, 2.0 ** -25, 2.0 ** -24, 0.5, 1.0,
                                                   0.99951171875, 0.999755859375]])
    for x in xs:
        assert orc.double_to_half_bits(float(x)) == int(np.float64(x).astype(np.float16).view(np.uint16))
        h = int(np.float64(x).astype(np.float16).view(np.uint16))
        assert orc.half_to_float(h) == float(np.float16(np.float64(x)))


def _single_block_case():
    """One 8^3 block with every neighbour present as itself (a periodic cube)."""
    nbr = np.ones(27, dtype=np.int32)
    return dict(neighbor_table=nbr, map_x=np.array([2], np.int32), map_y=np.array([2], np.int32),
                map_z=np.array([2], np.int32), n_blocks=1,
                obstacle=np.zeros(512, np.uint8), sponge=np.zeros(512, np.float32),
                wall_dist=np.full(512, 100.0, np.float32))


def _params(op, **kw):
    p = dict(op=op, tau_molecular=0.52, tau_parent=0.5, c_wale=0.0, nu_sgs_background=0.0,
             is_level_1=1, is_symmetric=0, nx_global=100, ny_global=100, nz_global=100,
             u_inlet=0.05, wall_model_active=0, time_step_seed=1, store_post_collision=0,
             inlet_turbulence=0.0, temporal_weight=0.0, use_temporal_interp=0,
             sponge_blend_distributions=0, omega_bulk=1.0, omega_3=1.0, omega_4=1.0,
             adaptive_omega4=1, lambda_param=1.0 / 6.0, limiter_type=0, compressible_corr=0)
    p.update(kw)
    return p


@pytest.mark.parametrize("op", [0, 1])
def test_collision_conserves_mass_and_momentum(op):
    blk = _single_block_case()
    f_in, vel = perturbed_state(1, seed=11, amp=0.02)
    f_in = f_in.astype(np.float64)
    out = np.zeros_like(f_in)
    rho = np.zeros(512)
    vout = np.zeros(3 * 512)
    orc.stream_collide(dict(blk, f_out=out, f_in=f_in, rho=rho, vel_out=vout,
                            vel_in=vel.astype(np.float64)), None, _params(op), np.float64)
    cx, cy, cz = lattice()
    # pulled values (periodic block) -> per-cell sums before collision
    fi = f_in.reshape(27, 8, 8, 8)
    pulled = np.stack([np.roll(fi[k], shift=(cz[k], cy[k], cx[k]), axis=(0, 1, 2)) for k in range(27)])
    fo = out.reshape(27, 8, 8, 8)
    np.testing.assert_allclose(fo.sum(0), pulled.sum(0), rtol=0, atol=1e-13)
    for c in (cx, cy, cz):
        np.testing.assert_allclose((fo * c[:, None, None, None]).sum(0),
                                   (pulled * c[:, None, None, None]).sum(0), rtol=0, atol=1e-13)


@pytest.mark.parametrize("op", [0, 1])
def test_rest_state_is_fixed_point(op):
    blk = _single_block_case()
    cx, cy, cz = lattice()
    d2 = cx * cx + cy * cy + cz * cz
    w = np.where(d2 == 0, 8 / 27, np.where(d2 == 1, 2 / 27, np.where(d2 == 2, 1 / 54, 1 / 216)))
    f = np.repeat(w, 512)
    out = np.zeros_like(f)
    orc.stream_collide(dict(blk, f_out=out, f_in=f, rho=np.zeros(512), vel_out=np.zeros(1536),
                            vel_in=np.zeros(1536)), None, _params(op), np.float64)
    np.testing.assert_allclose(out, f, rtol=0, atol=1e-15)
    assert w.sum() == pytest.approx(1.0, abs=1e-15)
    assert weights32().astype(np.float64).sum() == pytest.approx(1.0, abs=1e-7)


@pytest.mark.parametrize("q,expect", [(0.5, "halfway"), (1.0, "average")])
def test_bouzidi_special_q(q, expect):
    nbr = np.ones(27, dtype=np.int32)
    rng = np.random.default_rng(5)
    f_post = rng.uniform(0.01, 0.1, 27 * 512).astype(np.float32)
    qmap = np.zeros(27 * 512, np.uint16)
    cell = 3 + 8 * 4 + 64 * 5
    k = 14  # (+1, 0, 0)
    qmap[cell + k * 512] = int(np.float16(q).view(np.uint16))
    f_out = f_post.copy()
    orc.bouzidi(f_out, f_post, qmap, np.array([1], np.int32), np.array([4], np.int8),
                np.array([5], np.int8), np.array([6], np.int8), nbr, 1, 0.001)
    ko = 26 - k
    got = f_out[cell + ko * 512]
    if expect == "halfway":
        assert got == f_post[cell + k * 512]
    else:
        assert got == pytest.approx(0.5 * f_post[cell + k * 512] + 0.5 * f_post[cell + ko * 512],
                                    rel=1e-6)
    changed = np.nonzero(f_out != f_post)[0]
    assert set(changed.tolist()) <= {cell + ko * 512}


def _restrict_setup(f_fine, dtype):
    """One parent block (coords 1,1,1) fully covered by two child blocks."""
    mx = np.array([1, 2], np.int32)
    my = np.array([1, 1], np.int32)
    mz = np.array([1, 1], np.int32)
    f_c = np.repeat(np.asarray(weights32(), dtype), 512).astype(dtype)
    rho_c = np.ones(512, dtype)
    vel_c = np.zeros(3 * 512, dtype)
    orc.restrict(f_fine, np.zeros(2 * 512, np.uint8), mx, my, mz, 2, f_c, rho_c, vel_c,
                 np.zeros(512, np.uint8), np.array([1], np.int32), (1, 1, 1), 1,
                 0.53, 0.56, 0, dtype)
    return f_c, rho_c, vel_c


def test_restriction_keeps_equilibrium_and_conserves_mass_momentum():
    """Fine-to-coarse restriction (opt-in extension): an equilibrium state is
    a fixed point, and the restricted cell keeps the children's mean mass and
    momentum (the non-equilibrium rescaling adds neither)."""
    cx, cy, cz = lattice()
    w = weights32().astype(np.float64)
    rho, ux, uy, uz = 1.02, 0.05, -0.01, 0.02
    cu = cx * ux + cy * uy + cz * uz
    feq = rho * w * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (ux * ux + uy * uy + uz * uz))
    f_c, rho_c, vel_c = _restrict_setup(np.repeat(feq, 2 * 512), np.float64)
    # the children cover parent cells x = 0..7, y = 0..3, z = 0..3
    covered = [x + 8 * y + 64 * z for z in range(4) for y in range(4) for x in range(8)]
    F_c = f_c.reshape(27, 512)
    for c in covered:
        np.testing.assert_allclose(F_c[:, c], feq, rtol=1e-12)
    untouched = 7 + 8 * 7 + 64 * 7
    np.testing.assert_array_equal(F_c[:, untouched], w)
    assert rho_c[0] == pytest.approx(feq.sum(), rel=1e-12)       # FP32 weights: sum != 1 exactly
    assert vel_c[0] == pytest.approx((feq * cx).sum() / feq.sum(), rel=1e-12)
    # random children: mean mass and momentum kept
    rng = np.random.default_rng(11)
    f_f = (np.repeat(w, 2 * 512) * rng.uniform(0.9, 1.1, 27 * 2 * 512)).astype(np.float64)
    f_c, rho_c, vel_c = _restrict_setup(f_f, np.float64)
    F = f_f.reshape(27, 2 * 512)
    for c in (0, 9, 63, 200, 511):
        x, y, z = c % 8, (c // 8) % 8, c // 64
        fb, lx = divmod(x, 4)
        kids = [fb * 512 + (2 * lx + a) + 8 * (2 * y % 8 + b) + 64 * (2 * z % 8 + d)
                for d in (0, 1) for b in (0, 1) for a in (0, 1)] if y < 4 and z < 4 else None
        if kids is None:
            continue
        mean = F[:, kids].mean(axis=1)
        got = f_c.reshape(27, 512)[:, c]
        assert got.sum() == pytest.approx(mean.sum(), rel=1e-12)
        assert (got * cx).sum() == pytest.approx((mean * cx).sum(), abs=1e-12)
        assert (got * cz).sum() == pytest.approx((mean * cz).sum(), abs=1e-12)


def test_net_forces_of_a_plate_at_rest():
    """Two-sided net force (surface.jl:511-700) on an open plate in fluid at
    rest with uniform density: both sides see the same pressure (up to the
    rounding of the fluid-weighted trilinear average) and no shear, so the
    open-surface net force vanishes per triangle, while the closed-body mode
    (minus side zero) leaves the one-sided -p n A."""
    import types
    from openludwig_b200 import domain, geometry as geo, scaling, solver as S, workloads
    c, _ = workloads.sphere_1lvl(8)
    c.alpha_deg = 15.0
    mesh = geo.rotate_mesh(geo.flat_plate(1.0, 8), 15.0, 0.0)
    p = scaling.compute_domain_from_mesh(c, mesh.min_bounds, mesh.max_bounds)
    h = domain.setup_multilevel_domain(c, mesh, p)[-1]
    fp = S.force_params_for(types.SimpleNamespace(host=h), p, c)
    a = np.stack([mesh.centers[:, 0], mesh.centers[:, 1], mesh.centers[:, 2], mesh.normals[:, 0],
                  mesh.normals[:, 1], mesh.normals[:, 2], mesh.areas]).astype(np.float32)
    rho = np.full(512 * h.n_blocks, 1.02, np.float32)
    vel = np.zeros(3 * 512 * h.n_blocks, np.float32)
    maps, net = orc.surface_net_forces(a, rho, vel, h.obstacle, h.block_ptr, h.n_blocks, fp,
                                       False)
    p0 = np.float32((np.float32(1.02) - np.float32(1)) / np.float32(3)) * np.float32(fp.pressure_scale)
    # every triangle found fluid on both sides
    np.testing.assert_allclose(maps[0], p0, rtol=5e-5)
    np.testing.assert_allclose(maps[4], p0, rtol=5e-5)
    assert not maps[1:4].any() and not maps[5:8].any()
    assert np.abs(net).max() <= 5e-5 * p0 * a[6].max()
    maps, net = orc.surface_net_forces(a, rho, vel, h.obstacle, h.block_ptr, h.n_blocks, fp,
                                       True)
    assert not maps[4:].any()
    expect = -p0 * a[3:6] * a[6]
    np.testing.assert_allclose(net, expect, rtol=5e-5, atol=5e-5 * p0 * a[6].max())
