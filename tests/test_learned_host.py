"""Host logic of the learned warm start, on the CPU: the normalized grid's cases and sections, the section-wise resampling
(identity on equal sections, exact on fields linear in each section's index coordinate, never mixing sections, so the
solid block never bleeds into the fluid), the channel encoding round trip, the coarse solid mask against the normalized
case's block, and the network inputs."""
import numpy as np
import pytest

from bowshock_b200 import learned as lw


def test_normalized_case_grid_and_block():
    ps = lw.draw_sst(6, lw.TRAIN_SEED)
    for p in ps:
        c = lw.normalized_case(p, max_iter=1000)
        assert c.cells() == (128, 64)
        si, sj = lw.sections(c)
        assert si == lw.NORM_I and sj == lw.NORM_J
        assert c.numerics.max_iter == 1000 and c.viscous is not None and c.viscous.wall_i_start == 16
    # different seeds draw different cases; the same seed the same ones
    assert lw.draw_sst(3, lw.TRAIN_SEED) == lw.draw_sst(3, lw.TRAIN_SEED)
    assert lw.draw_sst(3, lw.TRAIN_SEED)[0]["mach"] != lw.draw_sst(3, lw.HELD_OUT_SEED)[0]["mach"]


def test_resample_identity_and_linear_fields():
    rng = np.random.default_rng(0)
    secs = ((16, 28, 44, 40), (12, 52))
    f = rng.standard_normal((64, 128, 3))
    assert np.allclose(lw.resample(f, secs, secs), f)
    # a field linear in each section's cell index is reproduced exactly on a refined copy of the sections
    src, dst = ((4, 6), (3, 5)), ((8, 12), (6, 10))
    jj, ii = np.meshgrid(np.arange(8), np.arange(10), indexing="ij")
    lin = np.stack([2.0 * ii + 3.0 * jj], -1).astype(float)
    out = lw.resample(lin, src, dst)
    ci, _, _ = lw._axis_map(src[0], dst[0])
    cj, _, _ = lw._axis_map(src[1], dst[1])
    assert np.allclose(out[..., 0], 2.0 * ci[None, :] + 3.0 * cj[:, None])


def test_resample_keeps_sections_apart():
    # a field constant per (i section, j section) block stays constant per block after resampling
    src, dst = ((16, 28, 44, 40), (12, 52)), ((20, 30, 70, 40), (8, 40))
    f = np.zeros((64, 128, 1))
    i0 = np.cumsum((0,) + src[0])
    j0 = np.cumsum((0,) + src[1])
    for a in range(4):
        for b in range(2):
            f[j0[b]:j0[b + 1], i0[a]:i0[a + 1]] = 10 * a + b
    out = lw.resample(f, src, dst)
    o0, p0 = np.cumsum((0,) + dst[0]), np.cumsum((0,) + dst[1])
    for a in range(4):
        for b in range(2):
            assert np.all(out[p0[b]:p0[b + 1], o0[a]:o0[a + 1]] == 10 * a + b)


def test_encode_decode_round_trip():
    rng = np.random.default_rng(1)
    n, mach, re_c = 50, 1.3, 2.0e6
    rho = rng.uniform(0.3, 3.0, n)
    vx, vr = rng.uniform(-0.5, 2.0, n), rng.uniform(-0.5, 0.5, n)
    p = rng.uniform(0.2, 3.0, n)
    u = np.stack([rho, rho * vx, rho * vr, p / 0.4 + 0.5 * rho * (vx * vx + vr * vr)], -1)
    turb = np.stack([rng.uniform(1e-9, 1e-3, n), rng.uniform(1.0, 1e6, n)], -1)
    ch = lw.encode(u, turb, mach, re_c)
    u2, t2, mt = lw.decode(ch, mach, re_c)
    assert np.allclose(u2, u, rtol=1e-12) and np.allclose(t2, turb, rtol=1e-12)
    assert np.all(mt <= 1e5 / re_c + 1e-30) and np.all(mt > 0)


def test_coarse_mask_matches_the_block():
    c = lw.normalized_case(lw.draw_sst(1, lw.TRAIN_SEED)[0])
    ni, nj, x, r, blk = c.grid()
    i_end, j_end, j_sting = blk
    fine = np.ones((nj, ni), dtype=np.uint8)
    fine[:j_end, :i_end] = 0
    coarse = fine.reshape(32, 2, 64, 2).min(axis=(1, 3))
    assert np.array_equal(coarse, lw.coarse_mask())
    assert np.array_equal(fine.reshape(32, 2, 64, 2).max(axis=(1, 3)), lw.coarse_mask())  # no coarse cell straddles the block


def test_features_of_sweep_cases():
    from bowshock_b200.sweep import sweep_cases
    cs = [c for c in sweep_cases(32) if c.viscous is not None]
    F = np.stack([lw.features(c) for c in cs])
    assert F.shape == (16, 16) and np.all(np.isfinite(F))
    assert np.all(F[:, 14:] == 0) and np.all(F[:, :3].sum(1) == 1)
    assert np.all(np.abs(F[:, 3:14]) <= 4.0)
