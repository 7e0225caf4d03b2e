"""Pins of the oracle's point kernels: ports of the reference's own unit tests of flux.rs, bc.rs and implicit.rs.

Each test names the reference test it ports (crates/bowshock-cfd/src/<file>.rs:<line>) and keeps its tolerance.
"""
import math

import numpy as np
import pytest

import oracle_ffi as o

G = o.GAMMA


def test_hllc_consistency():  # flux.rs:248-262
    states = [[1.0, 2.0, 0.0, 1.0 / G], [0.3, -1.5, 0.7, 0.2], [2.5, 0.0, 0.0, 3.0], [1.2, 0.3, -2.4, 0.9], [0.9, 5.0, 3.0, 1.3]]
    for w in states:
        for k in range(16):
            a = 0.4 * k
            nr, nx = math.sin(a), math.cos(a)
            f = o.hllc(w, w, nx, nr)
            g = o.physical_flux(w, nx, nr)
            assert np.all(np.abs(f - g) <= 1e-13 * (1.0 + np.abs(g))), (w, a)


def test_hllc_resolves_stationary_contact():  # flux.rs:265-272
    f = o.hllc([1.0, 0.0, 0.0, 1.0], [0.125, 0.0, 0.0, 1.0], 1.0, 0.0)
    assert abs(f[0]) < 1e-14 and abs(f[3]) < 1e-14
    assert abs(f[1] - 1.0) < 1e-14 and abs(f[2]) < 1e-14


def test_limiters_are_consistent():  # flux.rs:275-281
    for lim in (o.MINMOD, o.VAN_ALBADA, o.VENKATAKRISHNAN):
        assert abs(o.limited_slope(0.7, 0.7, lim) - 0.7) < 1e-12
        assert o.limited_slope(1.0, -1.0, lim) == 0.0
    assert o.limited_slope(1.0, 3.0, o.MINMOD) == 1.0


def test_venkatakrishnan_properties():  # flux.rs:284-306
    v = lambda a, b: o.limited_slope(a, b, o.VENKATAKRISHNAN)
    assert v(1.0, -1.0) == 0.0 and v(-0.3, 2.0) == 0.0 and v(0.0, 1.0) == 0.0
    for a in (1e-3, 0.7, 40.0, -2.5):
        assert abs(v(a, a) - a) < 1e-12 * max(abs(a), 1.0)
    prev = 0.0
    for k in range(1, 400):
        r = k * 0.05
        s = v(r, 1.0)
        assert s <= 2.0 * min(r, 1.0) + 1e-12 and s <= 1.10 and (r > 1.0 or s >= prev - 1e-15)
        assert abs(s - 2.0 * r * (r + 1.0) / (2.0 * r * r + r + 1.0)) < 1e-9
        prev = s
    assert abs(v(-0.4, -1.3) + v(0.4, 1.3)) < 1e-15


def test_rusanov_consistency_and_shock_blend():  # flux.rs:309-328
    w = [0.9, 5.0, 3.0, 1.3]
    for k in range(8):
        nr, nx = math.sin(0.8 * k), math.cos(0.8 * k)
        f, g = o.rusanov(w, w, nx, nr), o.physical_flux(w, nx, nr)
        assert np.all(np.abs(f - g) <= 1e-13 * (1.0 + np.abs(g)))
    assert o.shock_weight(1.0, 1.0 + 0.5 * 0.002) == 0.0
    assert o.shock_weight(1.0, 1.5) == 1.0
    assert o.shock_weight(1.0, 1.0 + 0.5 * (0.002 + 0.02)) > 0.4
    a, b = [1.0, 2.0, 0.0, 0.7], [1.5, 1.7, 0.2, 1.0]
    f = o.face_flux(a, a, b, b, o.FIRST_ORDER, 1.0, 0.0)
    r = o.rusanov(a, b, 1.0, 0.0)
    assert np.all(np.abs(f - r) < 1e-14)


def test_low_mach_flux_is_consistent_and_reduces_to_the_standard_flux():  # flux.rs:331-349
    w = [1.1, 0.04, -0.02, 0.8]
    for k in range(8):
        nr, nx = math.sin(0.8 * k), math.cos(0.8 * k)
        f = o.face_flux_lm(w, w, w, w, o.VAN_ALBADA, nx, nr, True)
        g = o.physical_flux(w, nx, nr)
        assert np.all(np.abs(f - g) <= 1e-13 * (1.0 + np.abs(g)))
    a, b, c, d = [1.0, 0.1, 0.0, 0.7], [1.01, 0.12, 0.01, 0.71], [1.02, 0.15, 0.02, 0.72], [1.04, 0.2, 0.0, 0.73]
    assert np.array_equal(o.face_flux_lm(a, b, c, d, o.MINMOD, 0.6, 0.8, False), o.face_flux(a, b, c, d, o.MINMOD, 0.6, 0.8))
    l, r = [1.0, 1.3, 0.0, 0.714], [1.1, 1.5, 0.1, 0.8]
    lm, rm = o.low_mach_states(l, r, 1.0, 0.0)
    assert np.array_equal(lm, l) and np.array_equal(rm, r)
    assert np.array_equal(o.face_flux_lm(l, l, r, r, o.FIRST_ORDER, 1.0, 0.0, True), o.face_flux(l, l, r, r, o.FIRST_ORDER, 1.0, 0.0))


def test_low_mach_scaling_reduces_the_normal_velocity_jump_only():  # flux.rs:352-365
    l, r = [1.0, 0.12, 0.05, 0.714], [1.0, 0.08, 0.05, 0.714]
    lm, rm = o.low_mach_states(l, r, 1.0, 0.0)
    m_local = math.hypot(0.12, 0.05) / math.sqrt(G * 0.714)
    assert abs((rm[1] - lm[1]) - m_local * (0.08 - 0.12)) < 1e-14
    assert abs(0.5 * (lm[1] + rm[1]) - 0.10) < 1e-14
    assert (lm[0], lm[2], lm[3]) == (l[0], l[2], l[3]) and (rm[0], rm[2], rm[3]) == (r[0], r[2], r[3])
    a, b = [1.0, 1e-6, 0.0, 0.714], [1.0, -1e-6, 0.0, 0.714]
    am, bm = o.low_mach_states(a, b, 1.0, 0.0)
    assert abs((bm[1] - am[1]) - 0.05 * (-2e-6)) < 1e-18


def test_regime_selected_by_normal_mach():  # bc.rs:111-131
    mk = lambda u, v: [1.0, u, v, 1.0 / G]
    assert o.regime(mk(-1.5, 0), 1, 0) == o.regime(mk(-1.0, 0), 1, 0) == 0
    assert o.regime(mk(-0.5, 0), 1, 0) == 1
    assert o.regime(mk(0.5, 0), 1, 0) == o.regime(mk(0.0, 0), 1, 0) == 2
    assert o.regime(mk(1.0, 0), 1, 0) == o.regime(mk(2.0, 0), 1, 0) == 3
    assert o.regime(mk(0.5, 0), -1, 0) == 1 and o.regime(mk(2.0, 0), -1, 0) == 0
    assert o.regime(mk(3.0, 0), 0, 1) == 2
    nx, nr = 0.5, math.sqrt(3.0) / 2.0
    assert o.regime(mk(1.9, 0), nx, nr) == 2 and o.regime(mk(2.1, 0), nx, nr) == 3


def test_ghost_follows_regime():  # bc.rs:134-160
    fs = o.freestream(0.9)
    s = lambda w: w[3] / w[0] ** G
    c = lambda w: math.sqrt(G * w[3] / w[0])
    it = [1.3, 2.0, 0.1, 1.2]
    g, r = o.characteristic_ghost(fs, it, -1.0, 0.0)
    assert r == 0 and np.array_equal(g, fs)
    g, r = o.characteristic_ghost(fs, it, 1.0, 0.0)
    assert r == 3 and np.array_equal(g, it)
    it = [1.1, 0.4, 0.2, 0.8]
    g, r = o.characteristic_ghost(fs, it, 1.0, 0.0)
    assert r == 2 and abs(g[2] - it[2]) < 1e-14 and abs(s(g) - s(it)) < 1e-13
    g1 = G - 1.0
    assert abs(g[1] + 2 * c(g) / g1 - (it[1] + 2 * c(it) / g1)) < 1e-12
    assert abs(g[1] - 2 * c(g) / g1 - (fs[1] - 2 * c(fs) / g1)) < 1e-12
    g, r = o.characteristic_ghost(fs, it, -1.0, 0.0)
    assert r == 1 and abs(g[2] - fs[2]) < 1e-14 and abs(s(g) - s(fs)) < 1e-13


def test_freestream_is_a_fixed_point_for_any_normal():  # bc.rs:163-174
    for mach in (0.3, 0.5, 0.9, 0.98, 1.0, 1.1, 2.0):
        fs = o.freestream(mach)
        for k in range(16):
            a = 2 * math.pi * k / 16
            g, _ = o.characteristic_ghost(fs, fs, math.cos(a), math.sin(a))
            assert np.all(np.abs(g - fs) < 1e-13), (mach, a)


def test_pressure_outflow_sets_static_pressure_only_when_subsonic():  # bc.rs:177-183
    assert np.array_equal(o.pressure_outflow_ghost(0.7, [1.0, 0.5, 0.1, 0.9], 1.0, 0.0), [1.0, 0.5, 0.1, 0.7])
    it = [1.0, 1.5, 0.1, 0.9]
    assert np.array_equal(o.pressure_outflow_ghost(0.7, it, 1.0, 0.0), it)


def test_flux_jacobian_matches_finite_differences():  # implicit.rs:703-721
    w = [1.2, 0.7, -0.3, 0.9]
    for nx, nr in ((1.0, 0.0), (0.0, 1.0), (0.6, -0.8), (-0.28, 0.96)):
        a = o.flux_jacobian(w, nx, nr)
        u0 = o.prim_to_cons(w)
        for q in range(4):
            h = 1e-6
            up, um = u0.copy(), u0.copy()
            up[q] += h
            um[q] -= h
            fd = (o.physical_flux(o.cons_to_prim(up), nx, nr) - o.physical_flux(o.cons_to_prim(um), nx, nr)) / (2 * h)
            assert np.all(np.abs(fd - a[:, q]) < 1e-7)


def _lcg(seed):
    state = [seed]

    def rnd():
        state[0] = (state[0] * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        return (state[0] >> 33) / float(1 << 31) - 0.5

    return rnd


def test_block_solver_inverts_a_random_diagonally_dominant_system():  # implicit.rs:724-766
    n = 7
    rnd = _lcg(12345)

    def blocks(diag):
        m = np.array([0.3 * rnd() for _ in range(16)]).reshape(4, 4)
        m += diag * np.eye(4)
        return m

    lo = np.array([blocks(0.0) for _ in range(n)])
    d = np.array([blocks(3.0) for _ in range(n)])
    up = np.array([blocks(0.0) for _ in range(n)])
    rhs = np.array([[rnd(), rnd(), rnd(), rnd()] for _ in range(n)])
    x = o.block_thomas(lo.reshape(n, 16), d.reshape(n, 16), up.reshape(n, 16), rhs)
    for k in range(n):
        r = d[k] @ x[k]
        if k > 0:
            r += lo[k] @ x[k - 1]
        if k + 1 < n:
            r += up[k] @ x[k + 1]
        assert np.all(np.abs(r - rhs[k]) < 1e-12)


def test_abs_jacobian_squares_to_a_squared():  # implicit.rs:769-780
    w = [1.2, 0.5, -0.2, 0.9]
    for nx, nr in ((1.0, 0.0), (0.0, 1.0), (0.6, 0.8), (-0.8, 0.6)):
        a = o.flux_jacobian(w, nx, nr)
        ab = o.abs_jacobian(w, w, nx, nr, 0.1)
        assert np.all(np.abs(a @ a - ab @ ab) < 1e-10)


def test_inv4_inverts_with_pivoting():
    rnd = _lcg(7)
    m = np.array([rnd() for _ in range(16)]).reshape(4, 4)
    m[0, 0] = 0.0  # forces a row swap
    assert np.allclose(o.inv4(m) @ m, np.eye(4), atol=1e-12)


def test_aupoix_wall_limits():  # turbulence.rs:836-868
    nu, d, speed = 1e-6, 1e-4, 1.0
    smooth = 60.0 * nu / (0.075 * d * d)
    k_w, om_w, nut = o.aupoix_wall(nu, speed, d, 1e-9)
    assert (k_w, om_w, nut) == (0.0, smooth, 0.0)
    assert np.all(np.isfinite(o.aupoix_wall(nu, 0.0, d, 1e-3)))

    def ks_plus_of(ks):
        nt = o.aupoix_wall(nu, speed, d, ks)[2]
        return math.sqrt((nu + nt) * speed / d) * ks / nu

    lo, hi = 1e-4, 1e-2
    for _ in range(60):
        mid = math.sqrt(lo * hi)
        if ks_plus_of(mid) < 100.0:
            lo = mid
        else:
            hi = mid
    ks = math.sqrt(lo * hi)
    k_w, om_w, nut = o.aupoix_wall(nu, speed, d, ks)
    u2 = (nu + nut) * speed / d
    ks_plus = math.sqrt(u2) * ks / nu
    assert abs(ks_plus / 100.0 - 1.0) < 1e-6
    t = math.tanh(ks_plus / 125.0)
    k_plus = max(math.tanh((math.log10(ks_plus / 30.0) + 1.0 - t) * t), 0.0) / math.sqrt(0.09)
    om_plus = 300.0 / ks_plus**2 / math.tanh(15.0 / (4.0 * ks_plus)) + 191.0 / ks_plus * (1.0 - math.exp(-ks_plus / 250.0))
    assert abs(k_w / u2 / k_plus - 1.0) < 2e-2
    assert abs(om_w * nu / u2 / om_plus - 1.0) < 2e-2
    assert abs(nut - k_w / om_w) <= 1e-15 * nut and nut > 0.0 and om_w < smooth


def test_isa_sea_level_and_tropopause():  # atmosphere.rs:117-133
    s = o.isa(0.0)
    assert s["temperature_k"] == 288.15 and abs(s["pressure_pa"] - 101325.0) < 1e-6
    assert abs(s["density"] - 1.2250) < 1e-4 and abs(s["sound_speed"] - 340.29) < 0.01
    assert abs(s["viscosity"] - 1.789e-5) / 1.789e-5 < 0.005
    s = o.isa(11000.0)
    assert abs(s["temperature_k"] - 216.65) < 1e-9 and abs(s["pressure_pa"] - 22632.0) < 5.0
    with pytest.raises(ValueError):
        o.isa(-1.0)


def test_geometric_offsets_close_exactly():  # grid.rs:199-228
    v = o.geometric_offsets(0.01, 3.0, 20)
    assert v[0] == 0.0 and v[-1] == 3.0 and np.all(np.diff(v) > 0)
    q = np.diff(v)[1:-1] / np.diff(v)[:-2]
    assert np.allclose(q, q[0], rtol=1e-9)
