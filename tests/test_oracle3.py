"""The 3D oracle (oracle/solver3.cpp) pinned by ports of the reference's own 3D unit tests: gas3.rs, bc3.rs, flux3.rs,
grid3.rs, implicit3.rs and solver3.rs (the cases without fins), with the reference's tolerances."""
import numpy as np
import pytest

import oracle_ffi as o


def _unit(rng):
    n = rng.uniform(-1, 1, 3)
    return n / np.linalg.norm(n)


def _state(rng, vmax):
    return np.array([rng.uniform(0.5, 2.0), *rng.uniform(-vmax, vmax, 3), rng.uniform(0.5, 2.0)])


def test_gas3_round_trip_and_flux_matches_2d_in_xz_plane():  # gas3.rs:59-90
    w = np.array([1.3, 0.7, -0.2, 0.4, 0.9])
    assert np.max(np.abs(o.cons_to_prim3(o.prim_to_cons3(w)) - w)) < 1e-14
    nx, nr = 0.6, 0.8
    w3 = np.array([1.2, 0.9, 0.0, -0.35, 0.7])
    f3 = o.physical_flux3(w3, [nx, 0.0, nr])
    f2 = o.physical_flux([w3[0], w3[1], w3[3], w3[4]], nx, nr)
    assert f3[2] == 0.0
    assert np.max(np.abs(f3[[0, 1, 3, 4]] - f2)) < 1e-14


def test_characteristic_ghost3_matches_2d_in_xz_plane():  # bc3.rs:85-116
    rng = np.random.default_rng(5)
    for it in range(2000):
        vmax = (0.3, 1.0, 3.0)[it % 3]
        t = rng.uniform(0, 2 * np.pi)
        nx, nr = np.cos(t), np.sin(t)
        w = _state(rng, vmax)
        w[2] = 0.0
        fs3 = o.freestream3(rng.uniform(0.3, 3.0), rng.uniform(-0.3, 0.3))
        g3 = o.characteristic_ghost3(fs3, w, [nx, 0.0, nr])
        g2 = np.asarray(o.characteristic_ghost([fs3[0], fs3[1], fs3[3], fs3[4]], [w[0], w[1], w[3], w[4]], nx, nr)[0])
        assert g3[2] == 0.0
        assert np.max(np.abs(g3[[0, 1, 3, 4]] - g2)) < 1e-12 * (1 + np.max(np.abs(g2)))


def _rot_x(phi):
    c, s = np.cos(phi), np.sin(phi)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])


def test_face_flux3_matches_2d_in_xz_plane_and_about_x():  # flux3.rs:261-393
    rng = np.random.default_rng(7)
    for it in range(400):
        lim = (o.FIRST_ORDER, o.MINMOD, o.VAN_ALBADA)[it % 3]
        low_mach = it % 2 == 1
        t = rng.uniform(0, 2 * np.pi)
        n2 = np.array([np.cos(t), np.sin(t)])
        st = []
        for _ in range(4):
            w = _state(rng, 1.5)
            w[2] = 0.0
            st.append(w)
        # face centroid in the x-z half plane (azimuth 0): the cylindrical frame is (radial = z, tangential = -y)
        f3 = o.face_flux3(*st, lim, [n2[0], 0.0, n2[1]], [0.0, 1.0], low_mach)
        f2 = o.face_flux_lm(*[[w[0], w[1], w[3], w[4]] for w in st], lim, n2[0], n2[1], low_mach)
        assert abs(f3[2]) < 1e-13
        assert np.max(np.abs(f3[[0, 1, 3, 4]] - f2)) < 1e-12 * (1 + np.max(np.abs(f2)))
        # rotation about x by phi: states, normal and face azimuth rotate together, the flux rotates with them
        phi = rng.uniform(-np.pi, np.pi)
        R = _rot_x(phi)
        rs = [np.concatenate([[w[0]], R @ w[1:4], [w[4]]]) for w in st]
        n3 = R @ np.array([n2[0], 0.0, n2[1]])
        c = R @ np.array([0.0, 0.0, 1.0])
        rot = [c[1], c[2]]
        g = o.face_flux3(*rs, lim, n3, rot, low_mach)
        assert abs(g[0] - f3[0]) < 1e-11 * (1 + abs(f3[0])) and abs(g[4] - f3[4]) < 1e-11 * (1 + abs(f3[4]))
        assert np.max(np.abs(g[1:4] - R @ f3[1:4])) < 1e-11 * (1 + np.max(np.abs(f3)))


def test_hllc3_consistency():  # flux3.rs:395-409
    rng = np.random.default_rng(11)
    for _ in range(200):
        w = _state(rng, 2.0)
        n = _unit(rng)
        assert np.max(np.abs(o.hllc3(w, w, n) - o.physical_flux3(w, n))) < 1e-13 * (1 + np.max(np.abs(o.physical_flux3(w, n))))


def test_flux_jacobian3_matches_finite_differences():  # implicit3.rs:497-518
    rng = np.random.default_rng(1)
    for _ in range(50):
        w = np.array([rng.uniform(0.5, 2.0), *rng.uniform(-1.5, 1.5, 3), rng.uniform(0.5, 2.0)])
        n = _unit(rng)
        a = o.flux_jacobian3(w, n)
        u0 = o.prim_to_cons3(w)
        for q in range(5):
            h = 1e-6
            up, um = u0.copy(), u0.copy()
            up[q] += h
            um[q] -= h
            fd = (o.physical_flux3(o.cons_to_prim3(up), n) - o.physical_flux3(o.cons_to_prim3(um), n)) / (2 * h)
            assert np.max(np.abs(fd - a[:, q])) < 1e-7


def test_abs_jacobian3_squares_to_a_squared_and_reflection():  # implicit3.rs:520-546
    rng = np.random.default_rng(2)
    for _ in range(50):
        w = np.array([rng.uniform(0.5, 2.0), rng.uniform(0.3, 1.5), *rng.uniform(-1.5, 1.5, 2), rng.uniform(0.5, 2.0)])
        n = _unit(rng)
        a = o.flux_jacobian3(w, n)
        ab = o.abs_jacobian3(w, w, n, 1e-3)
        a2, b2 = a @ a, ab @ ab
        assert np.all(np.abs(a2 - b2) < 1e-9 * (1 + np.abs(a2)))
    w = np.array([1.2, 0.5, -0.4, 0.9, 0.8])
    n = _unit(np.random.default_rng(3))
    got = o.reflection3(n) @ o.prim_to_cons3(w)
    un = w[1:4] @ n
    wr = np.concatenate([[w[0]], w[1:4] - 2 * un * n, [w[4]]])
    assert np.max(np.abs(got - o.prim_to_cons3(wr))) < 1e-14


def test_inv5_and_block_thomas5():  # implicit3.rs:548-600
    rng = np.random.default_rng(4)
    m = rng.uniform(-1, 1, (5, 5)) + 2.0 * np.eye(5)
    assert np.max(np.abs(o.inv5(m) @ m - np.eye(5))) < 1e-12
    n = 40
    lo, up = rng.uniform(-1, 1, (n, 5, 5)), rng.uniform(-1, 1, (n, 5, 5))
    d = rng.uniform(-1, 1, (n, 5, 5)) + 12.0 * np.eye(5)
    x = rng.uniform(-1, 1, (n, 5))
    rhs = np.array([d[k] @ x[k] + (lo[k] @ x[k - 1] if k > 0 else 0) + (up[k] @ x[k + 1] if k + 1 < n else 0) for k in range(n)])
    got = o.block_thomas5(lo.reshape(n, 25), d.reshape(n, 25), up.reshape(n, 25), rhs)
    assert np.max(np.abs(got - x)) < 1e-12


def _perturbed_unit_grid(ni, nj, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros((nj + 1, ni + 1))
    r = np.zeros((nj + 1, ni + 1))
    for j in range(nj + 1):
        for i in range(ni + 1):
            xx, rr = i / ni, j / nj
            if 0 < i < ni and 0 < j < nj:
                xx += 0.1 * (2 * rng.random() - 1) / ni
                rr += 0.1 * (2 * rng.random() - 1) / nj
            x[j, i], r[j, i] = xx, rr
    return x, r


def test_revolved_grid_volume_closure():  # grid3.rs:246-266
    ni, nj, nk = 8, 6, 24
    x, r = _perturbed_unit_grid(ni, nj, 3)
    theta = np.pi * np.arange(nk + 1) / nk
    s = o.Solver3(ni, nj, x, r, nk, theta, ni, 0.5, 0.0, implicit=False)
    for fam in range(3):
        n, a, c = s.faces(fam)
        assert np.all(np.isfinite(n)) and np.all(a >= 0)
    v = s.vol
    assert np.all(v >= -1e-14) and v.sum() > 0


@pytest.mark.parametrize("implicit", [False, True])
def test_freestream_is_preserved(implicit):  # solver3.rs:433-469
    ni, nj, nk = 8, 8, 8
    x, r = _perturbed_unit_grid(ni, nj, 0x12345678)
    k = np.arange(nk + 1) / nk
    theta = np.pi * (k - 0.06 * np.sin(2 * np.pi * k))
    fs = o.freestream3(0.8, np.radians(6.0))
    p = o.implicit3_params(cfl_max=20.0, growth=5.0)
    s = o.Solver3(ni, nj, x, r, nk, theta, ni, 0.8, np.radians(6.0), limiter=o.VAN_ALBADA, implicit=implicit, params=p)
    s.steps(1)
    assert np.max(np.abs(s.u - o.prim_to_cons3(fs))) <= 1e-12


def cone_like_grid(ni, nj, half_angle_deg=15.0):
    """An H-grid about a cone tip at x = 0 (axis upstream, x in [-0.5, 1]), the far boundary at r = 1 + x tan: a stand-in for
    the reference's `cone_grid` test grid. Returns (x, r, n_up)."""
    xs = np.linspace(-0.5, 1.0, ni + 1)
    t = np.tan(np.radians(half_angle_deg))
    rw = np.where(xs > 0, xs * t, 0.0)
    r_far = 1.0 + np.maximum(xs, 0) * t
    f = (np.arange(nj + 1) / nj) ** 1.5
    x = np.tile(xs, (nj + 1, 1))
    r = rw[None, :] + f[:, None] * (r_far - rw)[None, :]
    n_up = int(np.sum(xs[1:] <= 1e-12))
    return x, r, n_up


@pytest.mark.parametrize("implicit,lim,tol,tol_p", [(False, o.MINMOD, 1e-12, 1e-10), (True, o.MINMOD, 1e-9, 1e-10)])
def test_axisymmetric_flow_stays_axisymmetric(implicit, lim, tol, tol_p):  # solver3.rs:486-525
    ni, nj, nk = 32, 16, 8
    x, r, n_up = cone_like_grid(ni, nj)
    theta = np.pi * np.arange(nk + 1) / nk
    s = o.Solver3(ni, nj, x, r, nk, theta, n_up, 2.0, 0.0, limiter=lim, implicit=implicit, params=o.implicit3_params(cfl_max=20.0))
    s.steps(50)
    w = o.cons_to_prim3(s.u).reshape(nk, nj, ni, 5)
    xc = s.xc.reshape(nk, nj, ni, 3)
    th = np.arctan2(xc[..., 1], xc[..., 2])
    az = np.max(np.abs(w[..., 2] * np.cos(th) - w[..., 3] * np.sin(th)))
    dp = np.max(np.abs(w[..., 4] - w[0:1, :, :, 4]))
    assert az <= tol and dp <= tol_p, (az, dp)


def fin_grid():
    """solver3.rs:589-604 `fin_grid`: a rectangular 10 x 8 grid (x in [0, 2], r in [0, 1]) revolved over 8 cells of [0, pi],
    the whole j = 0 row on the axis, one solid box i 3..5, j 0..3, k 3..4."""
    ni, nj, nk = 10, 8, 8
    x = np.tile(2.0 * np.arange(ni + 1) / ni, (nj + 1, 1))
    r = np.tile((np.arange(nj + 1) / nj)[:, None], (1, ni + 1))
    theta = np.pi * np.arange(nk + 1) / nk
    return ni, nj, nk, x, r, theta, ((3, 5), (0, 3), (3, 4))


def _solid_mask(ni, nj, nk, box):
    m = np.zeros((nk, nj, ni), bool)
    (i0, i1), (j0, j1), (k0, k1) = box
    m[k0:k1, j0:j1, i0:i1] = True
    return m


def test_fin_wall_is_impermeable_and_the_run_converges():  # solver3.rs:606-670
    ni, nj, nk, x, r, theta, box = fin_grid()
    fs = o.freestream3(2.0, 0.0)
    s = o.Solver3(ni, nj, x, r, nk, theta, ni, 2.0, 0.0, limiter=o.VAN_ALBADA, first_order_iters=50, implicit=True,
                  params=o.implicit3_params(cfl_max=20.0))
    s.set_solid([box])
    res = s.steps(200)
    u = s.u
    assert np.all(np.isfinite(u))
    assert res[-1] <= 1e-2 * res.max(), (res.max(), res[-1])
    solid = _solid_mask(ni, nj, nk, box).reshape(-1)
    assert np.array_equal(u[solid], np.tile(o.prim_to_cons3(fs), (solid.sum(), 1)))  # solid cells untouched
    s.eval_residual()
    scale = fs[0] * fs[1]
    m = _solid_mask(ni, nj, nk, box)
    worst, nwall = 0.0, 0
    fi = s.face_fluxes(0).reshape(nk, nj, ni + 1, 5)
    fj = s.face_fluxes(1).reshape(nk, nj + 1, ni, 5)
    fk = s.face_fluxes(2).reshape(nk + 1, nj, ni, 5)
    pad = lambda a, ax: np.concatenate([np.zeros_like(np.take(a, [0], axis=ax)), a, np.zeros_like(np.take(a, [0], axis=ax))], axis=ax)
    for f, ax in ((fi, 2), (fj, 1), (fk, 0)):
        mp = pad(m, ax)
        lo, hi = np.take(mp, range(0, mp.shape[ax] - 1), axis=ax), np.take(mp, range(1, mp.shape[ax]), axis=ax)
        wall = lo != hi
        nwall += int(wall.sum())
        worst = max(worst, float(np.max(np.abs(f[..., 0][wall]))))
    assert nwall > 0 and worst <= 1e-14 * scale, (nwall, worst)
    # residual and time step vanish in the solid cells; the density norm is over the fluid cells
    assert np.all(s.res[solid] == 0.0) and np.all(s.dt[solid] == 0.0)


def test_fin_faces_carry_forces():
    """run3.rs:130-212: with the solid box the forces gain the pressure of every fluid-solid face; the sum over a box in a
    uniform stream at zero incidence has no normal force from the symmetric side faces (k faces at theta = 3 pi / 8 and
    pi / 2 are not mirror images, so only the axial part is checked against a direct sum)."""
    ni, nj, nk, x, r, theta, box = fin_grid()
    s = o.Solver3(ni, nj, x, r, nk, theta, 0, 2.0, 0.0, limiter=o.VAN_ALBADA, implicit=True, params=o.implicit3_params(cfl_max=20.0))
    s.set_solid([box])
    s.steps(5)
    f = s.forces(10.0)
    plain = o.Solver3(ni, nj, x, r, nk, theta, 0, 2.0, 0.0, limiter=o.VAN_ALBADA, implicit=True, params=o.implicit3_params(cfl_max=20.0))
    plain.u = s.u
    g = plain.forces(10.0)
    # direct sum of the fin faces' axial force: i faces between a fluid and a solid cell, first-cell extrapolation
    w = o.cons_to_prim3(s.u).reshape(nk, nj, ni, 5)
    n, a, c = s.faces(0)
    n, a, c = n.reshape(nk, nj, ni + 1, 3), a.reshape(nk, nj, ni + 1), c.reshape(nk, nj, ni + 1, 3)
    xc = s.xc.reshape(nk, nj, ni, 3)
    m = _solid_mask(ni, nj, nk, box)
    p_inf = 1.0 / 1.4
    fx = 0.0
    for k in range(nk):
        for j in range(nj):
            for i in range(1, ni):
                sa, sb = m[k, j, i - 1], m[k, j, i]
                if sa == sb:
                    continue
                ia, ib, sign = (i - 1, i - 2, 1.0) if not sa else (i, i + 1, -1.0)
                p0 = w[k, j, ia, 4]
                pw = p0
                if 0 <= ib < ni and not m[k, j, ib]:
                    d0 = np.linalg.norm(xc[k, j, ia] - c[k, j, i])
                    d1 = np.linalg.norm(xc[k, j, ib] - c[k, j, i])
                    pw = p0 + (p0 - w[k, j, ib, 4]) * d0 / (d1 - d0)
                fx += (pw - p_inf) * a[k, j, i] * sign * n[k, j, i, 0]
    # the k and j faces of the box have no x component on this grid, so the fin part of CA is the i faces' sum
    norm = 2.0 / (0.5 * 2.0 * 2.0 * np.pi / 4.0)
    assert abs((f["ca"] - g["ca"]) - norm * fx) <= 1e-12 * max(1.0, abs(norm * fx)), (f["ca"], g["ca"], norm * fx)
    assert abs(norm * fx) > 1e-3


def test_force_parts_sum_to_the_totals():
    """run3.rs `breakdown_on`: the five parts (nose, afterbody, fin sides, edges, tips) of the fin grid's forces add up to
    `forces_on`; the fin parts carry the solid box's faces (the k faces of a box in a uniform stream at zero incidence
    have no axial component)."""
    ni, nj, nk, x, r, theta, box = fin_grid()
    s = o.Solver3(ni, nj, x, r, nk, theta, 0, 2.0, np.radians(4.0), limiter=o.VAN_ALBADA, implicit=True,
                  params=o.implicit3_params(cfl_max=20.0))
    s.set_solid([box])
    s.steps(20)
    tot = s.forces(10.0)
    parts = s.forces_parts(10.0, 0.8)
    norm_sum = lambda key: sum(p[key] for p in parts.values())
    assert abs(norm_sum("cn") - tot["cn"]) <= 1e-12 * max(1.0, abs(tot["cn"]))
    assert abs(norm_sum("ca") - tot["ca"]) <= 1e-12 * max(1.0, abs(tot["ca"]))
    assert parts["fin_edges"]["ca"] != 0.0 and parts["fin_sides"]["ca"] == 0.0
    assert abs(parts["fin_sides"]["cn"]) > 0.0
