"""The device mesher (bowshock_mesh_batch, csrc/mesher_dev.cu) against the host mesher it mirrors (csrc/mesher.cuh, bit
for bit the reference's body_grid.rs / grid.rs): nodes of every sweep grid and of every nose shape within 1e-13 relative
(they differ only where the device's tanh, tan, pow, acos and sin round differently from the host C library; 59 % of the
nodes are bit-identical), the FP64 metrics (grid.rs:65-119, restated here in numpy from the host nodes) within 1e-10
relative (3e-12 measured: the areas of the thin wall cells, differences of nearly equal products of node coordinates,
amplify the nodes' last-bit differences), and a
batched arena built from device grids converging to the same CDs as one built from host grids."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _metrics_np(ni, nj, x, r):
    """grid.rs:65-119 in numpy: i faces, j faces, cells (the reference's two-triangle split of every quad)."""
    X, R = x.reshape(nj + 1, ni + 1), r.reshape(nj + 1, ni + 1)
    dx, dr = X[1:, :] - X[:-1, :], R[1:, :] - R[:-1, :]
    ln = np.hypot(dx, dr)
    m = {"if_nx": dr / ln, "if_nr": -dx / ln, "if_len": ln, "if_rm": 0.5 * (R[:-1, :] + R[1:, :])}
    dx, dr = X[:, 1:] - X[:, :-1], R[:, 1:] - R[:, :-1]
    ln = np.hypot(dx, dr)
    m.update({"jf_nx": -dr / ln, "jf_nr": dx / ln, "jf_len": ln, "jf_rm": 0.5 * (R[:, :-1] + R[:, 1:])})
    p = [(X[:-1, :-1], R[:-1, :-1]), (X[:-1, 1:], R[:-1, 1:]), (X[1:, 1:], R[1:, 1:]), (X[1:, :-1], R[1:, :-1])]
    a = v = sx = sr = 0.0
    for t in ((0, 1, 2), (0, 2, 3)):
        (x0, r0), (x1, r1), (x2, r2) = (p[k] for k in t)
        at = 0.5 * ((x1 - x0) * (r2 - r0) - (x2 - x0) * (r1 - r0))
        cx, cr = (x0 + x1 + x2) / 3.0, (r0 + r1 + r2) / 3.0
        a, v, sx, sr = a + at, v + at * cr, sx + at * cx, sr + at * cr
    m.update({"area": a, "vol": v, "xc": sx / a, "rc": sr / a})
    return m


def _cases():
    from bowshock_b200.case import (NOSE_CONE, NOSE_HAACK, NOSE_PARABOLIC, NOSE_POWER, NOSE_TANGENT_OGIVE, WAKE_BASE, WAKE_STING, Body,
                                    Case)
    from bowshock_b200.configs import config0_case, config1_case
    from bowshock_b200.sweep import sweep_cases
    extra = []
    for nose, kw in ((NOSE_CONE, dict(half_angle=0.2)), (NOSE_POWER, dict(fineness=3.0, param=0.6)),
                     (NOSE_PARABOLIC, dict(fineness=2.5, param=0.75)), (NOSE_HAACK, dict(fineness=3.5, param=1.0 / 3.0)),
                     (NOSE_TANGENT_OGIVE, dict(fineness=3.0))):
        body = Body(nose, segments=((4.0, 0.0), (1.0, -0.1)), **kw)
        extra += [Case.new(1.3, body, 0, WAKE_BASE), Case.new(0.7, body, 1, WAKE_STING)]
    return list(sweep_cases()) + [config0_case(), config1_case()] + extra


def test_device_mesher_matches_the_host_mesher():
    from bowshock_b200.case import METRIC_NAMES, mesh_batch
    cases = _cases()
    grids, mets, ms = mesh_batch(cases)
    assert ms > 0
    same = total = 0
    worst_node = worst_met = 0.0
    for c, (ni, nj, x, r, blk), m in zip(cases, grids, mets):
        hni, hnj, hx, hr, hblk = c.grid()
        assert (ni, nj, blk) == (hni, hnj, hblk)
        scale = 1.0 + np.maximum(np.abs(hx), np.abs(hr))
        err = np.maximum(np.abs(x - hx), np.abs(r - hr)) / scale
        worst_node = max(worst_node, float(err.max()))
        same += int(np.sum((x == hx) & (r == hr)))
        total += x.size
        ref = _metrics_np(ni, nj, hx, hr)
        for name in METRIC_NAMES:
            e = np.abs(m[name] - ref[name]) / (np.abs(ref[name]) + 1e-300)
            if name in ("if_nx", "if_nr", "jf_nx", "jf_nr"):  # unit normals: relative to 1
                e = np.abs(m[name] - ref[name])
            worst_met = max(worst_met, float(e.max()))
    print(f"{len(cases)} grids, {total} nodes, {same / total:.4f} bit-identical, node err {worst_node:.2e}, metric err {worst_met:.2e}, "
          f"{ms:.2f} ms on the device")
    assert worst_node <= 1e-13
    assert worst_met <= 1e-10
    assert same >= 0.5 * total


def test_arena_on_device_grids_converges_like_host_grids():
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    cs = [sweep_cases()[k] for k in (2, 6, 12, 20)]  # Euler cases that stop on the residual drop
    host = Arena(cs).solve()
    dev = Arena(cs, device_mesh=True).solve()
    for h, d in zip(host, dev):
        print(h["iters"], d["iters"], h["stop_reason"], d["stop_reason"], f"{d['cd_total'] - h['cd_total']:.2e}")
        assert d["stop_reason"] == h["stop_reason"] == "residual drop"
        assert abs(d["iters"] - h["iters"]) <= 50
        assert abs(d["cd_total"] - h["cd_total"]) <= 1e-8
