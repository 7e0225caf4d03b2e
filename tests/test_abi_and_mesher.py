"""CPU checks of the product library without a GPU: the C ABI loads and exports every entry point that
include/bowshock_b200.h declares, the library's FP64 mesher reproduces the oracle's restatement of the reference
mesher (body_grid.rs) bit for bit, and its host-side wall distance matches the oracle's."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle_ffi as o

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "bowshock_b200.h")).read()
    return sorted(set(re.findall(r"\b(bowshock_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    from bowshock_b200 import _ffi
    lib = _ffi.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _ffi.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in header_symbols():
        assert hasattr(lib, s)
    # and the Python binding binds every one of them
    assert set(header_symbols()) <= set(_ffi.SIGNATURES)


def _bodies():
    from bowshock_b200.case import Body
    yield Body(0, fineness=3.0, segments=((6.0, 0.0),)), o.body(o.NOSE_TANGENT_OGIVE, fineness=3.0, segments=((6.0, 0.0),))
    seg = ((6.0, 0.0), (1.0, -0.1))
    yield Body(0, fineness=3.0, segments=seg), o.body(o.NOSE_TANGENT_OGIVE, fineness=3.0, segments=seg)
    yield Body(4, fineness=4.2, param=0.0, segments=((9.0, 0.0),)), o.body(o.NOSE_HAACK, fineness=4.2, param=0.0, segments=((9.0, 0.0),))
    import math
    yield Body(1, half_angle=math.atan(0.5 / 2.5), segments=((7.0, 0.0),)), o.body(o.NOSE_CONE, half_angle=math.atan(0.5 / 2.5), segments=((7.0, 0.0),))


@pytest.mark.parametrize("wake", [0, 1])
@pytest.mark.parametrize("viscous", [False, True])
def test_mesher_matches_the_oracle_bit_for_bit(wake, viscous):
    from bowshock_b200.case import Case, rans_params
    re_c, suth = rans_params(0.0, 0.1)
    for pb, ob in _bodies():
        if viscous:
            pc = Case.viscous_case(0.9, pb, 0, wake, re_c, suth, 0.9)
            oc = o.case_viscous(0.9, ob, 0, wake, re_c, suth, 0.9)
        else:
            pc = Case.new(0.9, pb, 0, wake)
            oc = o.case_new(0.9, ob, 0, wake)
        ni, nj, x, r, blk = pc.grid()
        s = o.Solver.from_case(oc)
        assert (ni, nj) == s.dims == pc.cells()
        ox, orr = s.nodes
        assert np.array_equal(x, ox) and np.array_equal(r, orr)
        assert blk == s.block
        assert pc.config().first_order_iters == s.config.first_order_iters


@pytest.mark.parametrize("wake", [0, 1])
def test_wall_distance_matches_the_oracle(wake):
    """The arena's SST wall distance (bowshock_case_wall_distance, host only: the search over every no-slip segment with
    bounding-box skips) against the oracle's full search (turbulence.rs:91-125) on the viscous cases of the mesher
    test, sting and base wakes: equal bit for bit."""
    from bowshock_b200.case import Case, rans_params
    re_c, suth = rans_params(0.0, 0.1)
    for pb, ob in _bodies():
        pc = Case.viscous_case(0.9, pb, 0, wake, re_c, suth, 0.9)
        oc = o.case_viscous(0.9, ob, 0, wake, re_c, suth, 0.9)
        d = pc.wall_distance().ravel()
        ref = np.asarray(o.Solver.from_case(oc).dwall, dtype=float).ravel()
        fin = np.isfinite(ref)
        assert fin.any() and np.array_equal(np.isfinite(d), fin)
        assert np.array_equal(d[fin], ref[fin])  # bit for bit: the skips drop no minimum


def test_rans_params_match_the_oracle_atmosphere():
    from bowshock_b200.case import isa
    for h in (0.0, 3000.0, 11000.0, 15000.0):
        a, b = isa(h), o.isa(h)
        for k in a:
            assert abs(a[k] - b[k]) <= 1e-12 * abs(b[k])


def test_line_tuning_struct_matches_the_header():
    """The ctypes mirror of bowshock_line_tuning has the header's fields, in the header's order."""
    from bowshock_b200 import _ffi
    hdr = open(os.path.join(ROOT, "include", "bowshock_b200.h")).read()
    m = re.search(r"typedef struct \{\s*int32_t ([^;]*);\s*\} bowshock_line_tuning;", hdr)
    assert m, "bowshock_line_tuning not found in the header"
    names = [n.strip() for n in m.group(1).replace("\n", " ").split(",")]
    assert names == [n for n, _ in _ffi.LineTuning._fields_]


def test_limit_cycle_cd_comparison():
    """bench.py compares a case that both sides stopped on a limit cycle by the mean of the last compared window, any
    other case by its final total CD."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    ours = dict(stop_reason="mean stationary", cd_window=0.3200, cd_total=0.3210)
    assert abs(bench.cd_error(ours, dict(stop="mean stationary", cd_window=0.3199, cd_total=0.3190)) - 1e-4) < 1e-12
    assert abs(bench.cd_error(ours, dict(stop="CD stationary", cd_window=0.3199, cd_total=0.3190)) - 2e-3) < 1e-12


def test_mesh_dims_match_the_host_mesher():
    """bowshock_mesh_dims (the device mesher's sizes, from the cell counts) against the host mesher's grids, for every
    sweep case; and the host mesher's argument checks refuse the same requests."""
    from bowshock_b200 import BowshockError
    from bowshock_b200.sweep import sweep_cases
    for c in sweep_cases():
        ni, nj, x, r, blk = c.grid()
        assert c.mesh_dims() == (ni, nj, blk)
        assert (ni, nj) == c.cells()
    bad = sweep_cases()[0]
    bad.grid_sting.n_nose = 1
    bad.grid_base.n_nose = 1
    with pytest.raises(BowshockError):
        bad.mesh_dims()
