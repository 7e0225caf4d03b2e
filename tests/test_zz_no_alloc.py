"""The allocation-free iteration entry point (bowshock_solver_run_noalloc) against the existing one
(bowshock_solver_run): two solvers on the same case, two calls in a row each, the same states and residual histories
within the parity tolerance of the GPU tests; the size limit of its static scratch; no device memory allocated by it.

It is for hosts that set solvers up once and then step them from code that may not allocate device memory (the GPU's
free memory belongs to the host's own pool, or the loop cannot take an allocation's device synchronisation). Collected
last on purpose, so that a run that stops at the first failure has already run every other test; it passes alone in a
fresh process as well as after the other tests."""
import ctypes as C

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu


def _pair(spec):
    a = cases.gpu_solver(spec)
    b = cases.gpu_solver(spec)
    return a, b


@pytest.mark.parametrize("maker", [cases.subsonic_base, cases.g3_body])
def test_noalloc_matches_run_on_two_calls(maker):
    spec = maker(0.5) if maker is cases.subsonic_base else maker()
    a, b = _pair(spec)
    for call in range(2):
        ra = a.run(15)
        rb = b.run_noalloc(15)
        d = cases.state_diff(b.state_f64(), a.state_f64())
        assert d < 1e-5, f"call {call}: state diff {d:.3e}"
        assert cases.residual_diff(rb, ra) < 1e-4, f"call {call}: residuals {rb[:3]} vs {ra[:3]}"
        if spec.viscous is not None:
            ta, _ = a.turb_state()
            tb, _ = b.turb_state()
            fl = ta[:, 0] > 0
            assert np.max(np.abs(tb[fl] - ta[fl]) / np.abs(ta[fl])) < 1e-4


def test_noalloc_allocates_no_device_memory():
    import torch
    spec = cases.subsonic_base(0.5)
    s = cases.gpu_solver(spec)
    s.run_noalloc(2)  # first call on the device: module load and the scratch address lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    s.run_noalloc(20)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_rejects_a_solver_beyond_the_static_scratch():
    from bowshock_b200 import _ffi
    from bowshock_b200._ffi import BowshockError
    from tests.test_oracle_solver import curved_grid
    import oracle_ffi as o
    ni, nj = 512, 256  # 131,072 cells, 768 lines: 139 MB of line records
    assert 928 * ni * nj + 22528 * (ni + nj) > 64 << 20
    x, r = curved_grid(ni, nj)
    spec = cases.Spec(ni, nj, x, r, 0.5, o.MINMOD, tuple(o.freestream(0.5)),
                      (o.BC_CHARACTERISTIC, o.BC_CHARACTERISTIC, o.BC_SLIPWALL, o.BC_CHARACTERISTIC), 0, label="large")
    s = cases.gpu_solver(spec)
    with pytest.raises(BowshockError) as e:
        s.run_noalloc(1)
    assert e.value.status == _ffi.INVALID and "static maximum" in str(e.value)
