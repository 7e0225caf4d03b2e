"""The allocation-free iteration entry point (bowshock_solver_run_noalloc) against the existing one
(bowshock_solver_run): two solvers on the same case, two calls in a row each, bit-identical mean-flow and turbulence
states, residual histories and turbulence residuals to round-off; the size limit of its static scratch; no device memory
allocated by it.

It is for hosts that set solvers up once and then step them from code that may not allocate device memory (the GPU's
free memory belongs to the host's own pool, or the loop cannot take an allocation's device synchronisation). Both entry
points launch the same kernels in the same order (the graph of bowshock_solver_run replays them bit for bit), so the
states compare exactly; the FP64 residual norms are sums of per-block partial sums added atomically in whatever order
the blocks finish, so they compare to round-off (1e-12 relative). Collected last on purpose, so that a run that stops
at the first failure has already run every other test; it passes alone in a fresh process as well as after the other
tests."""
import os

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
        assert np.array_equal(b.state_f64(), a.state_f64()), f"call {call}: states differ"
        assert np.allclose(rb, ra, rtol=1e-12, atol=0.0), f"call {call}: residuals {rb[:3]} vs {ra[:3]}"
        if spec.viscous is not None:
            ta, ma = a.turb_state()
            tb, mb = b.turb_state()
            assert np.array_equal(tb, ta) and np.array_equal(mb, ma), f"call {call}: turbulence states differ"
            tra, trb = a.turb_residual(), b.turb_residual()
            assert tra > 0.0 and abs(trb - tra) <= 1e-12 * tra, f"call {call}: turbulence residuals {trb} vs {tra}"


def _process_device_bytes():
    """Device memory the driver attributes to this process (read-only NVML query), or None where NVML cannot say."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            idx = torch.cuda.current_device()
            uuid = torch.cuda.get_device_properties(idx).uuid
            h = None
            for k in range(pynvml.nvmlDeviceGetCount()):
                hk = pynvml.nvmlDeviceGetHandleByIndex(k)
                u = pynvml.nvmlDeviceGetUUID(hk)
                u = u.decode() if isinstance(u, bytes) else u
                if str(uuid) in u:
                    h = hk
            if h is None:
                return None
            for p in pynvml.nvmlDeviceGetComputeRunningProcesses(h):
                if p.pid == os.getpid() and p.usedGpuMemory is not None:
                    return int(p.usedGpuMemory)
            return None
        finally:
            pynvml.nvmlShutdown()
    except Exception:
        return None


def test_noalloc_allocates_no_device_memory():
    import torch
    spec = cases.subsonic_base(0.5)
    s = cases.gpu_solver(spec)
    s.run_noalloc(2)  # first call on the device: module load and the scratch address lookup
    torch.cuda.synchronize()
    reserved0 = torch.cuda.memory_reserved(0)
    proc0 = _process_device_bytes()
    # the device-wide free memory also moves with other processes' allocations on a shared GPU: a drop counts only if it
    # is seen on every one of three tries
    drops = 0
    for _ in range(3):
        free0, _ = torch.cuda.mem_get_info(0)
        s.run_noalloc(20)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        drops += free1 < free0
    assert drops < 3, "device free memory dropped across every allocation-free call"
    assert torch.cuda.memory_reserved(0) == reserved0
    proc1 = _process_device_bytes()
    if proc0 is not None and proc1 is not None:
        assert proc1 == proc0, f"this process's device memory grew from {proc0} to {proc1} bytes"


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
