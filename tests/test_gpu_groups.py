"""Case groups of the batched arena (bowshock_arena_set_case_groups): the active cases split into independent chains of
the chunk's CUDA graph give the states of the ungrouped graph bit for bit (every kernel of an iteration reads and
writes only its own cases' data), with all cases active and with a few left; the residual histories to the order of the
FP64 atomic block sums of the norm."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("groups", [2, 3])
def test_case_groups_give_the_ungrouped_states(groups):
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    cs = [sweep_cases(32)[k] for k in (0, 1, 2, 3, 6, 9)]  # Euler and SST, uneven grids
    out = []
    for g in (1, groups):
        a = Arena(cs)
        a.set_case_groups(g)
        r1 = a.run(100)
        a.set_active([1, 1, 0, 1, 0, 1])  # a few left, as in a census tail
        r2 = a.run(100)
        out.append((r1, r2, [a.state(k) for k in range(len(cs))], [a.turb_state(k)[0] for k in (1, 3, 5)]))
    (r1a, r2a, sa, ta), (r1b, r2b, sb, tb) = out
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    for x, y in zip(ta, tb):
        assert np.array_equal(x, y)
    for x, y in ((r1a, r1b), (r2a, r2b)):
        m = np.isfinite(x) & (x > 0)
        assert np.array_equal(np.isfinite(x), np.isfinite(y))
        assert np.max(np.abs(x[m] - y[m]) / x[m]) < 1e-12
