"""The warm-start network's CPU oracle (oracle/net_oracle.py) pinned on its own: its analytic gradient of the masked loss
against central finite differences in float64 (every layer, weights and biases), the layer table's parameter count, and
the BF16 rounding helper against torch's BF16 conversion."""
import numpy as np
import pytest

import net_oracle as no


def _problem(seed=3, B=2):
    L, n = no.layers()
    rng = np.random.default_rng(seed)
    p = no.init_params(seed, L, n).astype(np.float64)
    for l in L:  # non-zero biases so that their gradients are exercised
        p[l["boff"]:l["boff"] + l["cout"]] = 0.05 * rng.standard_normal(l["cout"])
    x = rng.standard_normal((B, no.NET_IN))
    t = rng.standard_normal((B, no.NET_CELLS, no.NET_OUT))
    mask = (rng.random(no.NET_CELLS) > 0.2).astype(np.uint8)
    return L, n, p, x, t, mask


def test_layer_table_size():
    L, n = no.layers()
    assert len(L) == 11
    weights = sum(l["cout"] * l["kin"] + l["cout"] for l in L)
    assert weights == 1_841_168 and n >= weights and n % 8 == 0


def test_oracle_gradient_matches_finite_differences():
    L, n, p, x, t, mask = _problem()
    loss, g = no.loss_and_grad(p, x, t, mask, L)
    assert loss > 0
    rng = np.random.default_rng(11)
    picks = []
    for l in L:  # three weights and one bias of every layer
        picks += list(rng.integers(l["woff"], l["woff"] + l["cout"] * l["kin"], 3)) + [l["boff"] + int(rng.integers(0, l["cout"]))]
    for q in picks:
        h = 1e-6 * max(1.0, abs(p[q]))
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (no.loss_and_grad(pp, x, t, mask, L)[0] - no.loss_and_grad(pm, x, t, mask, L)[0]) / (2 * h)
        # round-off of the difference quotient: ~1e-16 x loss / h ~ 1e-10
        assert abs(fd - g[q]) <= 1e-4 * abs(fd) + 2e-9, f"param {q}: fd {fd:.6e} analytic {g[q]:.6e}"


def test_bf16_rounding_matches_torch():
    import torch
    a = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * 37.0
    ours = no.bf16_round(a)
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(ours, ref)
