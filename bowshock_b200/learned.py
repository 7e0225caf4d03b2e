"""Learned warm start for the RANS k-omega SST cases: a conv decoder (bowshock_b200.net, tensor-core forward and
backward passes) predicts a coarse flowfield from the body's geometry, the Mach number and the Reynolds number; the
prediction is resampled onto the case's own grid and replaces the free-stream start of the solve. No counterpart in the
reference, whose only warm start is the previous Mach point's field (crates/bowshock-core/src/engine/run.rs:54-63,
analysis.rs:744-748: keep the state, skip the first-order start-up, measure the drop from the cold run's residual peak).

  data      SST cases drawn from the sweep's distribution (bowshock_b200.sweep.draw: nose shape, fineness, cylinder L/D,
            boattail, Mach U[0.3, 3.0], ISA altitude U[0, 10] km) from SplitMix64 seed TRAIN_SEED, each meshed on its own
            grid as the sweep's cases are (96 x 48 to 320 x 160) and solved by the batched arena to the reference's stop
            rules (iterations capped); the converged state and (k, omega) as 6 channels (log rho, u / M, v / M,
            log(p gamma), log(k / k_inf), log(omega / omega_inf)), resampled onto the normalized 128 x 64 base-wake grid
            (fixed section counts: 16 upstream, 28 nose, 44 body, 40 wake cells along the body; 12 base-gap and 52 outer
            cells across), averaged 2 x 2 to the 64 x 32 coarse level and standardized. Solves that end non-finite are
            left out.
  network   16 inputs (12 geometry parameters, Mach, log10 Re, 2 zeros) -> 6 channels at 64 x 32 (bowshock_b200.net).
  start     the prediction mapped section by section onto the case's grid (bilinear in each section's normalized index
            coordinate, so the nose, body, wake, gap and outer blocks of any cell counts line up), decoded to the
            conserved state and (k, omega, mu_t); the run then starts warm: no first-order phase, the drop measured from
            the cold run's residual peak r_ref.
  fallback  the free-stream (cold) start whenever the predicted field's first residual exceeds 10 x the cold start's
            first residual; and, as the reference keeps a warm result only when it converged or became stationary, a
            warm run that ends otherwise is solved again cold.
"""
from __future__ import annotations

import json
import math
import os
import time
from dataclasses import replace

import numpy as np

from .case import NOSE_CONE, NOSE_HAACK, NOSE_TANGENT_OGIVE, WAKE_BASE, Case, rans_params
from .net import H_OUT, NET_CELLS, NET_IN, NET_OUT, W_OUT, Net
from .sweep import D_NOSE, _scale_counts, body_of, draw

TRAIN_SEED = 0x0B057EA1
HELD_OUT_SEED = 0x0B057E57
GAMMA = 1.4
K_INF = 9e-9  # turbulence.rs:238 free-stream k (nondimensional)
FALLBACK_RATIO = 10.0
# the normalized base-wake grid and its coarse level: cell counts of the sections along i (upstream, nose, body, wake)
# and along j (base gap, outer)
NORM_I, NORM_J = (16, 28, 44, 40), (12, 52)
COARSE_I, COARSE_J = (8, 14, 22, 20), (6, 26)
HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "warmstart_sst.npz")


# ---------------------------------------------------------------------------------------------------- cases and inputs
def draw_sst(n, seed):
    """n SST cases' parameters from the sweep's distribution (its draw order; every case viscous)."""
    ps = draw(n, seed)
    for p in ps:
        p["viscous"] = True
    return ps


def sweep_case(p, max_iter=None) -> Case:
    """The SST case of parameters p on its own grid, sized as the sweep's cases are (bowshock_b200.sweep.make_case:
    96 x 48 to 320 x 160 with the body length, the wall cell from the reference's y+ ~ 1 rule)."""
    from .sweep import make_case
    c = make_case(dict(p, viscous=True))
    if max_iter is not None:
        c.numerics = replace(c.numerics, max_iter=int(max_iter))
    return c


def normalized_case(p, max_iter=None) -> Case:
    """The SST case of parameters p on the normalized 128 x 64 base-wake grid."""
    body = body_of(p)
    re_c, suth = rans_params(p["altitude"], D_NOSE)
    c = Case.viscous_case(p["mach"], body, 0, WAKE_BASE, re_c, suth, p["mach"])
    g = c.grid_base
    g.n_up, g.n_nose, g.n_wake = NORM_I[0], NORM_I[1], NORM_I[3]
    g.n_seg = _scale_counts(list(g.n_seg), NORM_I[2], 4) if len(g.n_seg) > 1 else [NORM_I[2]]
    g.n_gap, g.nj_out = NORM_J
    c.viscous.wall_i_start = g.n_up
    if max_iter is not None:
        c.numerics = replace(c.numerics, max_iter=int(max_iter))
    assert c.cells() == (sum(NORM_I), sum(NORM_J))
    return c


def sections(case: Case):
    """(i sections, j sections) of a base-wake case: upstream, nose, body, wake cells; base gap (with any sting rows),
    outer cells."""
    g = case.grid_base
    return (g.n_up, g.n_nose, int(sum(g.n_seg)), g.n_wake), (g.n_sting + g.n_gap, g.nj_out)


def features(case: Case) -> np.ndarray:
    """The network's 16 inputs of a case: nose shape (3, one-hot cone / tangent ogive / von Karman), nose length,
    cylinder length, boattail flag, boattail length, aft diameter, body length, base radius, nose fraction, boattail
    slope (12 geometry parameters, lengths in nose diameters, each scaled to about [-1, 1]), Mach, log10 Re, 2 zeros."""
    b = case.body
    segs = list(b.segments)
    bt = len(segs) > 1
    fin, cyl = b.nose_length(), segs[0][0]
    bt_len, bt_slope = (segs[1][0], segs[1][1]) if bt else (0.0, 0.0)
    L, rb = b.x_base(), b.base_radius()
    re_c = case.viscous.re_c if case.viscous is not None else rans_params(0.0, D_NOSE)[0]
    x = np.zeros(NET_IN, dtype=np.float32)
    x[0], x[1], x[2] = float(b.nose_kind == NOSE_CONE), float(b.nose_kind == NOSE_TANGENT_OGIVE), float(b.nose_kind == NOSE_HAACK)
    x[3] = (fin - 3.5) / 1.5
    x[4] = (cyl - 10.0) / 5.0
    x[5] = 1.0 if bt else -1.0
    x[6] = (bt_len - 1.0) / 0.5 if bt else 0.0
    x[7] = (2.0 * rb - 0.9) / 0.1
    x[8] = (L - 14.0) / 5.0
    x[9] = (rb - 0.45) / 0.05
    x[10] = (fin / L - 0.25) / 0.1
    x[11] = bt_slope / 0.15
    x[12] = (case.mach - 1.65) / 1.35
    x[13] = (math.log10(re_c) - 6.15) / 0.25
    return x


# ---------------------------------------------------------------------------------------------------- fields
def encode(u, turb, mach, re_c):
    """Conserved state u [n, 4] and (k, omega) [n, 2] -> the 6 channels [n, 6]."""
    u = np.asarray(u, dtype=np.float64).reshape(-1, 4)
    rho = np.maximum(u[:, 0], 1e-12)
    vx, vr = u[:, 1] / rho, u[:, 2] / rho
    p = np.maximum((GAMMA - 1.0) * (u[:, 3] - 0.5 * rho * (vx * vx + vr * vr)), 1e-12)
    w_inf = 1e-6 * re_c
    t = np.asarray(turb, dtype=np.float64).reshape(-1, 2)
    return np.stack([np.log(rho), vx / mach, vr / mach, np.log(p * GAMMA), np.log(np.maximum(t[:, 0], 1e-30) / K_INF),
                     np.log(np.maximum(t[:, 1], 1e-30) / w_inf)], axis=-1)


def decode(ch, mach, re_c):
    """6 channels [n, 6] -> conserved state [n, 4], (k, omega) [n, 2] and mu_t [n] (rho k / omega, capped at 1e5 / re_c
    as the SST update caps it)."""
    ch = np.asarray(ch, dtype=np.float64).reshape(-1, 6)
    rho = np.exp(np.clip(ch[:, 0], -6.0, 4.0))
    vx, vr = mach * ch[:, 1], mach * ch[:, 2]
    p = np.exp(np.clip(ch[:, 3], -8.0, 5.0)) / GAMMA
    u = np.stack([rho, rho * vx, rho * vr, p / (GAMMA - 1.0) + 0.5 * rho * (vx * vx + vr * vr)], axis=-1)
    w_inf = 1e-6 * re_c
    k = K_INF * np.exp(np.clip(ch[:, 4], -20.0, 30.0))
    om = w_inf * np.exp(np.clip(ch[:, 5], -20.0, 40.0))
    mu_t = np.minimum(rho * k / om, 1e5 / re_c)
    return u, np.stack([k, om], axis=-1), mu_t


def _axis_map(src, dst):
    """Continuous source cell coordinate of every destination cell centre, section by section (each section's normalized
    index coordinate kept), clamped inside the section; also each coordinate's section bounds."""
    c, lo, hi = [], [], []
    s0 = 0
    for ns, nd in zip(src, dst):
        f = (np.arange(nd) + 0.5) / nd
        c.append(np.clip(s0 + f * ns - 0.5, s0, s0 + ns - 1))
        lo.append(np.full(nd, s0))
        hi.append(np.full(nd, s0 + ns - 1))
        s0 += ns
    return np.concatenate(c), np.concatenate(lo), np.concatenate(hi)


def resample(field, src_sections, dst_sections):
    """field [nj, ni, C] on a grid of sections src -> [nj', ni', C] on sections dst (bilinear within sections)."""
    (si, sj), (di, dj) = src_sections, dst_sections
    ci, _, hi_i = _axis_map(si, di)
    cj, _, hi_j = _axis_map(sj, dj)
    i0 = np.floor(ci).astype(int)
    j0 = np.floor(cj).astype(int)
    i1, j1 = np.minimum(i0 + 1, hi_i), np.minimum(j0 + 1, hi_j)
    wi, wj = (ci - i0)[None, :, None], (cj - j0)[:, None, None]
    f = np.asarray(field)
    a = f[j0][:, i0] * (1 - wi) + f[j0][:, i1] * wi
    b = f[j1][:, i0] * (1 - wi) + f[j1][:, i1] * wi
    return a * (1 - wj) + b * wj


def coarse_mask():
    """Fluid cells of the 64 x 32 coarse level (the solid block: the nose and body sections below the base gap)."""
    m = np.ones((H_OUT, W_OUT), dtype=np.uint8)
    m[:COARSE_J[0], :sum(COARSE_I[:3])] = 0
    return m


def target_of(case: Case, u, turb):
    """Converged state of a case -> the 6 channels on the 64 x 32 coarse level [32, 64, 6] (unstandardized)."""
    ni, nj = case.cells()
    ch = encode(u, turb, case.mach, case.viscous.re_c).reshape(nj, ni, 6)
    fine = resample(ch, sections(case), (NORM_I, NORM_J))
    return fine.reshape(H_OUT, 2, W_OUT, 2, 6).mean(axis=(1, 3))


# ---------------------------------------------------------------------------------------------------- the model
class WarmStart:
    """The trained network with its channel statistics."""

    def __init__(self, params, mean, std, net: Net | None = None, device=0):
        self.net = net or Net(max_batch=64, device=device)
        self.net.set_params(params)
        self.mean, self.std = np.asarray(mean, np.float64), np.asarray(std, np.float64)

    @staticmethod
    def load(path=WEIGHTS, device=0):
        z = np.load(path)
        bits = z["params_bf16"].astype(np.uint32) << 16
        params = bits.view(np.float32).copy()
        return WarmStart(params, z["mean"], z["std"], device=device)

    def save(self, path=WEIGHTS, meta=None):
        p = self.net.params()
        bits = (np.ascontiguousarray(p).view(np.uint32) + 0x7FFF + ((p.view(np.uint32) >> 16) & 1)) >> 16  # BF16, ties to even
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez_compressed(path, params_bf16=bits.astype(np.uint16), mean=self.mean, std=self.std,
                            meta=json.dumps(meta or {}))

    def predict(self, cases):
        """Coarse channels [n, 32, 64, 6] (unstandardized) of every case."""
        x = np.stack([features(c) for c in cases])
        y = self.net.forward(x).astype(np.float64)
        return y * self.std + self.mean

    def start_fields(self, cases):
        """(u [n_cells, 4], turb [n_cells, 2], mu_t [n_cells]) on each case's own grid; solid cells at the free stream."""
        from .solver import freestream
        out = []
        for c, y in zip(cases, self.predict(cases)):
            ni, nj = c.cells()
            ch = resample(y, (COARSE_I, COARSE_J), sections(c)).reshape(-1, 6)
            u, t, mt = decode(ch, c.mach, c.viscous.re_c)
            g = c.grid_base
            solid = np.zeros((nj, ni), dtype=bool)
            solid[:g.n_sting + g.n_gap, :g.n_up + g.n_nose + int(sum(g.n_seg))] = True
            w = freestream(c.mach)
            q = np.array([w[0], w[0] * w[1], w[0] * w[2], w[3] / (GAMMA - 1.0) + 0.5 * w[0] * (w[1] ** 2 + w[2] ** 2)])
            u[solid.ravel()] = q
            t[solid.ravel()] = [K_INF, 1e-6 * c.viscous.re_c]
            mt[solid.ravel()] = 0.0
            out.append((u, t, mt))
        return out


ACCEPTED = ("residual drop", "CD stationary", "mean stationary", "base pressure stationary")


def warm_solve(arena, model: WarmStart, r_ref, cold_first, device=0):
    """Warm-start every case of `arena` (all SST) from the model and solve to the stop rules. r_ref[k]: the drop reference
    (a cold run's residual peak); cold_first[k]: the cold start's first residual (the fallback threshold's base). As the
    reference's sweep keeps a warm result only when it converged or became stationary and solves the point cold
    otherwise (analysis.rs:744-771), a warm run that ends non-finite or at the iteration cap is solved again from the
    free stream (in a second arena of those cases). Returns (results, fallback flags, first residuals of the predicted
    fields, indices re-solved cold, device seconds of the re-solve)."""
    from .arena import Arena
    fields = model.start_fields(arena.cases)
    for k, (u, t, mt) in enumerate(fields):
        arena.set_state(k, u)
        arena.set_turb(k, t, mt)
    first = arena.first_residuals([1] * arena.ncases)
    fallback = [bool(not np.isfinite(first[k]) or first[k] > FALLBACK_RATIO * cold_first[k]) for k in range(arena.ncases)]
    for k, c in enumerate(arena.cases):
        if fallback[k]:
            arena.set_run(k, c.numerics, warm=False)
        else:
            arena.set_run(k, c.numerics, warm=True, r_ref=float(r_ref[k]))
    res = arena.solve()
    redo = [k for k in range(arena.ncases) if not fallback[k] and res[k]["stop_reason"] not in ACCEPTED]
    redo_s = 0.0
    if redo:
        b = Arena([arena.cases[k] for k in redo], device=device)
        rr = b.solve()
        redo_s = b.last_solve_ms() / 1000.0
        for q, k in enumerate(redo):
            res[k] = rr[q]
        del b
    return res, fallback, first, redo, redo_s


def iters_to_drop(hist, r_ref, orders):
    """First iteration whose residual is `orders` decades below r_ref (None if never)."""
    hit = np.nonzero(np.asarray(hist) <= r_ref * 10.0 ** (-orders))[0]
    return int(hit[0]) + 1 if hit.size else None


def _cd(r):
    return r["cd_window"] if r["stop_reason"] == "mean stationary" else r["cd_total"]


# ---------------------------------------------------------------------------------------------------- pipeline
def generate(n, seed, max_iter, batch=250, device=0, log=print):
    """Solve n SST cases of the sweep's distribution on their own grids with the batched arena and resample each
    converged field onto the normalized grid's coarse level: (features [n', 16], coarse targets [n', 32, 64, 6], per-case
    results); the cases whose solve ended non-finite are left out (n' <= n)."""
    from .arena import Arena
    ps = draw_sst(n, seed)
    X, T, R = [], [], []
    for b0 in range(0, n, batch):
        cs = [sweep_case(p, max_iter) for p in ps[b0:b0 + batch]]
        t0 = time.perf_counter()
        a = Arena(cs, device=device)
        res = a.solve()
        for k, c in enumerate(cs):
            R.append({key: res[k][key] for key in ("iters", "stop_reason", "cd_total", "cd_window", "residual_peak")})
            if res[k]["stop_reason"] == "non-finite residual":
                continue  # a diverged solve is no training target
            t, _ = a.turb_state(k)
            tg = target_of(c, a.state(k), t)
            if not np.all(np.isfinite(tg)):
                continue
            T.append(tg)
            X.append(features(c))
        log(f"generated {b0 + len(cs)}/{n} ({time.perf_counter() - t0:.1f} s, device {a.last_solve_ms() / 1000:.1f} s)")
        del a
    return np.stack(X), np.stack(T), R


def standardize(T, mask):
    f = T[:, mask.astype(bool)]
    return f.mean(axis=(0, 1)), f.std(axis=(0, 1)) + 1e-6


def train(X, T, steps=3000, batch=64, lr=1e-3, seed=0, device=0, log=print):
    """Train a fresh network on (X, T): the learning rate held for 60 % of the steps, then 0.3x and 0.1x."""
    mask = coarse_mask()
    mean, std = standardize(T, mask)
    Tn = ((T - mean) / std) * mask[None, :, :, None]
    net = Net(max_batch=batch, device=device)
    net.set_params(init_params(seed, net.layout(), net.nparams))
    net.set_mask(mask)
    net.set_dataset(X, Tn.astype(np.float32))
    losses = []
    t_ms = 0.0
    for frac, scale in ((0.6, 1.0), (0.25, 0.3), (0.15, 0.1)):
        s = max(1, int(steps * frac))
        losses.append(net.train(s, batch, lr * scale, seed=seed + len(losses)))
        t_ms += net.last_train_ms()
        log(f"train: {s} steps at lr {lr * scale:.1e}: loss {losses[-1][:5].mean():.4e} -> {losses[-1][-20:].mean():.4e}")
    return WarmStart(net.params(), mean, std, net=net), np.concatenate(losses), t_ms


def init_params(seed, net_layout, n):
    """He-uniform initial weights for the leaky ReLU layers, a small output layer, zero biases, for the layer table of
    the CUDA network (bowshock_net_layout)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    for fc, cin, cout, H, W, up, act, woff, boff in net_layout:
        kin = cin if fc else 9 * cin
        gain = math.sqrt(2.0 / (1.0 + 0.1 ** 2)) if act else 0.1
        bound = gain * math.sqrt(3.0 / kin)
        p[woff:woff + cout * kin] = rng.uniform(-bound, bound, cout * kin).astype(np.float32)
    return p


def evaluate(model: WarmStart, n, seed, max_iter, device=0, log=print):
    """Held-out evaluation on n SST cases of the sweep's distribution (their own grids): each solved cold and then warm
    (from the model, with the fallback rule and the cold re-run of a warm run that does not converge) in one arena, both
    to the reference's stop rules (iterations capped at max_iter); the warm run's drop measured from the cold run's
    residual peak, as the reference's warm runs measure theirs (analysis.rs:744-748). Cases whose cold run ends
    non-finite have no reference to compare with and are counted apart."""
    from .arena import Arena
    ps = draw_sst(n, seed)
    cs = [sweep_case(p, max_iter) for p in ps]
    a = Arena(cs, device=device)
    t0 = time.perf_counter()
    cold = a.solve()
    cold_s = a.last_solve_ms() / 1000.0
    hist_c = [a.residual_history(k) for k in range(n)]
    ok = [k for k in range(n) if cold[k]["stop_reason"] != "non-finite residual"]
    T = {}
    for k in ok:
        t, _ = a.turb_state(k)
        T[k] = target_of(cs[k], a.state(k), t)
    r_ref = [r["residual_peak"] for r in cold]
    warm, fallback, first, redo, redo_s = warm_solve(a, model, r_ref, [h[0] for h in hist_c], device=device)
    warm_s = a.last_solve_ms() / 1000.0 + redo_s
    hist_w = [a.residual_history(k) for k in range(n)]
    warm_iters = [warm[k]["iters"] + (len(hist_w[k]) if k in redo else 0) for k in range(n)]  # a re-run pays for both runs
    log(f"held-out: cold {cold_s:.1f} s, warm {warm_s:.1f} s of device time ({time.perf_counter() - t0:.1f} s wall), "
        f"{len(ok)} of {n} cold runs finite, {len(redo)} warm runs re-solved cold")
    mask = coarse_mask().astype(bool)
    pred = model.predict([cs[k] for k in ok])
    held_loss = float(np.mean((((pred - np.stack([T[k] for k in ok])) / model.std) ** 2)[:, mask])) if ok else None
    rep = {"cases": n, "seed": hex(seed), "max_iter": max_iter, "cold_finite": len(ok), "fallbacks": int(sum(fallback)),
           "warm_resolved_cold": len(redo), "cold_device_s": cold_s, "warm_device_s": warm_s, "held_out_loss_standardized": held_loss,
           "first_residual_ratio_median": float(np.median([first[k] / hist_c[k][0] for k in ok])) if ok else None,
           "stop_cold": {}, "stop_warm": {}, "drop": {}}
    for k in ok:
        rep["stop_cold"][cold[k]["stop_reason"]] = rep["stop_cold"].get(cold[k]["stop_reason"], 0) + 1
        rep["stop_warm"][warm[k]["stop_reason"]] = rep["stop_warm"].get(warm[k]["stop_reason"], 0) + 1
    direct = [k for k in ok if k not in redo and not fallback[k]]
    for orders in (1, 2, 3, 4, 5):
        ic = {k: iters_to_drop(hist_c[k], r_ref[k], orders) for k in direct}
        iw = {k: iters_to_drop(hist_w[k], r_ref[k], orders) for k in direct}
        both = [k for k in direct if ic[k] is not None and iw[k] is not None]
        rep["drop"][str(orders)] = {"reached_cold": sum(v is not None for v in ic.values()), "reached_warm": sum(v is not None for v in iw.values()),
                                    "median_iters_cold": float(np.median([ic[k] for k in both])) if both else None,
                                    "median_iters_warm": float(np.median([iw[k] for k in both])) if both else None,
                                    "mean_ratio_warm_over_cold": float(np.mean([iw[k] / ic[k] for k in both])) if both else None}
    conv = [k for k in ok if cold[k]["stop_reason"] in ACCEPTED and warm[k]["stop_reason"] in ACCEPTED]
    dcd = [abs(_cd(warm[k]) - _cd(cold[k])) for k in conv]
    rep["converged_both"] = len(conv)
    rep["dcd_max"] = float(max(dcd)) if dcd else None
    rep["dcd_median"] = float(np.median(dcd)) if dcd else None
    rep["within_1e-4"] = int(sum(d <= 1e-4 for d in dcd))
    rep["iters_cold_total"] = int(sum(cold[k]["iters"] for k in ok))
    rep["iters_warm_total"] = int(sum(warm_iters[k] for k in ok))
    rep["per_case"] = [{"mach": ps[k]["mach"], "cold": [cold[k]["iters"], cold[k]["stop_reason"], _cd(cold[k])],
                        "warm": [warm_iters[k], warm[k]["stop_reason"], _cd(warm[k])], "fallback": fallback[k],
                        "resolved_cold": k in redo} for k in range(n)]
    return rep


def main():
    import argparse
    ap = argparse.ArgumentParser(description="train the warm-start network on solver-generated SST solutions and evaluate it")
    ap.add_argument("--train-cases", type=int, default=2000)
    ap.add_argument("--eval-cases", type=int, default=200)
    ap.add_argument("--max-iter", type=int, default=4000, help="iteration cap of the training solves")
    ap.add_argument("--eval-max-iter", type=int, default=8000)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--dataset", default=None, help="an .npz of (X, T) to train on instead of generating")
    ap.add_argument("--save-dataset", default=None)
    ap.add_argument("--eval-only", action="store_true", help="evaluate the committed network (--out) on the held-out cases, no training")
    args = ap.parse_args()
    rep = {}
    if args.eval_only:
        model = WarmStart.load(args.out)
        ev = evaluate(model, args.eval_cases, HELD_OUT_SEED, args.eval_max_iter)
        rep["held_out"] = ev
        print(json.dumps({k: v for k, v in ev.items() if k != "per_case"}), flush=True)
        if args.report:
            with open(args.report, "w") as f:
                json.dump(rep, f, indent=1)
        return
    t0 = time.perf_counter()
    if args.dataset:
        z = np.load(args.dataset)
        X, T = z["X"], z["T"]
    else:
        X, T, R = generate(args.train_cases, TRAIN_SEED, args.max_iter)
        rep["generation_wall_s"] = time.perf_counter() - t0
        stops = {}
        for r in R:
            stops[r["stop_reason"]] = stops.get(r["stop_reason"], 0) + 1
        rep["generation_stops"] = stops
        if args.save_dataset:
            np.savez_compressed(args.save_dataset, X=X, T=T.astype(np.float16))
    model, losses, train_ms = train(X, T, steps=args.steps, batch=args.batch, lr=args.lr)
    layout = model.net.layout()
    from .net import flops_per_sample
    fl = 3.0 * flops_per_sample(layout) * args.batch * args.steps  # forward + backward (two GEMMs per layer)
    rep.update({"train_samples": int(len(X)), "steps": args.steps, "batch": args.batch, "train_device_ms": train_ms,
                "train_ms_per_step": train_ms / args.steps, "train_tflops": fl / (train_ms / 1000.0) / 1e12,
                "loss_first": float(losses[:10].mean()), "loss_last": float(losses[-50:].mean()), "params": int(model.net.nparams)})
    model.save(args.out, meta={k: v for k, v in rep.items() if not isinstance(v, dict)})
    print(json.dumps({k: v for k, v in rep.items()}), flush=True)
    if args.eval_cases > 0:
        ev = evaluate(model, args.eval_cases, HELD_OUT_SEED, args.eval_max_iter)
        rep["held_out"] = ev
        print(json.dumps({k: v for k, v in ev.items() if k != "per_case"}), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
