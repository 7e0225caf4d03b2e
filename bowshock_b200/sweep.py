"""The seeded mixed sweep of uneven cases that the batched metric is quoted on: 32 bodies drawn from a SplitMix64 stream
(seed 0x0B05C0C2), nose shape uniform over {cone, tangent ogive, von Karman}, nose fineness U[2,5], cylinder L/D U[5,15],
a boattail with probability 0.5 (length U[0.5,1.5] D, aft diameter U[0.7,0.9] D), Mach U[0.3,3.0], ISA altitude
U[0,10] km; even cases Euler on the sting grid (`Numerics::auto`), odd cases RANS k-omega SST with a base wake
(`Numerics::viscous`, wall-resolved first cell); grids from 96 x 48 to 320 x 160 cells scaled with the body length:
ni = even-round(96 + 224 (L/D - 7) / 14.5) clamped to [96, 320], nj = ni / 2. Nose diameter D = 0.10 m.

The per-case layout follows the reference's level-0 case (crates/bowshock-core/src/engine/case.rs:51-102), its cell
counts scaled to the requested ni x nj."""
from __future__ import annotations

import math

from .case import NOSE_CONE, NOSE_HAACK, NOSE_TANGENT_OGIVE, WAKE_BASE, WAKE_STING, Body, Case, Numerics, layer_count, rans_params

SEED = 0x0B05C0C2
D_NOSE = 0.10
MASK = (1 << 64) - 1


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014): the published 64-bit mixer, uniform doubles from the top 53 bits."""

    def __init__(self, seed: int):
        self.s = seed & MASK

    def next_u64(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))


def _even_round(x):
    return 2 * int(round(x / 2.0))


def _scale_counts(counts, total, minimum):
    """Scale a list of cell counts to sum to `total`, each at least `minimum`, the largest absorbing the rounding."""
    s = sum(counts)
    out = [max(minimum, int(round(c * total / s))) for c in counts]
    k = out.index(max(out))
    out[k] += total - sum(out)
    return out


def draw(n_cases=32, seed=SEED):
    """The drawn parameters of each case (draw order: shape, fineness, L/D, boattail?, length, aft diameter, Mach, altitude)."""
    g = SplitMix64(seed)
    out = []
    for k in range(n_cases):
        u = [g.uniform() for _ in range(8)]
        shape = (NOSE_CONE, NOSE_TANGENT_OGIVE, NOSE_HAACK)[min(int(u[0] * 3), 2)]
        out.append(dict(shape=shape, fineness=2.0 + 3.0 * u[1], cyl=5.0 + 10.0 * u[2], boattail=u[3] < 0.5, bt_len=0.5 + u[4],
                        bt_aft=0.7 + 0.2 * u[5], mach=0.3 + 2.7 * u[6], altitude=10000.0 * u[7], viscous=k % 2 == 1))
    return out


def body_of(p) -> Body:
    segs = [(p["cyl"], 0.0)]
    if p["boattail"]:
        segs.append((p["bt_len"], (0.5 * p["bt_aft"] - 0.5) / p["bt_len"]))
    if p["shape"] == NOSE_CONE:
        return Body(NOSE_CONE, fineness=p["fineness"], half_angle=math.atan(0.5 / p["fineness"]), segments=tuple(segs))
    return Body(p["shape"], fineness=p["fineness"], param=0.0, segments=tuple(segs))


def grid_size(body: Body):
    ld = body.x_base()
    ni = min(320, max(96, _even_round(96 + 224 * (ld - 7.0) / 14.5)))
    return ni, ni // 2


def make_case(p) -> Case:
    body = body_of(p)
    ni, nj = grid_size(body)
    if p["viscous"]:
        re_c, suth = rans_params(p["altitude"], D_NOSE)
        c = Case.viscous_case(p["mach"], body, 0, WAKE_BASE, re_c, suth, p["mach"])
        g = c.grid_base
        counts = _scale_counts([g.n_up, g.n_nose] + list(g.n_seg) + [g.n_wake], ni, 4)
        g.n_up, g.n_nose, g.n_seg, g.n_wake = counts[0], counts[1], counts[2:-1], counts[-1]
        if (g.n_up + g.n_nose + sum(g.n_seg)) % 2:  # even block index
            g.n_up += 1
            g.n_wake -= 1
        gap = max(4, _even_round(nj * g.n_gap / (g.n_gap + g.nj_out)))
        g.n_gap, g.nj_out = gap, nj - gap
        c.viscous.wall_i_start = g.n_up  # the no-slip wall starts at the nose tip (case.rs:96-97)
    else:
        c = Case.new(p["mach"], body, 0, WAKE_STING, Numerics.auto(p["mach"], 0, WAKE_STING))
        g = c.grid_sting
        counts = _scale_counts([g.n_up, g.n_nose] + list(g.n_seg) + [g.n_ext], ni, 4)
        g.n_up, g.n_nose, g.n_seg, g.n_ext = counts[0], counts[1], counts[2:-1], counts[-1]
        g.nj = nj
    assert c.cells() == (ni, nj), (c.cells(), ni, nj)
    return c


def sweep_cases(n_cases=32, seed=SEED):
    return [make_case(p) for p in draw(n_cases, seed)]
