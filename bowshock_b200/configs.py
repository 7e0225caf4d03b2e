"""The two single-case workloads of the path, as bowshock_b200 cases (the oracle's copies come from
tests/golden/sweep_oracle.oracle_case):

  config 0  Euler, tangent-ogive nose 0.30 m x 0.10 m + 0.60 m cylinder, base wake, Mach 1.5, ISA sea level, 128 x 64 cells
            (n_up 16, n_nose 32, n_seg [40], n_wake 40; n_gap 12, nj_out 52), far field at 10 body lengths, radial growth
            1.05 away from the body (dr_wall solved from the geometric series), the transonic numerics preset.
  config 1  RANS k-omega SST, the same body plus a 0.10 m boattail to 0.08 m, base wake, Mach 0.9, ISA sea level, wall cell
            from the reference's y+ ~ 1 rule, cell counts scaled to 256 x 128, the viscous numerics preset with the implicit
            CFL limit of its supersonic variant (20): with the subsonic limit of 50 the run diverges (non-finite residual
            near iteration 290) in the oracle and on the GPU alike, on this grid and on the case's own 180 x 126 grid."""
from dataclasses import replace

from .case import NOSE_TANGENT_OGIVE, WAKE_BASE, Body, Case, rans_params
from .sweep import _even_round, _scale_counts

D_NOSE = 0.10


def config0_case():
    body = Body(NOSE_TANGENT_OGIVE, fineness=0.30 / D_NOSE, segments=((0.60 / D_NOSE, 0.0),))
    c = Case.new(1.5, body, 0, WAKE_BASE)
    g = c.grid_base
    g.n_up, g.n_nose, g.n_seg, g.n_wake, g.n_gap, g.nj_out = 16, 32, [40], 40, 12, 52
    q, n = 1.05, g.nj_out
    g.dr_wall = (g.r_far - body.base_radius()) * (q - 1.0) / (q ** n - 1.0)
    assert c.cells() == (128, 64)
    return c


def config1_case():
    body = Body(NOSE_TANGENT_OGIVE, fineness=0.30 / D_NOSE, segments=((0.60 / D_NOSE, 0.0), (0.10 / D_NOSE, (0.04 - 0.05) / 0.10)))
    re_c, suth = rans_params(0.0, D_NOSE)
    c = Case.viscous_case(0.9, body, 0, WAKE_BASE, re_c, suth, 0.9)
    g = c.grid_base
    ni, nj = 256, 128
    counts = _scale_counts([g.n_up, g.n_nose] + list(g.n_seg) + [g.n_wake], ni, 4)
    g.n_up, g.n_nose, g.n_seg, g.n_wake = counts[0], counts[1], counts[2:-1], counts[-1]
    if (g.n_up + g.n_nose + sum(g.n_seg)) % 2:
        g.n_up += 1
        g.n_wake -= 1
    gap = max(4, _even_round(nj * g.n_gap / (g.n_gap + g.nj_out)))
    g.n_gap, g.nj_out = gap, nj - gap
    c.viscous.wall_i_start = g.n_up
    c.numerics.scheme = replace(c.numerics.scheme, cfl_max=20.0)
    assert c.cells() == (ni, nj)
    return c


CONFIGS = {"config0": config0_case, "config1": config1_case}
