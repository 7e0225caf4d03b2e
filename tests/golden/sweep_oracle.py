"""TEST INFRASTRUCTURE. The oracle's `Case` for each case of the seeded 32-case sweep (bowshock_b200.sweep): the same body,
Mach number, viscous parameters, grid counts and numerics preset, built through the oracle's own case assembly
(case.rs:51-102 restated in oracle/engine.cpp) so that the oracle meshes and runs it independently of the CUDA library."""
import oracle_ffi as o


def oracle_case(c):
    """OrcCase of a bowshock_b200 Case of the sweep (body, Mach, wake, rescaled cell counts, viscous parameters)."""
    b = c.body
    ob = o.body(b.nose_kind, fineness=b.fineness, half_angle=b.half_angle, param=b.param, segments=b.segments,
                sting_radius=b.sting_radius)
    if c.viscous is not None:
        v = c.viscous
        oc = o.case_viscous(c.mach, ob, 0, c.wake, v.re_c, v.sutherland, c.mach)
        oc.wall_i_start = v.wall_i_start
    else:
        oc = o.case_new(c.mach, ob, 0, c.wake)
    g, og = c.grid_base, oc.grid_base
    og.n_up, og.n_nose, og.n_wake, og.n_sting, og.n_gap, og.nj_out = g.n_up, g.n_nose, g.n_wake, g.n_sting, g.n_gap, g.nj_out
    og.dr_wall, og.gap_one_sided = g.dr_wall, int(g.gap_one_sided)
    for k, n in enumerate(g.n_seg):
        og.n_seg[k] = n
    g, og = c.grid_sting, oc.grid_sting
    og.n_up, og.n_nose, og.n_ext, og.nj, og.dr_wall = g.n_up, g.n_nose, g.n_ext, g.nj, g.dr_wall
    for k, n in enumerate(g.n_seg):
        og.n_seg[k] = n
    n, on = c.numerics, oc.numerics
    if on.scheme.kind == o.SCHEME_IMPLICIT and n.scheme.cfl_max != on.scheme.cfl_max:  # a preset whose CFL limit was changed
        on.scheme.cfl_max = n.scheme.cfl_max
    assert (on.max_iter, on.first_order_iters, on.limiter, bool(on.low_mach)) == (n.max_iter, n.first_order_iters, n.limiter,
                                                                                  bool(n.low_mach))
    return oc
