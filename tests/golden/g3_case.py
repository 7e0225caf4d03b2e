"""The reference's G3 gate body (crates/bowshock-core/tests/viscous.rs:8-48; converged values quoted in
crates/bowshock-cfd/README.md:795-797): tangent ogive 0.30 x 0.10 m + 0.60 m tube, Mach 0.5, ISA sea level,
Resolution::Coarse (level 0), SST, base wake, as `Analysis::case` assembles it (analysis.rs:447-469, 592-614)."""
import oracle_ffi as o  # noqa: E402

D_NOSE = 0.10
MACH = 0.5
REFERENCE = dict(cd_total=0.21300, cd_friction=0.09003, cd_base=0.12257, cp_base=-0.1226, y_plus_max=0.648,
                 iters=4000, stop_reason="CD stationary")


def g3_case():
    air = o.isa(0.0)
    re_c = air["density"] * air["sound_speed"] * D_NOSE / air["viscosity"]
    sutherland = 110.4 / air["temperature_k"]
    b = o.body(o.NOSE_TANGENT_OGIVE, fineness=0.30 / D_NOSE, segments=((0.60 / D_NOSE, 0.0),))
    return o.case_viscous(MACH, b, 0, o.WAKE_BASE, re_c, sutherland, MACH)
