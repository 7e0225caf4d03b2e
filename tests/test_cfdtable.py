"""Result storage (bowshock_b200/cfdtable.py), on the CPU: the CBOR codec against encodings from RFC 8949's appendix A,
the `.bowshock` envelope round trip, and the reference's table-store rules (crates/bowshock-model/src/cfd.rs:204-300:
a stack keeps its latest table, unsound tables are refused, at most eight are kept, the 3D solve survives a drag
re-solve, nothing is written while there is nothing to write)."""
import math

import pytest

from bowshock_b200 import cfdtable as ct

RFC_VECTORS = [  # (value, hex) from RFC 8949 appendix A (floats encoded there at binary64 width)
    (0, "00"), (1, "01"), (10, "0a"), (23, "17"), (24, "1818"), (100, "1864"), (1000, "1903e8"), (1000000, "1a000f4240"),
    (1000000000000, "1b000000e8d4a51000"), (18446744073709551615, "1bffffffffffffffff"), (-1, "20"), (-10, "29"), (-100, "3863"),
    (-1000, "3903e7"), (1.1, "fb3ff199999999999a"), (1.0e300, "fb7e37e43c8800759c"), (-4.1, "fbc010666666666666"),
    (False, "f4"), (True, "f5"), (None, "f6"), ("", "60"), ("a", "6161"), ("IETF", "6449455446"), ('"\\', "62225c"),
    ("ü", "62c3bc"), ("水", "63e6b0b4"), ([], "80"), ([1, 2, 3], "83010203"), ([1, [2, 3], [4, 5]], "8301820203820405"),
    ({}, "a0"), ({1: 2, 3: 4}, "a201020304"), ({"a": 1, "b": [2, 3]}, "a26161016162820203"), (["a", {"b": "c"}], "826161a161626163"),
    (b"\x01\x02\x03\x04", "4401020304"),
]
DECODE_ONLY = [  # narrower floats and indefinite lengths, read as the RFC gives them
    ("f90000", 0.0), ("f98000", -0.0), ("f93c00", 1.0), ("f93e00", 1.5), ("f97bff", 65504.0), ("fa47c35000", 100000.0),
    ("fa7f7fffff", 3.4028234663852886e38), ("f90001", 5.960464477539063e-8), ("f90400", 0.00006103515625), ("f9c400", -4.0),
    ("f97c00", math.inf), ("fa7f800000", math.inf), ("fbfff0000000000000", -math.inf), ("9fff", []),
    ("9f018202039f0405ffff", [1, [2, 3], [4, 5]]), ("bf61610161629f0203ffff", {"a": 1, "b": [2, 3]}), ("7f657374726561646d696e67ff", "streaming"),
]


@pytest.mark.parametrize("value,hexs", RFC_VECTORS)
def test_cbor_encodes_rfc_vectors(value, hexs):
    assert ct.dumps(value).hex() == hexs
    back = ct.loads(bytes.fromhex(hexs))
    assert back == value


@pytest.mark.parametrize("hexs,value", DECODE_ONLY)
def test_cbor_decodes_rfc_vectors(hexs, value):
    v = ct.loads(bytes.fromhex(hexs))
    assert v == value and (not isinstance(value, float) or math.copysign(1, v) == math.copysign(1, value))


def point(mach, cd=0.4):
    return ct.CfdPoint(mach=mach, cd=cd, friction=0.1, pressure=0.1, base=0.1, fins=0.1, other=0.0, quality="Converged")


def table(stage, key):
    return ct.CfdTable(key=key, geometry=7, stage=stage, solved_at=1_700_000_000, solve_seconds=12.5, backend="GPU (B200)",
                       fallback=None, altitude=120.0, notes=["note"], points=[point(0.3), point(0.9), point(2.0)])


def lift(key):
    p = lambda m, a: ct.CfdLiftPoint(mach=m, alpha_deg=a, cn=0.2, x_cp=1.0, quality="Converged")
    return ct.CfdLiftTable(key=key, solved_at=1_700_000_100, solve_seconds=90.0, backend="GPU (B200)", points=[p(0.5, 2.0), p(0.5, 6.0)])


def test_store_rules():
    ts, ok = ct.store([], table(1, 1))
    assert ok
    ts, _ = ct.store(ts, table(1, 2))
    ts, _ = ct.store(ts, table(2, 3))
    assert len(ts) == 2 and [t.key for t in ts if t.stage == 1] == [2]
    bad = table(1, 4)
    bad.points[1].mach = 0.2
    nan = table(1, 5)
    nan.points[0].cd = math.nan
    empty = table(1, 6)
    empty.points = []
    for t in (bad, nan, empty):
        ts2, ok = ct.store(ts, t)
        assert not ok and ts2 == ts
    for stage in range(1, 13):
        ts, _ = ct.store(ts, table(stage, stage))
    assert len(ts) == ct.MAX_CFD_TABLES and ts[-1].stage == 12


def test_the_3d_solve_survives_a_drag_re_solve():
    t = table(1, 1)
    t.lift = lift(9)
    ts, _ = ct.store([], t)
    ts, _ = ct.store(ts, table(1, 2))
    assert ts[0].key == 2 and ts[0].lift == lift(9)


def test_document_round_trip_keeps_the_rocket():
    rocket = {"name": "test", "designer": "", "parts": [{"id": 1, "kind": "nose"}], "next_id": 2, "flights": []}
    doc = ct.write_document(rocket)
    assert doc[:8] == b"BOWSHOCK" and doc[8:10] == b"\x01\x00"
    back, v = ct.read_document(doc)
    assert v == 1 and back == rocket and "cfd" not in back  # nothing written while there is nothing to write
    t = table(1, 42)
    t.lift = lift(3)
    doc2 = ct.with_table(doc, t)
    r2, _ = ct.read_document(doc2)
    assert {k: v for k, v in r2.items() if k != "cfd"} == rocket
    assert ct.tables_of(r2) == [t]
    with pytest.raises(ValueError):
        ct.read_document(b"NOTBOWSHOCK")


def test_table_from_point_results():
    res = [dict(cd_total=0.5, cd_friction=0.2, cd_nose=0.1, cd_aft=[0.05], cd_base=0.15, stop_reason=s)
           for s in ("residual drop", "CD stationary", "max iterations")]
    t = ct.table_from_results([2.0, 0.5, 1.2], res, key=1, geometry=2, cd_scale=2.0)
    assert [p.mach for p in t.points] == [0.5, 1.2, 2.0]
    assert [p.quality for p in t.points] == ["Stationary", "Stalled", "Converged"]
    assert t.points[0].cd == 1.0 and t.points[0].pressure == pytest.approx(0.3) and t.is_sound()
