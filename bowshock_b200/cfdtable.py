"""Result storage: the reference's solved-drag cache (`CfdTable`, crates/bowshock-model/src/cfd.rs:17-140) filled from this
backend's point results and written into, or read from, a `.bowshock` document, so that the app finds the tables it
would have solved itself.

  document   bytes 0..8 the magic `BOWSHOCK`, 8..10 the format version (u16, little-endian, 1), then the rocket serialised as
             CBOR (RFC 8949) and compressed as a raw deflate stream (crates/bowshock-model/src/format.rs:1-13, 86-96). The
             tables are the rocket map's `cfd` entry, an array of tables, absent while there are none (rocket.rs:132-134).
  table      a CBOR map with the fields of `CfdTable` in declaration order (serde's externally tagged encoding: unit enum
             variants as their names, `None` as null), the points as maps with the fields of `CfdPoint`.
  store      `Rocket::store_cfd_table` (cfd.rs:162-178): a table that is not sound (no points, Mach not ascending, a
             non-finite number) is refused; a stack keeps its latest table (its 3D solve carried over when the new one has
             none); at most 8 tables, the oldest dropped; loading drops unsound tables (cfd.rs:186-195).

The CBOR codec here is a small restatement of RFC 8949's encoding (major types 0-7; floats written as binary64, read at
any width), enough for the documents' maps, arrays, text, integers, floats, booleans and null."""
from __future__ import annotations

import math
import struct
import zlib
from dataclasses import asdict, dataclass, field

MAGIC = b"BOWSHOCK"
FORMAT_VERSION = 1
MAX_CFD_TABLES = 8


# ---------------------------------------------------------------------------------------------------- CBOR (RFC 8949)
class Tag:
    def __init__(self, tag, value):
        self.tag, self.value = tag, value

    def __eq__(self, o):
        return isinstance(o, Tag) and (self.tag, self.value) == (o.tag, o.value)


def _head(major, n):
    if n < 24:
        return bytes([major << 5 | n])
    for ai, fmt in ((24, ">B"), (25, ">H"), (26, ">I"), (27, ">Q")):
        if n < 1 << (8 * struct.calcsize(fmt)):
            return bytes([major << 5 | ai]) + struct.pack(fmt, n)
    raise ValueError("integer too large for CBOR")


def dumps(v) -> bytes:
    """CBOR encoding of None, bool, int, float, str, bytes, list/tuple, dict (keys in insertion order), Tag."""
    if v is None:
        return b"\xf6"
    if v is True:
        return b"\xf5"
    if v is False:
        return b"\xf4"
    if isinstance(v, int):
        return _head(0, v) if v >= 0 else _head(1, -1 - v)
    if isinstance(v, float):
        return b"\xfb" + struct.pack(">d", v)
    if isinstance(v, str):
        b = v.encode("utf-8")
        return _head(3, len(b)) + b
    if isinstance(v, (bytes, bytearray)):
        return _head(2, len(v)) + bytes(v)
    if isinstance(v, (list, tuple)):
        return _head(4, len(v)) + b"".join(dumps(x) for x in v)
    if isinstance(v, dict):
        return _head(5, len(v)) + b"".join(dumps(k) + dumps(x) for k, x in v.items())
    if isinstance(v, Tag):
        return _head(6, v.tag) + dumps(v.value)
    raise TypeError(f"cannot encode {type(v).__name__} as CBOR")


def _half(h):
    e, m = (h >> 10) & 0x1F, h & 0x3FF
    val = math.ldexp(m, -24) if e == 0 else (math.inf if m == 0 else math.nan) if e == 31 else math.ldexp(m + 1024, e - 25)
    return -val if h & 0x8000 else val


def _decode(b, i):
    ib = b[i]
    major, ai = ib >> 5, ib & 0x1F
    i += 1
    if major == 7:
        if ai == 20:
            return False, i
        if ai == 21:
            return True, i
        if ai in (22, 23):
            return None, i
        if ai == 25:
            return _half(struct.unpack_from(">H", b, i)[0]), i + 2
        if ai == 26:
            return struct.unpack_from(">f", b, i)[0], i + 4
        if ai == 27:
            return struct.unpack_from(">d", b, i)[0], i + 8
        if ai < 24:
            return ai, i  # simple value
        raise ValueError(f"unsupported CBOR simple value {ai}")
    if ai < 24:
        n = ai
    elif ai in (24, 25, 26, 27):
        size = 1 << (ai - 24)
        n = int.from_bytes(b[i:i + size], "big")
        i += size
    elif ai == 31 and major in (2, 3, 4, 5):
        n = None  # indefinite length
    else:
        raise ValueError(f"malformed CBOR head {ib:#x}")
    if major == 0:
        return n, i
    if major == 1:
        return -1 - n, i
    if major in (2, 3):
        if n is None:
            parts = []
            while b[i] != 0xFF:
                p, i = _decode(b, i)
                parts.append(p)
            i += 1
            return ("" if major == 3 else b"").join(parts), i
        raw = bytes(b[i:i + n])
        return (raw.decode("utf-8") if major == 3 else raw), i + n
    if major == 4:
        out = []
        while (n is None and b[i] != 0xFF) or (n is not None and len(out) < n):
            x, i = _decode(b, i)
            out.append(x)
        return out, i + (1 if n is None else 0)
    if major == 5:
        d = {}
        while (n is None and b[i] != 0xFF) or (n is not None and len(d) < n):
            k, i = _decode(b, i)
            x, i = _decode(b, i)
            d[k] = x
        return d, i + (1 if n is None else 0)
    if major == 6:
        x, i = _decode(b, i)
        return Tag(n, x), i
    raise ValueError("unreachable")


def loads(b: bytes):
    v, i = _decode(memoryview(bytes(b)), 0)
    if i != len(b):
        raise ValueError(f"{len(b) - i} bytes after the CBOR item")
    return v


# ---------------------------------------------------------------------------------------------------- the tables
QUALITIES = ("Converged", "Stationary", "Stalled")  # cfd.rs:17-25 `CfdQuality`
GRIDS = ("Coarse", "Medium")  # cfd.rs:50-57 `CfdGrid`


@dataclass
class CfdPoint:  # cfd.rs:27-47
    mach: float
    cd: float
    friction: float
    pressure: float
    base: float
    fins: float
    other: float
    quality: str = "Converged"


@dataclass
class CfdLiftPoint:  # cfd.rs:59-72
    mach: float
    alpha_deg: float
    cn: float
    x_cp: float
    quality: str = "Converged"


@dataclass
class CfdLiftTable:  # cfd.rs:74-92
    key: int
    solved_at: int
    solve_seconds: float
    backend: str
    points: list
    notes: list = field(default_factory=list)

    def is_sound(self):  # cfd.rs:94-100
        return bool(self.points) and math.isfinite(self.solve_seconds) and all(
            all(math.isfinite(v) for v in (p.mach, p.alpha_deg, p.cn, p.x_cp)) for p in self.points)


@dataclass
class CfdTable:  # cfd.rs:102-131
    key: int
    geometry: int
    stage: int
    solved_at: int
    solve_seconds: float
    backend: str
    fallback: str | None
    altitude: float
    notes: list
    points: list
    grid: str = "Coarse"
    lift: CfdLiftTable | None = None

    def is_sound(self):  # cfd.rs:133-139
        finite = lambda p: all(math.isfinite(v) for v in (p.mach, p.cd, p.friction, p.pressure, p.base, p.fins, p.other))
        return (bool(self.points) and all(finite(p) for p in self.points)
                and all(a.mach < b.mach for a, b in zip(self.points, self.points[1:])) and math.isfinite(self.solve_seconds))

    def to_value(self):
        d = asdict(self)
        d["lift"] = None if self.lift is None else asdict(self.lift)
        return d

    @staticmethod
    def from_value(d):
        lift = d.get("lift")
        return CfdTable(key=int(d["key"]), geometry=int(d["geometry"]), stage=int(d["stage"]), solved_at=int(d["solved_at"]),
                        solve_seconds=float(d["solve_seconds"]), backend=d["backend"], fallback=d.get("fallback"),
                        altitude=float(d["altitude"]), notes=list(d.get("notes", [])),
                        points=[CfdPoint(**{k: (v if k == "quality" else float(v)) for k, v in p.items()}) for p in d["points"]],
                        grid=d.get("grid", "Coarse"),
                        lift=None if lift is None else CfdLiftTable(
                            key=int(lift["key"]), solved_at=int(lift["solved_at"]), solve_seconds=float(lift["solve_seconds"]),
                            backend=lift["backend"], notes=list(lift.get("notes", [])),
                            points=[CfdLiftPoint(**{k: (v if k == "quality" else float(v)) for k, v in p.items()})
                                    for p in lift["points"]]))


def quality_of(stop_reason: str) -> str:
    """A point's CfdQuality from its stop rule: residual drop -> Converged, a stationary rule -> Stationary, otherwise
    (the iteration cap) Stalled."""
    if stop_reason == "residual drop":
        return "Converged"
    if stop_reason in ("CD stationary", "mean stationary", "base pressure stationary"):
        return "Stationary"
    return "Stalled"


def table_from_results(machs, results, *, key, geometry, stage=1, altitude=0.0, solve_seconds=0.0, solved_at=0, grid="Coarse",
                       notes=(), backend="GPU (B200)", cd_scale=1.0):
    """A CfdTable of one stack from the point results of its Mach sweep (bowshock_b200's point dicts), ascending Mach.
    cd_scale converts the solver's coefficients (on the body's nose cross-section) to the vehicle's reference area. Fins
    and the parts the solver does not model are empirical in the reference (left at 0 here)."""
    pts = []
    for m, r in sorted(zip(machs, results), key=lambda t: t[0]):
        pressure = r["cd_nose"] + sum(r["cd_aft"])
        pts.append(CfdPoint(mach=float(m), cd=float(r["cd_total"]) * cd_scale, friction=float(r["cd_friction"]) * cd_scale,
                            pressure=float(pressure) * cd_scale, base=float(r["cd_base"]) * cd_scale, fins=0.0, other=0.0,
                            quality=quality_of(r["stop_reason"])))
    return CfdTable(key=int(key), geometry=int(geometry), stage=int(stage), solved_at=int(solved_at), solve_seconds=float(solve_seconds),
                    backend=backend, fallback=None, altitude=float(altitude), notes=list(notes), points=pts, grid=grid)


def store(tables, table: CfdTable):
    """Rocket::store_cfd_table (cfd.rs:162-178) on a list of tables; returns (tables, stored)."""
    if not table.is_sound():
        return list(tables), False
    if table.lift is None:
        old = next((t for t in tables if t.stage == table.stage), None)
        table.lift = old.lift if old is not None else None
    out = [t for t in tables if t.stage != table.stage] + [table]
    return out[max(0, len(out) - MAX_CFD_TABLES):], True


def repair(tables):
    """Rocket::repair_cfd (cfd.rs:186-195): unsound tables and 3D solves dropped, at most 8 kept."""
    out = [t for t in tables if t.is_sound()]
    for t in out:
        if t.lift is not None and not t.lift.is_sound():
            t.lift = None
    return out[max(0, len(out) - MAX_CFD_TABLES):]


# ---------------------------------------------------------------------------------------------------- documents
def read_document(data: bytes):
    """(rocket CBOR value, version) of a .bowshock file (format.rs:98-110)."""
    if len(data) < 10 or data[:8] != MAGIC:
        raise ValueError("not a Bowshock document")
    version = int.from_bytes(data[8:10], "little")
    if version != FORMAT_VERSION:
        raise ValueError(f"Bowshock format version {version} (this reader: {FORMAT_VERSION})")
    return loads(zlib.decompress(data[10:], wbits=-15)), version


def write_document(rocket) -> bytes:
    """A .bowshock file of a rocket CBOR value (format.rs:86-96)."""
    c = zlib.compressobj(9, zlib.DEFLATED, -15)
    return MAGIC + FORMAT_VERSION.to_bytes(2, "little") + c.compress(dumps(rocket)) + c.flush()


def tables_of(rocket):
    return repair([CfdTable.from_value(t) for t in rocket.get("cfd", [])])


def with_table(data: bytes, table: CfdTable) -> bytes:
    """The document `data` with `table` stored (the rest of the rocket untouched)."""
    rocket, _ = read_document(data)
    tables, ok = store(tables_of(rocket), table)
    if not ok:
        raise ValueError("the table is not sound (no points, Mach not ascending, or a non-finite number)")
    rocket = dict(rocket)
    rocket["cfd"] = [t.to_value() for t in tables]
    return write_document(rocket)
