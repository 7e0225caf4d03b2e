"""Batched case arena: many cases with uneven grids in one set of launches, with per-case convergence masks
(include/bowshock_b200.h, `bowshock_arena_*`). No counterpart in the reference, which runs Mach points one at a time
(crates/bowshock-core/src/analysis.rs:727-797); each case's numerics are those of the single-case solver."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi
from ._ffi import BowshockError
from .solver import point_dict, forces_dict


class Arena:
    def __init__(self, cases, device=0, grids=None, device_mesh=False):
        """`cases`: list of case.Case; `grids`: optional precomputed (ni, nj, x, r, block) per case; `device_mesh`: build
        every grid and its metrics on the device (bowshock_arena_create_meshed) instead of on the host."""
        lib = _ffi.load()
        self.cases = list(cases)
        self._descs = (_ffi.CaseDesc * len(self.cases))()
        self._keep = []
        h = C.c_void_p()
        if device_mesh:
            qs = (_ffi.MeshRequest * len(self.cases))()
            for k, c in enumerate(self.cases):
                ni, nj, blk = c.mesh_dims()
                n = (ni + 1) * (nj + 1)
                # the descriptor wants node arrays of the right size; the arena ignores their values
                d = c.case_desc((ni, nj, np.zeros(n), np.zeros(n), blk))
                self._keep.append((d._x, d._r))
                self._descs[k] = d
                qs[k] = c.mesh_request()
            rc = lib.bowshock_arena_create_meshed(len(self.cases), self._descs, qs, device, C.byref(h))
            if rc:
                raise BowshockError(rc, "bowshock_arena_create_meshed failed (invalid case, or no usable CUDA device)")
            self._h = h
            self.ncases = len(self.cases)
            return
        for k, c in enumerate(self.cases):
            d = c.case_desc(grids[k] if grids is not None else None)
            self._keep.append((d._x, d._r))
            self._descs[k] = d
        rc = lib.bowshock_arena_create(len(self.cases), self._descs, device, C.byref(h))
        if rc:
            raise BowshockError(rc, "bowshock_arena_create failed (invalid case, or no usable CUDA device)")
        self._h = h
        self.ncases = len(self.cases)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _ffi.load().bowshock_arena_destroy(h)
            self._h = None

    def _check(self, rc):
        if rc:
            m = _ffi.load().bowshock_arena_last_error(self._h)
            raise BowshockError(rc, m.decode() if m else "")

    @property
    def cells(self) -> int:
        n = C.c_uint64()
        self._check(_ffi.load().bowshock_arena_cells(self._h, C.byref(n)))
        return n.value

    def run(self, n: int) -> np.ndarray:
        """n iterations of every active case: the density residual history, shape (n, ncases)."""
        out = np.zeros(n * self.ncases)
        self._check(_ffi.load().bowshock_arena_run(self._h, int(n), _ffi.dptr(out)))
        return out.reshape(n, self.ncases)

    def prepare(self, n: int):
        """Build the CUDA graph run(n) launches first, without running it."""
        self._check(_ffi.load().bowshock_arena_prepare(self._h, int(n)))

    def ms_per_iter(self) -> float:
        d = C.c_double()
        self._check(_ffi.load().bowshock_arena_last_ms_per_iter(self._h, C.byref(d)))
        return d.value

    def last_solve_ms(self) -> float:
        """Device time of the last solve() (iterations and force passes, CUDA events), in milliseconds."""
        d = C.c_double()
        self._check(_ffi.load().bowshock_arena_last_solve_ms(self._h, C.byref(d)))
        return d.value

    PROFILE_GROUPS = ("prims", "viscous", "residual", "lines_i", "lines_j", "defect", "turbulence", "stage", "subst_i", "subst_j", "assemble",
                      "turb_lines", "transfer")

    def profile(self, n: int):
        """Per-kernel-group device time over n iterations launched one kernel at a time: {group: (ms, launches)}."""
        ms = np.zeros(len(self.PROFILE_GROUPS))
        cnt = (C.c_uint64 * len(self.PROFILE_GROUPS))()
        self._check(_ffi.load().bowshock_arena_profile(self._h, int(n), _ffi.dptr(ms), cnt))
        return {g: (float(ms[k]), int(cnt[k])) for k, g in enumerate(self.PROFILE_GROUPS)}

    def tuning(self):
        """Launch shapes of the line kernels the autotuner picked: lines per block and prefetching of the first pass per
        direction, lines per block of the substitution passes per direction and of the SST line kernel."""
        t = _ffi.LineTuning()
        self._check(_ffi.load().bowshock_arena_tuning(self._h, C.byref(t)))
        return {n: int(getattr(t, n)) for n, _ in _ffi.LineTuning._fields_}

    def set_tuning(self, **shape):
        """Pin launch shapes (the keys of tuning(); unspecified ones keep their current values)."""
        cur = self.tuning()
        cur.update(shape)
        t = _ffi.LineTuning(*[int(cur[n]) for n, _ in _ffi.LineTuning._fields_])
        self._check(_ffi.load().bowshock_arena_set_tuning(self._h, C.byref(t)))

    def set_case_groups(self, groups: int):
        """Split the active cases into `groups` (1 to 4) independent chains of the chunk's graph (same results)."""
        self._check(_ffi.load().bowshock_arena_set_case_groups(self._h, int(groups)))

    def solve(self, progress=None):
        """Cold-start every case and iterate each to its stop rule (converged cases are masked out)."""
        res = (_ffi.PointResult * self.ncases)()
        cb = _ffi.PROGRESS_FN(lambda u, k, it, r, m: 0 if progress(k, it, r, m) else 1) if progress else _ffi.PROGRESS_FN(0)
        self._check(_ffi.load().bowshock_arena_solve(self._h, res, cb, None))
        return [point_dict(res[k], len(self.cases[k].body.segments)) for k in range(self.ncases)]

    def forces(self):
        out = (_ffi.Forces * self.ncases)()
        self._check(_ffi.load().bowshock_arena_forces(self._h, out))
        return [forces_dict(out[k], len(self.cases[k].body.segments)) for k in range(self.ncases)]

    def state(self, k: int) -> np.ndarray:
        ni, nj = self._descs[k].ni, self._descs[k].nj
        u = np.zeros(4 * ni * nj)
        self._check(_ffi.load().bowshock_arena_state(self._h, k, _ffi.dptr(u)))
        return u.reshape(-1, 4)

    def set_state(self, k: int, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        self._check(_ffi.load().bowshock_arena_set_state(self._h, k, _ffi.dptr(u)))

    def set_active(self, mask):
        m = (C.c_int32 * self.ncases)(*[int(bool(v)) for v in mask])
        self._check(_ffi.load().bowshock_arena_set_active(self._h, m))

    def set_run(self, k: int, numerics, warm=False, r_ref=None):
        """Run parameters of case k for the next solve(): its numerics' stop rules, a warm start (keep the state and
        turbulence set through set_state / set_turb, no first-order start-up) and the drop reference r_ref."""
        p = numerics.run_params(self.cases[k].wake, warm, r_ref)
        self._check(_ffi.load().bowshock_arena_set_run(self._h, int(k), C.byref(p)))

    def turb_state(self, k: int):
        """(k, omega) [n, 2] and mu_t [n] of SST case k."""
        n = self._descs[k].ni * self._descs[k].nj
        t, m = np.zeros(2 * n), np.zeros(n)
        self._check(_ffi.load().bowshock_arena_turb_state(self._h, int(k), _ffi.dptr(t), _ffi.dptr(m)))
        return t.reshape(-1, 2), m

    def set_turb(self, k: int, turb, mu_t):
        t = np.ascontiguousarray(turb, dtype=np.float64).reshape(-1)
        m = np.ascontiguousarray(mu_t, dtype=np.float64).reshape(-1)
        self._check(_ffi.load().bowshock_arena_set_turb(self._h, int(k), _ffi.dptr(t), _ffi.dptr(m)))

    def first_residuals(self, warm) -> np.ndarray:
        """The density residual each case's run would see first from its current state (warm: per-case flags)."""
        w = (C.c_int32 * self.ncases)(*[int(bool(v)) for v in warm])
        out = np.zeros(self.ncases)
        self._check(_ffi.load().bowshock_arena_first_residuals(self._h, w, _ffi.dptr(out)))
        return out

    def residual_history(self, k: int) -> np.ndarray:
        """The density residual of every iteration of case k in the last solve()."""
        n = C.c_uint64()
        self._check(_ffi.load().bowshock_arena_residual_history(self._h, int(k), None, 0, C.byref(n)))
        out = np.zeros(n.value)
        self._check(_ffi.load().bowshock_arena_residual_history(self._h, int(k), _ffi.dptr(out), n.value, C.byref(n)))
        return out

    def set_sst_coupling(self, coupled: bool):
        """SST line systems of the implicit scheme: False (default) the reference's loose coupling (mean-flow 4x4
        lines, then the scalar k and omega lines); True the 6x6 block lines of (dU, dk, domega), solved by block
        substitution (same residuals and fixed point, another iteration path)."""
        self._check(_ffi.load().bowshock_arena_set_sst_coupling(self._h, int(bool(coupled))))

    def set_run_control(self, on_device: bool):
        """Stop rules of solve() on the device after every chunk (True, the default) or on the host (False)."""
        self._check(_ffi.load().bowshock_arena_set_run_control(self._h, int(bool(on_device))))
