"""The oracle: a CPU restatement of pantometry's 3D explicit staggered-grid path.

TEST INFRASTRUCTURE ONLY. Nothing in the product package (`pantometry_b200`) imports this
module; only the tests, `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` do, and
only as the checker or as the timed CPU baseline.

The arithmetic lives in `oracle/oracle.cpp` (built by `oracle/Makefile` into `liboracle.so`).
It restates, with operand order preserved:

* `Solid3D` — crates/pantometry-thermal/src/solid.rs:110-122, 377-421, 519-543, 588-784,
  1148-1229, 1269-1288, 1478-1535, 1557-1647, 1709-1950;
  `Environment::loss_from` — crates/pantometry-thermal/src/lib.rs:104-110.
* `Hall` — crates/pantometry-acoustic/src/hall.rs:99-210, 319-384, 401-555, 675-681.
* `Cavity` — crates/pantometry-em/src/cavity.rs:15, 211-458, 675-732, 766-947, 1035-1501,
  1520-1590; `Medium` — crates/pantometry-em/src/lib.rs:67-118.
* `Ledger`, `audit_with`, `Violation` — crates/pantometry-core/src/conserved.rs:37-363;
  `Simulation::advance`/`attribute` — crates/pantometry-core/src/sim.rs:947-1111, 1169-1223.
* `Rng` — crates/pantometry-core/src/rng.rs:36-100.

Pinning: the reference is Rust and cannot be built here, so the restatement is pinned against
the reference's own known-answer tests (restated in tests/test_oracle_*.py): the pinned RNG
digest (rng.rs:306-308), the exact eigen-decay and axis-permutation tests of Solid3D
(solid_closed_forms.rs:46-112), insulated conservation (:156-194), the Hall invariant drift and
startup order (hall_closed_forms.rs:132-181), the Cavity divergence identity
(against_closed_forms.rs:37-100) and the audit semantics (conserved.rs:376-460).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O2 -ffp-contract=off)."""
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


class Violation(C.Structure):
    """Mirror of `Violation` (crates/pantometry-core/src/conserved.rs:128-143)."""

    _fields_ = [
        ("quantity", C.c_char * 32),
        ("site", C.c_char * 96),
        ("before", C.c_double),
        ("after", C.c_double),
        ("scale", C.c_double),
        ("tolerance", C.c_double),
    ]

    def as_dict(self):
        return {
            "quantity": self.quantity.decode(),
            "site": self.site.decode(),
            "before": self.before,
            "after": self.after,
            "scale": self.scale,
            "tolerance": self.tolerance,
        }


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _declare(_lib)
    return _lib


def _declare(L):
    d, i, ll, u64, p = C.c_double, C.c_int, C.c_longlong, C.c_uint64, C.c_void_p
    dp = C.POINTER(C.c_double)
    vp = C.POINTER(Violation)
    sig = {
        "or_rng_new": (u64, [u64]),
        "or_rng_for_index": (u64, [u64, u64]),
        "or_rng_next_u64": (u64, [C.POINTER(u64)]),
        "or_rng_unit": (d, [C.POINTER(u64)]),
        "or_rng_range": (d, [C.POINTER(u64), d, d]),
        "or_rng_digest": (u64, [u64, i]),
        "or_audit_energy": (i, [C.c_char_p, d, d, d, d, d, vp]),
        "or_heat_new": (p, [C.c_char_p, i, i, i, d, d, d, d, d, i, d]),
        "or_heat_free": (None, [p]),
        "or_heat_losing_from": (None, [p, i, d, d, d]),
        "or_heat_fill": (None, [p, d, d, d, d, i, C.c_void_p]),
        "or_heat_empty": (None, [p, C.c_void_p]),
        "or_heat_sample": (None, [p, dp, dp, C.POINTER(C.c_int), dp]),
        "or_hall_sample": (None, [p, dp, dp, C.POINTER(C.c_int), dp]),
        "or_yee_sample": (None, [p, dp, dp, C.POINTER(C.c_int), dp]),
        "or_yee_cutoff_frequency": (C.c_double, [p, C.c_int, C.c_int]),
        "or_yee_mur_coefficient": (C.c_double, [p, C.c_double]),
        "or_yee_launch_along_z": (None, [p, dp, dp]),
        "or_yee_impress": (None, [p, C.c_int, dp]),
        "or_room_sample": (None, [p, dp, dp, C.POINTER(C.c_int), dp]),
        "or_bar_sample": (None, [p, dp, dp, C.POINTER(C.c_int), dp]),
        "or_heat_dissipating": (None, [p, d, C.c_void_p]),
        "or_heat_generated_power": (d, [p]),
        "or_heat_generated_energy": (d, [p]),
        "or_heat_gaps": (C.c_longlong, [p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong]),
        "or_heat_set_cells": (None, [p, dp]),
        "or_heat_get_cells": (None, [p, dp]),
        "or_heat_get_coefficients": (None, [p, dp, dp, dp, dp, dp]),
        "or_heat_max_stable_dt": (d, [p]),
        "or_heat_step": (i, [p, d, i, vp]),
        "or_heat_advance": (i, [p, d, i, d, vp]),
        "or_heat_ledger": (None, [p, dp, dp, dp, dp]),
        "or_heat_absorb": (None, [p, d]),
        "or_heat_checkpoint": (None, [p]),
        "or_heat_restore": (None, [p]),
        "or_heat_release_mode": (None, [p, i, i, i, d, d]),
        "or_heat_mode_amplitude": (d, [p, i, i, i]),
        "or_heat_mode_amplification": (d, [p, i, i, i, d]),
        "or_hall_new": (p, [C.c_char_p, d, d, d, i, d, d]),
        "or_hall_free": (None, [p]),
        "or_hall_nodes": (None, [p, C.POINTER(i), C.POINTER(i), C.POINTER(i), dp]),
        "or_hall_release": (None, [p, dp]),
        "or_hall_release_mode": (None, [p, i, i, i, d]),
        "or_hall_set_source": (None, [p, ll, dp, ll]),
        "or_hall_step": (i, [p, d, i, vp]),
        "or_hall_advance": (i, [p, d, i, d, vp]),
        "or_hall_get": (None, [p, dp, dp, dp, dp, dp]),
        "or_hall_ledger": (None, [p, dp, dp, dp, dp, dp]),
        "or_hall_max_stable_dt": (d, [p]),
        "or_hall_set_speed_blocks": (None, [p, C.c_int, dp, ll]),
        "or_hall_checkpoint": (None, [p]),
        "or_hall_restore": (None, [p]),
        "or_room_new": (p, [C.c_char_p, d, d, i, d, d, d]),
        "or_room_free": (None, [p]),
        "or_room_cells": (None, [p, C.POINTER(i), C.POINTER(i), dp]),
        "or_room_release": (None, [p, dp]),
        "or_room_step": (i, [p, d, i, vp]),
        "or_room_advance": (i, [p, d, i, d, vp]),
        "or_room_get": (None, [p, dp, dp, dp, dp]),
        "or_room_ledger": (None, [p, dp, dp, dp, dp]),
        "or_room_max_stable_dt": (d, [p]),
        "or_room_checkpoint": (None, [p]),
        "or_room_restore": (None, [p]),
        "or_tube_new": (p, [C.c_char_p, d, i, d, d, d]),
        "or_tube_free": (None, [p]),
        "or_tube_dx": (d, [p]),
        "or_tube_cells": (i, [p]),
        "or_tube_set_ends": (None, [p, i, d, i, d]),
        "or_tube_release": (None, [p, dp]),
        "or_tube_step": (i, [p, d, i, vp]),
        "or_tube_advance": (i, [p, d, i, d, vp]),
        "or_tube_get": (None, [p, dp, dp, dp]),
        "or_tube_ledger": (None, [p, dp, dp, dp, dp, dp]),
        "or_tube_max_stable_dt": (d, [p]),
        "or_tube_checkpoint": (None, [p]),
        "or_tube_restore": (None, [p]),
        "or_bar_new": (p, [C.c_char_p, i, d, d, d, d, d, i, d]),
        "or_bar_free": (None, [p]),
        "or_bar_cells": (i, [p]),
        "or_bar_set": (None, [p, dp]),
        "or_bar_get": (None, [p, dp]),
        "or_bar_absorb": (None, [p, d]),
        "or_bar_deposit": (None, [p, dp]),
        "or_bar_max_stable_dt": (d, [p]),
        "or_bar_fourier_number": (d, [p, d]),
        "or_bar_step": (i, [p, d, i, vp]),
        "or_bar_advance": (i, [p, d, i, d, vp]),
        "or_bar_ledger": (None, [p, dp, dp, dp]),
        "or_bar_checkpoint": (None, [p]),
        "or_bar_restore": (None, [p]),
        "or_yee_new": (p, [C.c_char_p, i, i, i, d, d, d, d]),
        "or_yee_free": (None, [p]),
        "or_yee_set_cells": (None, [p, dp, dp, dp]),
        "or_yee_obstruct": (None, [p, C.c_void_p]),
        "or_yee_set_boundary": (None, [p, i, i]),
        "or_yee_release_mode": (None, [p, i, i, d, d]),
        "or_yee_set_source": (None, [p, ll, dp, ll]),
        "or_yee_courant_limit": (d, [p]),
        "or_yee_step": (i, [p, d, i, vp]),
        "or_yee_advance": (i, [p, d, i, d, vp]),
        "or_yee_get": (None, [p, dp, dp, dp, dp, dp, dp]),
        "or_yee_set": (None, [p, dp, dp, dp, dp, dp, dp, i]),
        "or_yee_get_media": (None, [p, dp, dp, dp]),
        "or_yee_ledger": (None, [p, dp, dp, dp, dp, dp]),
        "or_yee_energies": (None, [p, dp, dp]),
        "or_yee_peak_divergence": (d, [p]),
        "or_yee_inject_divergence": (None, [p, i, i, i, d]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _out(n):
    return np.empty(n, dtype=np.float64)


class _Box:
    def _ledger5(self, fn):
        vals = [C.c_double() for _ in range(5)]
        fn(self._h, *[C.byref(v) for v in vals])
        return [v.value for v in vals]

    _sampler = None

    def sample(self, lo, hi, samples):
        """scene::capture's sampling of this domain's field over an extent (crates/pantometry-
        scene/src/lib.rs:391-420): samples = (nx, ny, nz) points from lo to hi (metres), x fastest."""
        n = (C.c_int * 3)(*[int(v) for v in samples])
        lo3, hi3 = (C.c_double * 3)(*map(float, lo)), (C.c_double * 3)(*map(float, hi))
        out = np.empty(int(np.prod([int(v) for v in samples])), dtype=np.float64)
        getattr(lib(), self._sampler)(self._h, lo3, hi3, n, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out


# --------------------------------------------------------------------------------------------
# Solid3D
# --------------------------------------------------------------------------------------------
FACES = ("XMin", "XMax", "YMin", "YMax", "ZMin", "ZMax")


class Heat(_Box):
    """`Solid3D` restated: `new`, `losing_from`, `fill`, `step`, `ledger`, `Simulation::advance`."""

    _sampler = "or_heat_sample"

    def __init__(self, counts, dx, density, conductivity, specific_heat, initial, emissivity=0.0,
                 thermal=True, name="block"):
        L = lib()
        self._h = L.or_heat_new(name.encode(), counts[0], counts[1], counts[2], dx, density,
                                conductivity, specific_heat, emissivity, int(thermal), initial)
        self.counts = tuple(max(1, c) for c in counts)
        self.n = self.counts[0] * self.counts[1] * self.counts[2]

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_heat_free(self._h)
            self._h = None

    def losing_from(self, face, ambient, convection, area):
        lib().or_heat_losing_from(self._h, FACES.index(face) if isinstance(face, str) else face,
                                  ambient, convection, area)
        return self

    def fill(self, mask, density, conductivity, specific_heat, emissivity=0.0, thermal=True):
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        lib().or_heat_fill(self._h, density, conductivity, specific_heat, emissivity, int(thermal),
                           m.ctypes.data_as(C.c_void_p))
        return self

    def empty(self, mask):
        """solid.rs:986-1005: the cells the mask selects become void."""
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        assert m.size == self.n
        lib().or_heat_empty(self._h, m.ctypes.data_as(C.c_void_p))
        return self

    def dissipating(self, watts, mask):
        """solid.rs:1045-1085: `watts` spread over the solid cells the mask selects."""
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        assert m.size == self.n
        lib().or_heat_dissipating(self._h, watts, m.ctypes.data_as(C.c_void_p))
        return self

    def generated_power(self):
        return lib().or_heat_generated_power(self._h)

    def generated_energy(self):
        return lib().or_heat_generated_energy(self._h)

    def gaps(self):
        """The gap pairs (a, b, coefficient) in the order the step applies them."""
        count = lib().or_heat_gaps(self._h, None, None, None, 0)
        a = np.zeros(count, dtype=np.int64)
        b = np.zeros(count, dtype=np.int64)
        g = np.zeros(count)
        lib().or_heat_gaps(self._h, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                           g.ctypes.data_as(C.c_void_p), count)
        return a, b, g

    @property
    def cells(self):
        out = _out(self.n)
        lib().or_heat_get_cells(self._h, _dp(out))
        return out

    @cells.setter
    def cells(self, t):
        t = np.ascontiguousarray(t, dtype=np.float64).reshape(-1)
        assert t.size == self.n
        lib().or_heat_set_cells(self._h, _dp(t))

    def coefficients(self):
        nx, ny, nz = self.counts
        kx, ky, kz = _out((nx + 1) * ny * nz), _out(nx * (ny + 1) * nz), _out(nx * ny * (nz + 1))
        mob, cap = _out(self.n), _out(self.n)
        lib().or_heat_get_coefficients(self._h, _dp(kx), _dp(ky), _dp(kz), _dp(mob), _dp(cap))
        return {"kx": kx, "ky": ky, "kz": kz, "mobility": mob, "capacity": cap}

    def max_stable_dt(self):
        return lib().or_heat_max_stable_dt(self._h)

    def step(self, dt, nsteps=1):
        v = Violation()
        rc = lib().or_heat_step(self._h, dt, nsteps, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def advance(self, dt, nsteps=1, tol=1e-9):
        v = Violation()
        rc = lib().or_heat_advance(self._h, dt, nsteps, tol, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def ledger(self):
        total, scale, stored, lost, _ = self._ledger5(
            lambda h, a, b, c, d, e: lib().or_heat_ledger(h, a, b, c, d))
        return {"total": total, "scale": scale, "stored": stored, "lost": lost}

    def absorb(self, joules):
        lib().or_heat_absorb(self._h, joules)

    def checkpoint(self):
        lib().or_heat_checkpoint(self._h)

    def restore(self):
        lib().or_heat_restore(self._h)

    def release_mode(self, mode, mean, amplitude):
        lib().or_heat_release_mode(self._h, *mode, mean, amplitude)

    def mode_amplitude(self, mode):
        return lib().or_heat_mode_amplitude(self._h, *mode)

    def mode_amplification(self, mode, dt):
        return lib().or_heat_mode_amplification(self._h, *mode, dt)


# --------------------------------------------------------------------------------------------
# Hall
# --------------------------------------------------------------------------------------------
class Hall(_Box):
    """`Hall` restated: `new`, `released_from`, `released_in_mode`, `step`, `ledger`."""

    _sampler = "or_hall_sample"

    def __init__(self, width, height, depth, across, speed, density, name="hall"):
        L = lib()
        self._h = L.or_hall_new(name.encode(), width, height, depth, across, speed, density)
        nx, ny, nz, dx = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        L.or_hall_nodes(self._h, C.byref(nx), C.byref(ny), C.byref(nz), C.byref(dx))
        self.nodes = (nx.value, ny.value, nz.value)
        self.dx = dx.value
        self.speed, self.density = speed, density

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_hall_free(self._h)
            self._h = None

    @property
    def n(self):
        nx, ny, nz = self.nodes
        return nx * ny * nz

    def release(self, pressure):
        p = np.ascontiguousarray(pressure, dtype=np.float64).reshape(-1)
        assert p.size == self.n
        lib().or_hall_release(self._h, _dp(p))
        return self

    def release_mode(self, mode, amplitude):
        lib().or_hall_release_mode(self._h, *mode, amplitude)
        return self

    def set_source(self, node, wave):
        w = np.ascontiguousarray(wave, dtype=np.float64)
        self._wave = w
        lib().or_hall_set_source(self._h, node, _dp(w), w.size)

    def set_speed_blocks(self, block, speeds):
        """Extension: one sound speed per cubic block of `block` nodes a side (x-fastest)."""
        s = np.ascontiguousarray(speeds, dtype=np.float64)
        self._speeds = s
        lib().or_hall_set_speed_blocks(self._h, int(block), _dp(s), s.size)

    def max_stable_dt(self):
        return lib().or_hall_max_stable_dt(self._h)

    def step(self, dt, nsteps=1):
        v = Violation()
        rc = lib().or_hall_step(self._h, dt, nsteps, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def advance(self, dt, nsteps=1, tol=1e-9):
        v = Violation()
        rc = lib().or_hall_advance(self._h, dt, nsteps, tol, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def fields(self):
        nx, ny, nz = self.nodes
        p, pp = _out(self.n), _out(self.n)
        vx, vy, vz = _out((nx - 1) * ny * nz), _out(nx * (ny - 1) * nz), _out(nx * ny * (nz - 1))
        lib().or_hall_get(self._h, _dp(p), _dp(pp), _dp(vx), _dp(vy), _dp(vz))
        return {"p": p, "p_prev": pp, "vx": vx, "vy": vy, "vz": vz}

    def ledger(self):
        total, scale, inv, off, inj = self._ledger5(lib().or_hall_ledger)
        return {"total": total, "scale": scale, "invariant": inv, "offset": off, "injected": inj}

    def checkpoint(self):
        lib().or_hall_checkpoint(self._h)

    def restore(self):
        lib().or_hall_restore(self._h)


class Room(_Box):
    """`Room` restated (crates/pantometry-acoustic/src/room.rs): `new`, `released_from`, `step`,
    `ledger`, `checkpoint`/`restore`. Pressure row-major (i + nx·j); vx (nx−1)·ny, vy nx·(ny−1)."""

    _sampler = "or_room_sample"

    def __init__(self, width, height, across, depth=1.0, density=1.204, speed=343.0, name="room"):
        L = lib()
        self._h = L.or_room_new(name.encode(), width, height, across, depth, density, speed)
        nx, ny, dx = C.c_int(), C.c_int(), C.c_double()
        L.or_room_cells(self._h, C.byref(nx), C.byref(ny), C.byref(dx))
        self.cells = (nx.value, ny.value)
        self.dx = dx.value
        self.speed, self.density, self.depth = speed, density, depth

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_room_free(self._h)
            self._h = None

    @property
    def n(self):
        return self.cells[0] * self.cells[1]

    def release(self, pressure):
        p = np.ascontiguousarray(pressure, dtype=np.float64).reshape(-1)
        assert p.size == self.n
        lib().or_room_release(self._h, _dp(p))
        return self

    def mode_profile(self, mx, my, amplitude):
        """`released_in_mode`'s profile (room.rs:166-183), sampled at the nodes."""
        nx, ny = self.cells
        lx, ly = (nx - 1) * self.dx, (ny - 1) * self.dx
        x = np.arange(nx) * self.dx
        y = np.arange(ny) * self.dx
        px = np.cos(mx * np.pi * x / lx) if lx > 0 else np.ones(nx)
        py = np.cos(my * np.pi * y / ly) if ly > 0 else np.ones(ny)
        return (amplitude * px[None, :] * py[:, None]).reshape(-1)

    def max_stable_dt(self):
        return lib().or_room_max_stable_dt(self._h)

    def step(self, dt, nsteps=1):
        v = Violation()
        rc = lib().or_room_step(self._h, dt, nsteps, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def advance(self, dt, nsteps=1, tol=1e-9):
        v = Violation()
        rc = lib().or_room_advance(self._h, dt, nsteps, tol, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def fields(self):
        nx, ny = self.cells
        p, pp, vx, vy = _out(self.n), _out(self.n), _out((nx - 1) * ny), _out(nx * (ny - 1))
        lib().or_room_get(self._h, _dp(p), _dp(pp), _dp(vx), _dp(vy))
        return {"p": p, "p_prev": pp, "vx": vx, "vy": vy}

    def ledger(self):
        vals = [C.c_double() for _ in range(4)]
        lib().or_room_ledger(self._h, *[C.byref(v) for v in vals])
        total, scale, inv, off = (v.value for v in vals)
        return {"total": total, "scale": scale, "invariant": inv, "offset": off}

    def checkpoint(self):
        lib().or_room_checkpoint(self._h)

    def restore(self):
        lib().or_room_restore(self._h)


END_KINDS = {"closed": 0, "open": 1, "matched": 2}


class Tube(_Box):
    """`Tube` restated (crates/pantometry-acoustic/src/lib.rs:107-560): `new`, `with_ends`,
    `released_from`, `step`, `ledger`, `checkpoint`/`restore`. Ends: ("closed" | "open" |
    "matched", z), z <= 0 meaning the tube's own impedance."""

    def __init__(self, length, cells, area=1e-4, density=1.204, speed=343.0, name="tube"):
        L = lib()
        self._h = L.or_tube_new(name.encode(), length, cells, area, density, speed)
        self.n = L.or_tube_cells(self._h)
        self.dx = L.or_tube_dx(self._h)
        self.speed, self.density, self.area = speed, density, area

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_tube_free(self._h)
            self._h = None

    def set_ends(self, left, right):
        (lk, lz), (rk, rz) = left, right
        lib().or_tube_set_ends(self._h, END_KINDS[lk], lz, END_KINDS[rk], rz)
        return self

    def release(self, pressure):
        p = np.ascontiguousarray(pressure, dtype=np.float64).reshape(-1)
        assert p.size == self.n
        lib().or_tube_release(self._h, _dp(p))
        return self

    def max_stable_dt(self):
        return lib().or_tube_max_stable_dt(self._h)

    def step(self, dt, nsteps=1):
        v = Violation()
        rc = lib().or_tube_step(self._h, dt, nsteps, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def advance(self, dt, nsteps=1, tol=1e-9):
        v = Violation()
        rc = lib().or_tube_advance(self._h, dt, nsteps, tol, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def fields(self):
        p, pp, v = _out(self.n), _out(self.n), _out(self.n - 1)
        lib().or_tube_get(self._h, _dp(p), _dp(pp), _dp(v))
        return {"p": p, "p_prev": pp, "v": v}

    def ledger(self):
        total, scale, inv, off, rad = self._ledger5(lib().or_tube_ledger)
        return {"total": total, "scale": scale, "invariant": inv, "offset": off, "radiated": rad}

    def checkpoint(self):
        lib().or_tube_checkpoint(self._h)

    def restore(self):
        lib().or_tube_restore(self._h)


class Bar(_Box):
    """`Bar1D` restated (crates/pantometry-thermal/src/lib.rs:425-660): insulated explicit
    conduction; the heat a step takes from the bus is handed in first (`absorb`: lumped, into
    the first cell; `deposit`: per cell)."""

    _sampler = "or_bar_sample"

    def __init__(self, cells, dx, area, density, conductivity, specific_heat, initial, thermal=True, name="bar"):
        L = lib()
        self._h = L.or_bar_new(name.encode(), cells, dx, area, density, conductivity, specific_heat, int(thermal),
                               initial)
        self.n = L.or_bar_cells(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_bar_free(self._h)
            self._h = None

    @property
    def cells(self):
        out = _out(self.n)
        lib().or_bar_get(self._h, _dp(out))
        return out

    @cells.setter
    def cells(self, t):
        t = np.ascontiguousarray(t, dtype=np.float64).reshape(-1)
        assert t.size == self.n
        lib().or_bar_set(self._h, _dp(t))

    def absorb(self, joules):
        lib().or_bar_absorb(self._h, joules)

    def deposit(self, joules):
        j = np.ascontiguousarray(joules, dtype=np.float64).reshape(-1)
        assert j.size == self.n
        lib().or_bar_deposit(self._h, _dp(j))

    def max_stable_dt(self):
        return lib().or_bar_max_stable_dt(self._h)

    def fourier_number(self, dt):
        return lib().or_bar_fourier_number(self._h, dt)

    def step(self, dt, nsteps=1):
        v = Violation()
        rc = lib().or_bar_step(self._h, dt, nsteps, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def advance(self, dt, nsteps=1, tol=1e-9):
        v = Violation()
        rc = lib().or_bar_advance(self._h, dt, nsteps, tol, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def ledger(self):
        vals = [C.c_double() for _ in range(3)]
        lib().or_bar_ledger(self._h, *[C.byref(v) for v in vals])
        total, scale, absorbed = (v.value for v in vals)
        return {"total": total, "scale": scale, "absorbed": absorbed}

    def checkpoint(self):
        lib().or_bar_checkpoint(self._h)

    def restore(self):
        lib().or_bar_restore(self._h)


# --------------------------------------------------------------------------------------------
# Cavity
# --------------------------------------------------------------------------------------------
WALL_KINDS = {"conducting": 0, "magnetic": 1, "open": 2}
# crates/pantometry-em/src/lib.rs:67-69: the permittivity (F/m) and permeability (H/m) of free space
EPSILON_0 = 8.854_187_812_8e-12
MU_0 = 1.256_637_062_12e-6


class Yee(_Box):
    """`Cavity` restated: `new`, `fill` (per cell), `obstruct`, `release_mode`, `step`, `ledger`."""

    _sampler = "or_yee_sample"

    def __init__(self, counts, dx, eps_r=1.0, mu_r=1.0, sigma=0.0, name="cavity"):
        L = lib()
        self._h = L.or_yee_new(name.encode(), counts[0], counts[1], counts[2], dx, eps_r, mu_r, sigma)
        self.counts = tuple(max(1, c) for c in counts)
        self.dx = dx
        # Medium::wave_speed (crates/pantometry-em/src/lib.rs:67-69, 104-112): 1/√(εμ)
        self.wave_speed = 1.0 / math.sqrt((EPSILON_0 * eps_r) * (MU_0 * mu_r))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_yee_free(self._h)
            self._h = None

    def shapes(self):
        nx, ny, nz = self.counts
        return {
            "ex": nx * (ny + 1) * (nz + 1), "ey": (nx + 1) * ny * (nz + 1), "ez": (nx + 1) * (ny + 1) * nz,
            "hx": (nx + 1) * ny * nz, "hy": nx * (ny + 1) * nz, "hz": nx * ny * (nz + 1),
        }

    def set_cells(self, eps_r=None, mu_r=None, sigma=None):
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                for a in (eps_r, mu_r, sigma)]
        lib().or_yee_set_cells(self._h, *[None if a is None else _dp(a) for a in keep])

    def obstruct(self, solid):
        m = np.ascontiguousarray(solid, dtype=np.uint8).reshape(-1)
        lib().or_yee_obstruct(self._h, m.ctypes.data_as(C.c_void_p))

    def mur_coefficient(self, dt):
        """`Cavity::mur_coefficient` (cavity.rs:588-591): (c·dt − dx)/(c·dt + dx)."""
        return lib().or_yee_mur_coefficient(self._h, float(dt))

    def cutoff_frequency(self, mode):
        """`Cavity::cutoff_frequency` (cavity.rs:559-563): the (m, n) mode's cutoff of the cross-section."""
        return lib().or_yee_cutoff_frequency(self._h, int(mode[0]), int(mode[1]))

    def launch_along_z(self, dt, envelope):
        """`Cavity::launch_along_z` (cavity.rs:488-521): `envelope(x, y, z)`, over numpy arrays of
        positions in metres, sets Ey at its edges and (as −envelope/η, z moved on by c·dt/2) Hx at its
        faces; the conducting walls are then cleared and the leapfrog counts as begun."""
        nx, ny, nz = self.counts
        x = np.arange(nx + 1, dtype=np.float64) * self.dx
        y = (np.arange(ny, dtype=np.float64) + 0.5) * self.dx
        ze = np.arange(nz + 1, dtype=np.float64) * self.dx
        zh = (np.arange(nz, dtype=np.float64) + 0.5) * self.dx + self.wave_speed * dt / 2.0
        ey = np.ascontiguousarray(envelope(x[None, None, :], y[None, :, None], ze[:, None, None]) *
                                  np.ones((nz + 1, ny, nx + 1)), dtype=np.float64)
        hx = np.ascontiguousarray(envelope(x[None, None, :], y[None, :, None], zh[:, None, None]) *
                                  np.ones((nz, ny, nx + 1)), dtype=np.float64)
        lib().or_yee_launch_along_z(self._h, _dp(ey), _dp(hx))

    def impress(self, plane, add):
        """`Cavity::impress` (cavity.rs:537-548): `add(x, y)` over numpy arrays of positions, added to
        Ey on the plane z = min(plane, nz)·dx, the conducting walls cleared after."""
        nx, ny, _ = self.counts
        x = np.arange(nx + 1, dtype=np.float64) * self.dx
        y = (np.arange(ny, dtype=np.float64) + 0.5) * self.dx
        a = np.ascontiguousarray(add(x[None, :], y[:, None]) * np.ones((ny, nx + 1)), dtype=np.float64)
        lib().or_yee_impress(self._h, int(plane), _dp(a))

    def set_boundary(self, wall, kind):
        lib().or_yee_set_boundary(self._h, wall, WALL_KINDS[kind] if isinstance(kind, str) else kind)

    def release_mode(self, mode, amplitude, dt):
        lib().or_yee_release_mode(self._h, mode[0], mode[1], amplitude, dt)

    def set_source(self, edge, current):
        w = np.ascontiguousarray(current, dtype=np.float64)
        self._current = w
        lib().or_yee_set_source(self._h, edge, _dp(w), w.size)

    def courant_limit(self):
        return lib().or_yee_courant_limit(self._h)

    def step(self, dt, nsteps=1):
        v = Violation()
        rc = lib().or_yee_step(self._h, dt, nsteps, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def advance(self, dt, nsteps=1, tol=1e-9):
        v = Violation()
        rc = lib().or_yee_advance(self._h, dt, nsteps, tol, C.byref(v))
        return None if rc == 0 else v.as_dict()

    def fields(self):
        s = self.shapes()
        out = {k: _out(v) for k, v in s.items()}
        lib().or_yee_get(self._h, *[_dp(out[k]) for k in ("ex", "ey", "ez", "hx", "hy", "hz")])
        return out

    def set_fields(self, f, started):
        keep = {k: np.ascontiguousarray(f[k], dtype=np.float64) for k in ("ex", "ey", "ez", "hx", "hy", "hz")}
        lib().or_yee_set(self._h, *[_dp(keep[k]) for k in ("ex", "ey", "ez", "hx", "hy", "hz")], int(started))

    def media(self):
        s = self.shapes()
        ne = s["ex"] + s["ey"] + s["ez"]
        nh = s["hx"] + s["hy"] + s["hz"]
        eps, sig, mu = _out(ne), _out(ne), _out(nh)
        lib().or_yee_get_media(self._h, _dp(eps), _dp(sig), _dp(mu))
        return {"eps": eps, "sigma": sig, "mu": mu}

    def ledger(self):
        total, scale, inv, diss, work = self._ledger5(lib().or_yee_ledger)
        return {"total": total, "scale": scale, "invariant": inv, "dissipated": diss, "work": work}

    def energies(self):
        e, m = C.c_double(), C.c_double()
        lib().or_yee_energies(self._h, C.byref(e), C.byref(m))
        return e.value, m.value

    def peak_divergence(self):
        return lib().or_yee_peak_divergence(self._h)

    def inject_divergence(self, i, j, k, amount):
        lib().or_yee_inject_divergence(self._h, i, j, k, amount)


# --------------------------------------------------------------------------------------------
# Rng and audit
# --------------------------------------------------------------------------------------------
def rng_digest(seed, draws=10_000):
    return lib().or_rng_digest(seed, draws)


def rng_for_index_units(seed, index, count):
    """`count` successive `unit()` draws of `Rng::for_index(seed, index)`."""
    L = lib()
    s = C.c_uint64(L.or_rng_for_index(seed, index))
    return [L.or_rng_unit(C.byref(s)) for _ in range(count)]


def audit_energy(site, before, after, tol):
    v = Violation()
    rc = lib().or_audit_energy(site.encode(), before[0], before[1], after[0], after[1], tol, C.byref(v))
    return None if rc == 0 else v.as_dict()
