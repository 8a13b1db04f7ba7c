"""Python face of the C ABI, shaped like pantometry's `Domain` implementations.

`Solid3D`, `Hall` and `Cavity` here hold a device handle each and answer what the Rust types
answer (crates/pantometry-core/src/sim.rs:77-252): `step` returns `None` or a violation dict
(the `Result<(), Violation>`), `ledger`, `max_stable_dt`, `checkpoint` and `restore`, plus the
constructors and setters the reference offers. Arrays are numpy f64 in the reference's index
order (x fastest). Everything runs on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N

FACES = ("XMin", "XMax", "YMin", "YMax", "ZMin", "ZMax")
WALLS = ("XLow", "XHigh", "YLow", "YHigh", "ZLow", "ZHigh")
BOUNDARY_KINDS = {"conducting": 0, "magnetic": 1, "open": 2}
# crates/pantometry-em/src/lib.rs:67-69: the permittivity (F/m) and permeability (H/m) of free space
EPSILON_0 = 8.854_187_812_8e-12
MU_0 = 1.256_637_062_12e-6


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _precision(p):
    if p in (N.PM_PLAIN_F64, "f64", "plain", "plain_f64"):
        return N.PM_PLAIN_F64
    if p in (N.PM_FIELDS_F32, "f32", "fields_f32"):
        return N.PM_FIELDS_F32
    raise ValueError(f"unknown precision {p!r}")


def _ledger(fn, handle):
    led = N.Ledger()
    N.check(fn(handle, C.byref(led)))
    return {
        "total": led.total,
        "scale": led.scale,
        "parts": [led.parts[q] for q in range(led.n_parts)],
        "steps": led.steps,
    }


def _step(fn, handle, dt, nsteps):
    v = N.Violation()
    st = fn(handle, float(dt), int(nsteps), C.byref(v))
    if st == N.PM_VIOLATION:
        return v.as_dict()
    N.check(st)
    return None


class _Domain:
    _destroy = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                getattr(N.load(), self._destroy)(h)
            except (TypeError, AttributeError):  # the interpreter is shutting down: the process frees it
                pass
            self._h = None

    def close(self):
        self.__del__()

    def set_stream(self, stream):
        """Run on a CUDA stream given as an integer handle (e.g. `torch.cuda.Stream().cuda_stream`)."""
        N.check(getattr(self._lib, self._prefix + "set_stream")(self._h, C.c_void_p(stream or 0)))

    def set_tolerance(self, tol):
        """The per-step audit's relative tolerance; negative turns the audit off."""
        N.check(getattr(self._lib, self._prefix + "set_tolerance")(self._h, float(tol)))

    def step(self, dt, nsteps=1):
        return _step(getattr(self._lib, self._prefix + "step"), self._h, dt, nsteps)

    def ledger(self):
        return _ledger(getattr(self._lib, self._prefix + "ledger"), self._h)

    def checkpoint(self):
        N.check(getattr(self._lib, self._prefix + "checkpoint")(self._h))

    def restore(self):
        N.check(getattr(self._lib, self._prefix + "restore")(self._h))


class _Field:
    """A domain that is a field: scene::capture's sampling of it (crates/pantometry-scene/src/lib.rs:
    347-420), run on the device over the resident state."""

    def sample(self, lo, hi, samples):
        """`ScalarField::at` at samples = (nx, ny, nz) points from lo to hi (metres), x fastest:
        a flat array of nx·ny·nz values, i / (n − 1) of the way along an axis of n > 1 samples and
        the middle of an axis of one."""
        n = (C.c_int * 3)(*[int(v) for v in samples])
        lo3, hi3 = (C.c_double * 3)(*map(float, lo)), (C.c_double * 3)(*map(float, hi))
        out = np.empty(int(n[0]) * int(n[1]) * int(n[2]), dtype=np.float64)
        fn = getattr(self._lib, self._prefix + "sample")
        N.check(fn(self._h, lo3, hi3, n, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        return out


class Solid3D(_Domain, _Field):
    """`Solid3D` (crates/pantometry-thermal/src/solid.rs) on the GPU."""

    _destroy = "pm_heat_destroy"
    _prefix = "pm_heat_"

    def __init__(self, counts, dx, density, conductivity, specific_heat, initial, emissivity=0.0,
                 thermal=True, precision="f64", name="block", device=0):
        self._lib = N.load()
        d = N.HeatDesc()
        self._name = name.encode()
        d.name = self._name
        d.nx, d.ny, d.nz = (max(1, int(c)) for c in counts)
        d.dx = dx
        d.substance = N.Substance(density, conductivity, specific_heat, emissivity, int(thermal))
        d.initial_kelvin = initial
        d.precision = _precision(precision)
        d.device = device
        h = C.c_void_p()
        N.check(self._lib.pm_heat_create(C.byref(d), C.byref(h)))
        self._h = h
        self.counts = (d.nx, d.ny, d.nz)
        self.n = d.nx * d.ny * d.nz
        self.precision = d.precision

    def losing_from(self, face, ambient, convection, area):
        f = FACES.index(face) if isinstance(face, str) else int(face)
        N.check(self._lib.pm_heat_losing_from(self._h, f, ambient, convection, area))
        return self

    def set_wait_budget(self, polls):
        """Polls per grid-wide wait of the many-step path (small plain f64 blocks); 0 makes every
        wait that is not already over give up at once (the call returns PM_DEVICE_TIMEOUT)."""
        N.check(self._lib.pm_heat_set_wait_budget(self._h, int(polls)))

    def step_kernel(self, nsteps):
        """The kernel a step call of `nsteps` steps would run on this block, and its launches."""
        buf = C.create_string_buffer(96)
        n = C.c_longlong()
        N.check(self._lib.pm_heat_step_kernel(self._h, int(nsteps), buf, 96, C.byref(n)))
        return buf.value.decode(), n.value

    def set_cells_per_thread(self, cells):
        """Cells of a row per thread: 1, or a wide form (the default where the block is one material
        and its rows allow): 2 or 4 for plain f64 (4 by default on rows of a multiple of 4), 4 for
        FP32. The fields agree bit for bit."""
        N.check(self._lib.pm_heat_set_cells_per_thread(self._h, int(cells)))

    def fill(self, mask, density, conductivity, specific_heat, emissivity=0.0, thermal=True):
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        s = N.Substance(density, conductivity, specific_heat, emissivity, int(thermal))
        N.check(self._lib.pm_heat_fill(self._h, C.byref(s), m.ctypes.data_as(C.c_void_p), m.size))
        return self

    def empty(self, mask):
        """`Solid3D::empty` (solid.rs:986-1005): the cells the mask selects become void."""
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        N.check(self._lib.pm_heat_empty(self._h, m.ctypes.data_as(C.c_void_p), m.size))
        return self

    def dissipating(self, watts, mask):
        """`Solid3D::dissipating` (solid.rs:1045-1085): `watts` spread over the solid cells the mask
        selects."""
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        N.check(self._lib.pm_heat_dissipating(self._h, float(watts), m.ctypes.data_as(C.c_void_p), m.size))
        return self

    def generated_power(self):
        w = C.c_double()
        N.check(self._lib.pm_heat_generated(self._h, C.byref(w), None))
        return w.value

    def generated_energy(self):
        j = C.c_double()
        N.check(self._lib.pm_heat_generated(self._h, None, C.byref(j)))
        return j.value

    def gaps(self):
        """The gap pairs (a, b, coefficient) in the order the step applies them."""
        count = C.c_size_t()
        N.check(self._lib.pm_heat_gaps(self._h, None, None, None, 0, C.byref(count)))
        a = np.zeros(count.value, dtype=np.int64)
        b = np.zeros(count.value, dtype=np.int64)
        g = np.zeros(count.value)
        N.check(self._lib.pm_heat_gaps(self._h, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                                       g.ctypes.data_as(C.c_void_p), count.value, C.byref(count)))
        return a, b, g

    @property
    def cells(self):
        out = np.empty(self.n, dtype=np.float64)
        N.check(self._lib.pm_heat_download(self._h, _ptr(out), out.size))
        return out

    @cells.setter
    def cells(self, t):
        t = _f64(t, self.n)
        N.check(self._lib.pm_heat_upload(self._h, _ptr(t), t.size))

    def max_stable_dt(self):
        out = C.c_double()
        N.check(self._lib.pm_heat_max_stable_dt(self._h, C.byref(out)))
        return out.value

    def absorb(self, joules):
        N.check(self._lib.pm_heat_absorb(self._h, float(joules)))


class Bar(_Domain, _Field):
    """`Bar1D` (crates/pantometry-thermal/src/lib.rs:425-660) on the GPU: insulated conduction along a
    bar. `absorb` (lumped, into the first cell) and `deposit` (per cell) hand it the heat its next
    step takes from the bus."""

    _destroy = "pm_bar_destroy"
    _prefix = "pm_bar_"

    def __init__(self, cells, dx, area, density, conductivity, specific_heat, initial, thermal=True,
                 precision="f64", name="bar", device=0):
        self._lib = N.load()
        d = N.BarDesc()
        self._name = name.encode()
        d.name = self._name
        d.cells, d.dx, d.area = int(cells), dx, area
        d.substance = N.Substance(density, conductivity, specific_heat, 0.0, int(thermal))
        d.initial_kelvin = initial
        d.precision = _precision(precision)
        d.device = device
        h = C.c_void_p()
        N.check(self._lib.pm_bar_create(C.byref(d), C.byref(h)))
        self._h = h
        self.n = max(2, int(cells))
        self.precision = d.precision

    @property
    def cells(self):
        out = np.empty(self.n, dtype=np.float64)
        N.check(self._lib.pm_bar_download(self._h, _ptr(out), out.size))
        return out

    @cells.setter
    def cells(self, t):
        t = _f64(t, self.n)
        N.check(self._lib.pm_bar_upload(self._h, _ptr(t), t.size))

    def absorb(self, joules):
        N.check(self._lib.pm_bar_absorb(self._h, float(joules)))

    def deposit(self, joules):
        j = _f64(joules, self.n)
        N.check(self._lib.pm_bar_deposit(self._h, _ptr(j), j.size))

    def max_stable_dt(self):
        out = C.c_double()
        N.check(self._lib.pm_bar_max_stable_dt(self._h, C.byref(out)))
        return out.value


class Hall(_Domain, _Field):
    """`Hall` (crates/pantometry-acoustic/src/hall.rs) on the GPU."""

    _destroy = "pm_hall_destroy"
    _prefix = "pm_hall_"

    def __init__(self, width, height, depth, across, speed, density, precision="f64", name="hall", device=0):
        self._lib = N.load()
        d = N.HallDesc()
        self._name = name.encode()
        d.name = self._name
        d.width, d.height, d.depth = width, height, depth
        d.across = across
        d.speed, d.density = speed, density
        d.precision = _precision(precision)
        d.device = device
        h = C.c_void_p()
        N.check(self._lib.pm_hall_create(C.byref(d), C.byref(h)))
        self._h = h
        nx, ny, nz, dx = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        N.check(self._lib.pm_hall_nodes(h, C.byref(nx), C.byref(ny), C.byref(nz), C.byref(dx)))
        self.nodes = (nx.value, ny.value, nz.value)
        self.dx = dx.value
        self.precision = d.precision

    @property
    def n(self):
        nx, ny, nz = self.nodes
        return nx * ny * nz

    def release(self, pressure):
        """`released_from` with the profile already sampled at the nodes."""
        p = _f64(pressure, self.n)
        N.check(self._lib.pm_hall_release(self._h, _ptr(p), p.size))
        return self

    def set_source(self, node, wave):
        w = _f64(wave)
        N.check(self._lib.pm_hall_set_source(self._h, int(node), _ptr(w), w.size))

    def set_speed_blocks(self, block, speeds):
        s = _f64(speeds)
        N.check(self._lib.pm_hall_set_speed_blocks(self._h, int(block), _ptr(s), s.size))

    def max_stable_dt(self):
        out = C.c_double()
        N.check(self._lib.pm_hall_max_stable_dt(self._h, C.byref(out)))
        return out.value

    def download_pressure(self, out):
        """The pressure field into a caller-owned f64 array (pinned memory makes this a DMA)."""
        if out.dtype != np.float64 or out.size != self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous f64 array with one value per node")
        N.check(self._lib.pm_hall_download(self._h, _ptr(out), None, None, None, None))
        return out

    def autotune(self, trial_steps=8):
        """Time every tile shape of the TMA-staged FP32 kernel on the present state and keep the
        fastest (the state and books are put back). Returns (planes, stages); (0, 0) where the hall
        does not use that kernel."""
        pl, st = C.c_int(), C.c_int()
        N.check(self._lib.pm_hall_autotune(self._h, int(trial_steps), C.byref(pl), C.byref(st)))
        return pl.value, st.value

    def set_tile(self, planes, stages):
        N.check(self._lib.pm_hall_set_tile(self._h, int(planes), int(stages)))

    def tile(self):
        pl, st = C.c_int(), C.c_int()
        N.check(self._lib.pm_hall_tile(self._h, C.byref(pl), C.byref(st)))
        return pl.value, st.value

    def fields(self):
        nx, ny, nz = self.nodes
        out = {
            "p": np.empty(self.n), "p_prev": np.empty(self.n),
            "vx": np.empty((nx - 1) * ny * nz), "vy": np.empty(nx * (ny - 1) * nz), "vz": np.empty(nx * ny * (nz - 1)),
        }
        N.check(self._lib.pm_hall_download(self._h, *[_ptr(out[k]) for k in ("p", "p_prev", "vx", "vy", "vz")]))
        return out


class Room(_Domain, _Field):
    """`Room` (crates/pantometry-acoustic/src/room.rs) on the GPU: the two-dimensional hall."""

    _destroy = "pm_room_destroy"
    _prefix = "pm_room_"

    def __init__(self, width, height, across, depth=1.0, density=1.204, speed=343.0, precision="f64", name="room",
                 device=0):
        self._lib = N.load()
        d = N.RoomDesc()
        self._name = name.encode()
        d.name = self._name
        d.width, d.height, d.across = width, height, across
        d.depth, d.density, d.speed = depth, density, speed
        d.precision = _precision(precision)
        d.device = device
        h = C.c_void_p()
        N.check(self._lib.pm_room_create(C.byref(d), C.byref(h)))
        self._h = h
        nx, ny, dx = C.c_int(), C.c_int(), C.c_double()
        N.check(self._lib.pm_room_cells(h, C.byref(nx), C.byref(ny), C.byref(dx)))
        self.cells = (nx.value, ny.value)
        self.dx = dx.value
        self.precision = d.precision

    @property
    def n(self):
        return self.cells[0] * self.cells[1]

    def release(self, pressure):
        """`released_from` with the profile already sampled at the nodes (i + nx·j)."""
        p = _f64(pressure, self.n)
        N.check(self._lib.pm_room_release(self._h, _ptr(p), p.size))
        return self

    def max_stable_dt(self):
        out = C.c_double()
        N.check(self._lib.pm_room_max_stable_dt(self._h, C.byref(out)))
        return out.value

    def fields(self):
        nx, ny = self.cells
        out = {"p": np.empty(self.n), "p_prev": np.empty(self.n), "vx": np.empty((nx - 1) * ny),
               "vy": np.empty(nx * (ny - 1))}
        N.check(self._lib.pm_room_download(self._h, *[_ptr(out[k]) for k in ("p", "p_prev", "vx", "vy")]))
        return out


END_KINDS = {"closed": 0, "open": 1, "matched": 2}


class Tube(_Domain):
    """`Tube` (crates/pantometry-acoustic/src/lib.rs:107-560) on the GPU: the one-dimensional hall,
    its ends closed, open or matched to an impedance."""

    _destroy = "pm_tube_destroy"
    _prefix = "pm_tube_"

    def __init__(self, length, cells, area=1e-4, density=1.204, speed=343.0, precision="f64", name="tube", device=0):
        self._lib = N.load()
        d = N.TubeDesc()
        self._name = name.encode()
        d.name = self._name
        d.length, d.cells, d.area = length, cells, area
        d.density, d.speed = density, speed
        d.precision = _precision(precision)
        d.device = device
        h = C.c_void_p()
        N.check(self._lib.pm_tube_create(C.byref(d), C.byref(h)))
        self._h = h
        n, dx = C.c_int(), C.c_double()
        N.check(self._lib.pm_tube_cells(h, C.byref(n), C.byref(dx)))
        self.n, self.dx = n.value, dx.value
        self.precision = d.precision

    def set_ends(self, left, right):
        """Each end ("closed" | "open" | "matched", z); z <= 0 is the tube's own impedance."""
        (lk, lz), (rk, rz) = left, right
        N.check(self._lib.pm_tube_set_ends(self._h, END_KINDS[lk], float(lz), END_KINDS[rk], float(rz)))
        return self

    def release(self, pressure):
        p = _f64(pressure, self.n)
        N.check(self._lib.pm_tube_release(self._h, _ptr(p), p.size))
        return self

    def max_stable_dt(self):
        out = C.c_double()
        N.check(self._lib.pm_tube_max_stable_dt(self._h, C.byref(out)))
        return out.value

    def fields(self):
        out = {"p": np.empty(self.n), "p_prev": np.empty(self.n), "v": np.empty(self.n - 1)}
        N.check(self._lib.pm_tube_download(self._h, *[_ptr(out[k]) for k in ("p", "p_prev", "v")]))
        return out


class Cavity(_Domain, _Field):
    """`Cavity` (crates/pantometry-em/src/cavity.rs) on the GPU."""

    _destroy = "pm_cavity_destroy"
    _prefix = "pm_cavity_"

    def __init__(self, counts, dx, eps_r=1.0, mu_r=1.0, sigma=0.0, precision="f64", name="cavity", device=0):
        self._lib = N.load()
        d = N.CavityDesc()
        self._name = name.encode()
        d.name = self._name
        d.nx, d.ny, d.nz = (max(1, int(c)) for c in counts)
        d.dx = dx
        d.eps_r, d.mu_r, d.sigma = eps_r, mu_r, sigma
        d.precision = _precision(precision)
        d.device = device
        h = C.c_void_p()
        N.check(self._lib.pm_cavity_create(C.byref(d), C.byref(h)))
        self._h = h
        self.counts = (d.nx, d.ny, d.nz)
        self.dx = dx
        self.precision = d.precision
        self._walls = [BOUNDARY_KINDS["conducting"]] * 6  # cavity.rs:230: conducting walls by default
        # Medium::permittivity / permeability / wave_speed (crates/pantometry-em/src/lib.rs:67-69,
        # 104-112), of the medium the cavity was made of
        self._eps, self._mu = EPSILON_0 * eps_r, MU_0 * mu_r
        self.wave_speed = 1.0 / math.sqrt(self._eps * self._mu)

    def shapes(self):
        nx, ny, nz = self.counts
        return {
            "ex": nx * (ny + 1) * (nz + 1), "ey": (nx + 1) * ny * (nz + 1), "ez": (nx + 1) * (ny + 1) * nz,
            "hx": (nx + 1) * ny * nz, "hy": nx * (ny + 1) * nz, "hz": nx * ny * (nz + 1),
        }

    def fill_cells(self, eps_r=None, mu_r=None, sigma=None):
        n = self.counts[0] * self.counts[1] * self.counts[2]
        arrs = [None if a is None else _f64(a, n) for a in (eps_r, mu_r, sigma)]
        N.check(self._lib.pm_cavity_fill_cells(self._h, *[_ptr(a) for a in arrs], n))

    def obstruct(self, mask):
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        N.check(self._lib.pm_cavity_obstruct(self._h, m.ctypes.data_as(C.c_void_p), m.size))

    def set_boundary(self, wall, kind):
        w = WALLS.index(wall) if isinstance(wall, str) else int(wall)
        k = BOUNDARY_KINDS[kind] if isinstance(kind, str) else int(kind)
        N.check(self._lib.pm_cavity_set_boundary(self._h, w, k))
        self._walls[w] = k

    def cutoff_frequency(self, mode):
        """`Cavity::cutoff_frequency` (cavity.rs:559-563, size() 639-647): the (m, n) mode's cutoff,
        (c/2)·√((m/a)² + (n/b)²) over the cross-section a = nx·dx, b = ny·dx, in hertz."""
        a = float(mode[0]) / (self.counts[0] * self.dx)
        b = float(mode[1]) / (self.counts[1] * self.dx)
        return 0.5 * self.wave_speed * math.sqrt(a * a + b * b)

    def launch_along_z(self, dt, envelope):
        """`Cavity::launch_along_z` (cavity.rs:488-521): `envelope(x, y, z)`, over numpy arrays of
        positions in metres, sets Ey at its edges (i·dx, (j+½)·dx, k·dx) and Hx = −envelope/η at its
        faces with z moved on by c·dt/2; the conducting walls' tangential E is cleared
        (`enforce_walls_where`, cavity.rs:1239-1293) and the next step continues the leapfrog rather
        than starting it. Built on the host and uploaded; the other components are kept."""
        nx, ny, nz = self.counts
        f = self.fields()
        x = np.arange(nx + 1, dtype=np.float64) * self.dx
        y = (np.arange(ny, dtype=np.float64) + 0.5) * self.dx
        ze = np.arange(nz + 1, dtype=np.float64) * self.dx
        zh = (np.arange(nz, dtype=np.float64) + 0.5) * self.dx + self.wave_speed * dt / 2.0
        eta = math.sqrt(self._mu / self._eps)
        ey = envelope(x[None, None, :], y[None, :, None], ze[:, None, None]) * np.ones((nz + 1, ny, nx + 1))
        hx = -(envelope(x[None, None, :], y[None, :, None], zh[:, None, None]) * np.ones((nz, ny, nx + 1))) / eta
        ex = f["ex"].reshape(nz + 1, ny + 1, nx)
        ez = f["ez"].reshape(nz, ny + 1, nx + 1)
        for w, kind in enumerate(self._walls):
            if kind != BOUNDARY_KINDS["conducting"]:
                continue
            if w < 2:
                edge = 0 if w == 0 else nx
                ey[:, :, edge] = 0.0
                ez[:, :, edge] = 0.0
            elif w < 4:
                edge = 0 if w == 2 else ny
                ex[:, edge, :] = 0.0
                ez[:, edge, :] = 0.0
            else:
                edge = 0 if w == 4 else nz
                ex[edge, :, :] = 0.0
                ey[edge, :, :] = 0.0
        f["ey"], f["hx"] = ey.reshape(-1), hx.reshape(-1)
        self.set_fields(f, started=True)
        return self

    def release_mode(self, mode, amplitude, dt):
        N.check(self._lib.pm_cavity_release_mode(self._h, int(mode[0]), int(mode[1]), float(amplitude), float(dt)))

    def set_fields(self, fields, started):
        s = self.shapes()
        arrs = [_f64(fields[k], s[k]) for k in ("ex", "ey", "ez", "hx", "hy", "hz")]
        N.check(self._lib.pm_cavity_upload(self._h, *[_ptr(a) for a in arrs], int(started)))

    def fields(self):
        s = self.shapes()
        out = {k: np.empty(v) for k, v in s.items()}
        N.check(self._lib.pm_cavity_download(self._h, *[_ptr(out[k]) for k in ("ex", "ey", "ez", "hx", "hy", "hz")]))
        return out

    def download_component(self, name, out):
        """One component into a caller-owned f64 array (pinned memory makes this a DMA)."""
        size = self.shapes()[name]
        if out.dtype != np.float64 or out.size != size or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous f64 array of {size} values")
        ptrs = [_ptr(out) if k == name else None for k in ("ex", "ey", "ez", "hx", "hy", "hz")]
        N.check(self._lib.pm_cavity_download(self._h, *ptrs))
        return out

    def set_source(self, edge, current):
        w = _f64(current)
        N.check(self._lib.pm_cavity_set_source(self._h, int(edge), _ptr(w), w.size))

    def autotune(self, trial_steps=8):
        """Time every tile shape of the TMA-staged FP32 kernel on the present state and keep the
        fastest (the state and books are put back). Returns (planes, stages); (0, 0) where the
        cavity does not use that kernel."""
        pl, st = C.c_int(), C.c_int()
        N.check(self._lib.pm_cavity_autotune(self._h, int(trial_steps), C.byref(pl), C.byref(st)))
        return pl.value, st.value

    def set_tile(self, planes, stages):
        N.check(self._lib.pm_cavity_set_tile(self._h, int(planes), int(stages)))

    def tile(self):
        pl, st = C.c_int(), C.c_int()
        N.check(self._lib.pm_cavity_tile(self._h, C.byref(pl), C.byref(st)))
        return pl.value, st.value

    def set_wall_split(self, on):
        """Step the lattice's last column and row by the TMA kernel's wall pass (where nx is a
        multiple of 32 and ny of 8), or by whole tiles; the fields agree bit for bit."""
        N.check(self._lib.pm_cavity_set_wall_split(self._h, 1 if on else 0))

    def wall_split(self):
        on = C.c_int()
        N.check(self._lib.pm_cavity_wall_split(self._h, C.byref(on)))
        return bool(on.value)

    def courant_limit(self):
        out = C.c_double()
        N.check(self._lib.pm_cavity_courant_limit(self._h, C.byref(out)))
        return out.value

    def energies(self):
        e, m = C.c_double(), C.c_double()
        N.check(self._lib.pm_cavity_energies(self._h, C.byref(e), C.byref(m)))
        return e.value, m.value


class Ensemble:
    """Many independent one-material `Solid3D` blocks of uneven sizes advanced together by one
    persistent brick-list kernel per step — the GPU form of `Ensemble::run` over `Solid3D`
    samples (crates/pantometry-core/src/ensemble.rs:102-140). Each block has its own substance,
    step, films (on all six faces at its own T0: 0 insulated, +inf Dirichlet) and FP64 books.

    `grids` is a list of dicts: counts, dx, substance (density, conductivity, specific_heat,
    emissivity), initial (T0, kelvin), convection (W/m²K) and dt (seconds)."""

    def __init__(self, grids, precision="f32", device=0):
        self._lib = N.load()
        self._desc = self.describe(grids)
        self.counts = [tuple(int(c) for c in g["counts"]) for g in grids]
        self.sizes = np.array([nx * ny * nz for nx, ny, nz in self.counts], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        self.n = int(self.offsets[-1])
        self.precision = _precision(precision)
        h = C.c_void_p()
        N.check(self._lib.pm_ensemble_create(self._desc, len(grids), self.precision, device, C.byref(h)))
        self._h = h

    @staticmethod
    def describe(grids):
        arr = (N.EnsembleGrid * len(grids))()
        for d, g in zip(arr, grids):
            d.nx, d.ny, d.nz = (int(c) for c in g["counts"])
            d.dx = g["dx"]
            s = g["substance"]
            d.substance = N.Substance(s["density"], s["conductivity"], s["specific_heat"], s.get("emissivity", 0.0), 1)
            d.initial_kelvin = g["initial"]
            d.convection_w_per_m2_k = g.get("convection", 0.0)
            d.dt = g.get("dt", 1.0)
        return arr

    @staticmethod
    def max_stable_dt(grids):
        """Each block's `max_stable_dt` (solid.rs:1709-1715), computed on the host."""
        desc = Ensemble.describe(grids)
        out = np.empty(len(grids))
        N.check(N.load().pm_ensemble_max_stable_dt(desc, len(grids), _ptr(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            N.load().pm_ensemble_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    def upload(self, kelvin):
        """Every block's cells, concatenated in block order; starts fresh books."""
        t = _f64(kelvin, self.n)
        N.check(self._lib.pm_ensemble_upload(self._h, _ptr(t), t.size))

    def download(self, out=None):
        if out is None:
            out = np.empty(self.n)
        if out.dtype != np.float64 or out.size != self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous f64 array with one value per cell")
        N.check(self._lib.pm_ensemble_download(self._h, _ptr(out), out.size))
        return out

    def block(self, cells, g):
        """Block g's cells out of a concatenated array."""
        return cells[self.offsets[g]:self.offsets[g + 1]]

    def set_tolerance(self, tol):
        N.check(self._lib.pm_ensemble_set_tolerance(self._h, float(tol)))

    def set_stream(self, stream):
        N.check(self._lib.pm_ensemble_set_stream(self._h, C.c_void_p(stream or 0)))

    def step(self, nsteps=1):
        v = N.Violation()
        st = self._lib.pm_ensemble_step(self._h, int(nsteps), C.byref(v))
        if st == N.PM_VIOLATION:
            return v.as_dict()
        N.check(st)
        return None

    def ledgers(self):
        out = (N.Ledger * len(self.counts))()
        N.check(self._lib.pm_ensemble_ledgers(self._h, out, len(self.counts)))
        return [{"total": l.total, "scale": l.scale, "parts": [l.parts[q] for q in range(l.n_parts)], "steps": l.steps}
                for l in out]

    def set_shape(self, brick_x, planes, brick_y=None):
        """The brick shape: x extent and planes (one cell per thread, y = 256 / x), or with
        `brick_y` any listed shape, among them the f32 quad shapes (16 × 64, 32 × 32, 64 × 16,
        128 × 8) and the f64 pair shapes (16 × 32, 32 × 16, 64 × 8)."""
        if brick_y is None:
            N.check(self._lib.pm_ensemble_set_shape(self._h, int(brick_x), int(planes)))
        else:
            N.check(self._lib.pm_ensemble_set_brick(self._h, int(brick_x), int(brick_y), int(planes)))

    def shape(self):
        bx, by, zc = C.c_int(), C.c_int(), C.c_int()
        N.check(self._lib.pm_ensemble_shape(self._h, C.byref(bx), C.byref(by), C.byref(zc)))
        return bx.value, by.value, zc.value

    def autotune(self, trial_steps=10):
        """Time every brick shape on the present state, keep the fastest; the state is put back.
        Returns the chosen shape as `shape()` gives it: (x, y, planes) in cells."""
        bx, zc = C.c_int(), C.c_int()
        N.check(self._lib.pm_ensemble_autotune(self._h, int(trial_steps), C.byref(bx), C.byref(zc)))
        return self.shape()


def device_count():
    n = C.c_int()
    st = N.load().pm_device_count(C.byref(n))
    return n.value if st == N.PM_OK else 0
