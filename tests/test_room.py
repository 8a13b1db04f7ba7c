"""`Room`, the two-dimensional acoustic domain (crates/pantometry-acoustic/src/room.rs).

The oracle is pinned by the reference's own known-answer tests (room.rs:1075-1329): the Courant
limit is dx/(c√2) and refused past it, excited modes invert in half a period and return in one,
a closed room keeps its energy within 2% over 3000 steps, the leapfrog start makes the scheme
second order (31 → 241 nodes falls more than 30×), the startup adjustment is declared and falls
about 16× over two doublings, and degenerate rooms are handled. The GPU forms are checked against
the oracle: plain f64 bit for bit with the ledger within 1e-12, FP32 within f32 bounds and audited.
"""
import math

import numpy as np
import pytest

import oracle

C_AIR, RHO_AIR = 343.0, 1.204


def square(cells):
    """`Room::of_air("room", 4 m, 4 m, cells)` (room.rs:755-757, 122-138)."""
    return oracle.Room(4.0, 4.0, cells)


def mode_frequency(room, mx, my):
    nx, ny = room.cells
    lx, ly = (nx - 1) * room.dx, (ny - 1) * room.dx
    a, b = mx / lx, my / ly
    return room.speed / 2.0 * math.sqrt(a * a + b * b)  # room.rs:291-300


def energy(room):
    return room.ledger()["total"]


def test_two_dimensions_tighten_the_courant_limit_by_root_two():  # room.rs:1075-1098
    room = square(41)
    limit = room.max_stable_dt()
    assert abs(limit * 1e6 - 206.2) < 0.5
    assert abs((0.1 / 343.0) / limit - math.sqrt(2.0)) < 1e-9
    assert abs(C_AIR * limit * math.sqrt(2.0) / room.dx - 1.0) < 1e-12
    assert room.step(limit) is None
    v = room.step(limit * 1.01)
    assert v is not None and v["quantity"] == "Courant number"


def test_an_excited_mode_oscillates_at_its_predicted_frequency():  # room.rs:1107-1143
    for mx, my in ((1, 0), (1, 1), (2, 1)):
        room = square(81)
        room.release(room.mode_profile(mx, my, 100.0))
        period = 1.0 / mode_frequency(room, mx, my)
        dt = room.max_stable_dt() * 0.5
        steps = round(period / dt)
        start = room.fields()["p"][0]
        assert abs(start) > 50.0
        assert room.step(dt, steps // 2) is None
        half = room.fields()["p"][0]
        assert half < -0.85 * start, (mx, my, start, half)
        assert room.step(dt, steps - steps // 2) is None
        whole = room.fields()["p"][0]
        assert abs(whole / start - 1.0) < 0.1, (mx, my, start, whole)


def gaussian_room(cells=61):
    room = square(cells)
    nx, ny = room.cells
    x = np.arange(nx) * room.dx - 2.0
    y = np.arange(ny) * room.dx - 2.0
    r2 = x[None, :] * x[None, :] + y[:, None] * y[:, None]
    room.release((200.0 * np.exp(-r2 / 0.09)).reshape(-1))
    return room


def test_a_closed_room_keeps_its_energy():  # room.rs:1145-1169
    room = gaussian_room()
    start = energy(room)
    assert start > 0.0
    assert room.step(room.max_stable_dt() * 0.5, 3000) is None
    assert abs(energy(room) / start - 1.0) < 0.02


def test_starting_the_leapfrog_correctly_makes_the_scheme_second_order():  # room.rs:1244-1275
    def worst(cells):
        room = oracle.Room(4.4, 3.1, cells)
        room.release(room.mode_profile(1, 1, 1.0))
        f = mode_frequency(room, 1, 1)
        steps = math.ceil(0.02 / room.max_stable_dt())
        h = 0.02 / steps
        t, w = 0.0, 0.0
        for _ in range(steps):
            assert room.step(h) is None
            t += h
            want = abs(math.cos(2.0 * math.pi * f * t))
            w = max(w, abs(np.abs(room.fields()["p"]).max() - want))
        return w

    assert worst(31) / worst(241) > 30.0


def test_the_startup_adjustment_is_second_order_and_declared():  # room.rs:1277-1302
    def relative(cells):
        room = square(cells)
        room.release(room.mode_profile(1, 1, 1.0))
        total = energy(room)
        assert room.step(room.max_stable_dt()) is None
        return abs(room.ledger()["offset"]) / total

    a, b = relative(31), relative(121)
    assert a > 1e-4
    assert 10.0 < a / b < 24.0


def test_degenerate_rooms_are_handled():  # room.rs:1304-1329
    tiny = oracle.Room(0.1, 0.1, 1)
    assert tiny.cells[0] >= 3 and tiny.cells[1] >= 3
    silent = oracle.Room(1.0, 1.0, 11, 1.0, 1.0, 0.0)
    assert not math.isfinite(silent.max_stable_dt())
    assert silent.step(1.0) is None
    assert np.abs(silent.fields()["p"]).max() == 0.0
    room = square(21)
    room.release(np.full(room.n, 7.0))
    before = room.fields()["p"].copy()
    assert room.step(0.0) is None
    assert np.array_equal(room.fields()["p"], before)


def test_an_audited_room_keeps_its_books():
    """`Simulation::advance` over a room (books_balance, room.rs:341-344): audited at 1e-9."""
    room = gaussian_room(41)
    assert room.advance(room.max_stable_dt() * 0.9, 400, tol=1e-9) is None


# ------------------------------------------------------------------------------------------
# The GPU forms against the oracle
# ------------------------------------------------------------------------------------------
def room_pair(width, height, across, pressure, precision="f64", speed=C_AIR):
    from pantometry_b200.domains import Room

    o = oracle.Room(width, height, across, 1.0, RHO_AIR, speed)
    g = Room(width, height, across, 1.0, RHO_AIR, speed, precision=precision)
    assert g.cells == o.cells and g.dx == o.dx
    p = pressure(o) if callable(pressure) else pressure
    o.release(p)
    g.release(p)
    return o, g


def noise(o, seed=3):
    from pantometry_b200 import workloads as W

    return W.Streams(seed, np.arange(o.n, dtype=np.uint64)).range(-1.0, 1.0)


def blobs(o, seed=5, count=4):
    """A smooth random start: Gaussian blobs of seeded centre, width and sign (white noise sits
    at the grid's Nyquist frequency, where the half-step start moves the invariant past 25%)."""
    from pantometry_b200 import workloads as W

    nx, ny = o.cells
    r = W.Streams(seed, np.arange(count, dtype=np.uint64))
    cx, cy = r.range(0.0, (nx - 1) * o.dx), r.range(0.0, (ny - 1) * o.dx)
    w, a = r.range(2.0, 6.0) * o.dx, r.range(-1.0, 1.0)
    x = np.arange(nx) * o.dx
    y = np.arange(ny) * o.dx
    p = np.zeros((ny, nx))
    for q in range(count):
        p += a[q] * np.exp(-((x[None, :] - cx[q]) ** 2 + (y[:, None] - cy[q]) ** 2) / (w[q] * w[q]))
    return p.reshape(-1)


def assert_bitexact(name, got, want):
    assert got.shape == want.shape, name
    bad = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
    assert bad.size == 0, f"{name}: {bad.size} values differ, first at {bad[0]}: {got[bad[0]]!r} vs {want[bad[0]]!r}"


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(4.0, 4.0, 61), (4.4, 3.1, 45), (0.5, 1.7, 7)])
@pytest.mark.parametrize("start", ["mode", "blobs"])
def test_room_plain_bitexact(shape, start):
    w, h, n = shape
    o, g = room_pair(w, h, n, (lambda r: r.mode_profile(1, 1, 2.0)) if start == "mode" else blobs)
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-9)
    assert o.advance(dt, 1, tol=1e-9) is None and g.step(dt, 1) is None  # the half-step start
    assert o.advance(dt, 150, tol=1e-9) is None and g.step(dt, 150) is None  # a graph run
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]
    assert abs(lg["parts"][1] - lo["offset"]) <= 1e-12 * lo["scale"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_room_startup_refusal_matches(precision):
    """White noise: the half-step start moves the invariant past the reference's 25% bound
    (room.rs:448-476), and both forms refuse the first step with the same violation."""
    o, g = room_pair(4.4, 3.1, 45, noise, precision=precision)
    dt = 0.9 * o.max_stable_dt()
    vo, vg = o.step(dt), g.step(dt)
    assert vo is not None and vg is not None
    assert vg["quantity"] == vo["quantity"] == "energy"
    assert vg["site"] == vo["site"] == "room (starting the leapfrog)"
    assert vg["tolerance"] == vo["tolerance"] == 0.25
    tol = 1e-12 if precision == "f64" else 1e-5
    for key in ("before", "after", "scale"):
        assert abs(vg[key] - vo[key]) <= tol * abs(vo[key]), key


@pytest.mark.gpu
def test_room_courant_refusal_and_degenerate_rooms_match():
    o, g = room_pair(4.0, 4.0, 41, noise)
    limit = o.max_stable_dt()
    vo, vg = o.step(limit * 1.01), g.step(limit * 1.01)
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert vg[key] == vo[key], key
    assert g.step(0.0) is None
    assert_bitexact("p", g.fields()["p"], o.fields()["p"])
    so, sg = room_pair(1.0, 1.0, 11, lambda r: np.full(r.n, 7.0), speed=0.0)
    assert not math.isfinite(sg.max_stable_dt())
    assert so.step(1.0) is None and sg.step(1.0) is None
    assert_bitexact("p", sg.fields()["p"], so.fields()["p"])


@pytest.mark.gpu
def test_room_checkpoint_restore_bitexact():
    o, g = room_pair(4.4, 3.1, 31, lambda r: r.mode_profile(2, 1, 1.0))
    dt = 0.8 * o.max_stable_dt()
    assert o.step(dt, 10) is None and g.step(dt, 10) is None
    o.checkpoint()
    g.checkpoint()
    assert o.step(dt, 70) is None and g.step(dt, 70) is None
    o.restore()
    g.restore()
    assert o.step(dt, 5) is None and g.step(dt, 5) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_room_closed_room_keeps_its_energy_on_the_gpu(precision):
    """room.rs:1145-1169 on the GPU: 3000 steps, the energy within 2%, audited every step."""
    from pantometry_b200.domains import Room

    o = gaussian_room()
    g = Room(4.0, 4.0, 61, precision=precision)
    g.release(o.fields()["p"])
    start = g.ledger()["total"]
    g.set_tolerance(1e-9 if precision == "f64" else 1e-5)
    assert g.step(g.max_stable_dt() * 0.5, 3000) is None
    assert abs(g.ledger()["total"] / start - 1.0) < 0.02


@pytest.mark.gpu
def test_room_f32_within_bounds():
    o, g = room_pair(4.4, 3.1, 121, blobs, precision="f32")
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-5)
    assert o.step(dt, 300) is None
    assert g.step(dt, 300) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "vx", "vy"):
        scale = float(np.abs(fo[k]).max())
        assert np.abs(fg[k] - fo[k]).max() < 1e-4 * scale, k
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-5 * lo["scale"]


@pytest.mark.gpu
def test_room_mode_period_on_the_gpu_f32():
    """room.rs:1107-1143 with the FP32 form: half a period inverts the (2,1) mode, one restores it."""
    from pantometry_b200.domains import Room

    o = square(81)
    g = Room(4.0, 4.0, 81, precision="f32")
    g.release(o.mode_profile(2, 1, 100.0))
    period = 1.0 / mode_frequency(o, 2, 1)
    dt = o.max_stable_dt() * 0.5
    steps = round(period / dt)
    start = g.fields()["p"][0]
    assert g.step(dt, steps // 2) is None
    assert g.fields()["p"][0] < -0.85 * start
    assert g.step(dt, steps - steps // 2) is None
    assert abs(g.fields()["p"][0] / start - 1.0) < 0.1
