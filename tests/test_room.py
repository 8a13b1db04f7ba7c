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
