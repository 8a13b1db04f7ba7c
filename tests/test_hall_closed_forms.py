"""`Hall`'s closed forms, restating the reference's crates/pantometry-acoustic/tests/hall_closed_forms.rs
beyond the invariant test (:132-181, restated with the other pins):
  * a released (1, 1, 1) mode tracks |cos 2πft| at its peak, and 13 → 97 nodes across (three
    doublings) cuts the worst departure more than 30×, to under 1e-3 Pa (:99-130);
  * the Courant limit is dx/(c√3), √1.5 below the 2D one, and 5% past it is refused as the
    "Courant number" with `after` = 1.05 while the limit itself is taken (:186-237);
  * a hall of zero depth is one node deep, its (1, 1, 0) mode passes through zero and never exceeds
    its release amplitude over 400 steps (:239-282).
The device's plain f64 form runs the first two bit for bit with the oracle, and its FP32 form
passes the same bounds.
"""
import math

import numpy as np
import pytest

import oracle

SPEED, AIR = 343.0, 1.204  # Hall::of_air (hall.rs:137-152)


def hall(across, depth=2.4, make=None, precision="f64"):
    """hall_closed_forms.rs:11-19: a 4.4 × 3.1 × 2.4 m hall of air, `across` nodes along its width."""
    if make is None:
        return oracle.Hall(4.4, 3.1, depth, across, SPEED, AIR)
    return make(4.4, 3.1, depth, across, SPEED, AIR, precision=precision)


def released(across, mode, amplitude, make=None, precision="f64"):
    """`released_in_mode` (hall.rs:190-210); the device is handed the oracle's mode profile through
    `released_from`, which is what `released_in_mode` calls."""
    o = hall(across).release_mode(mode, amplitude)
    if make is None:
        return o
    return hall(across, make=make, precision=precision).release(o.fields()["p"])


def mode_frequency(h, mode):
    """hall.rs:266-279: c/2·√Σ(n/L)², an axis of no length dropping out."""
    nx, ny, nz = h.nodes
    lengths = [(nx - 1) * h.dx, (ny - 1) * h.dx, (nz - 1) * h.dx]
    s = 0.0
    for n, length in zip(mode, lengths):
        s += (n / length) ** 2 if length > 0.0 else 0.0
    return SPEED / 2.0 * math.sqrt(s)


def peak_trace(h, dt, steps):
    """hall_closed_forms.rs:21-33: step at dt, recording (t, peak |p|) after each step."""
    t, out = 0.0, []
    for _ in range(steps):
        assert h.step(dt) is None
        t += dt
        out.append((t, float(np.abs(h.fields()["p"]).max())))  # peak_pressure, hall.rs:244-246
    return out


def worst_departure(h, ref):
    f = mode_frequency(ref, (1, 1, 1))
    dt = ref.max_stable_dt() * 0.9
    steps = int(round(0.006 / dt))
    return max(abs(peak - abs(math.cos(2.0 * math.pi * f * t))) for t, peak in peak_trace(h, dt, steps))


def check_second_order(make=None, precision="f64"):
    worst = {}
    for across in (13, 97):
        ref = hall(across)
        worst[across] = worst_departure(released(across, (1, 1, 1), 1.0, make, precision), ref)
    assert worst[13] / worst[97] > 30.0, worst
    assert worst[97] < 1e-3, worst
    return worst


def check_courant(make=None, precision="f64"):
    h = hall(45, make=make, precision=precision)
    ref = hall(45)
    dx = ref.dx
    limit = h.max_stable_dt()
    assert abs(limit / (dx / (SPEED * math.sqrt(3.0))) - 1.0) < 1e-12
    assert abs(SPEED * limit * math.sqrt(3.0) / dx - 1.0) < 1e-12  # Hall::courant, hall.rs:319-321
    assert abs((dx / (SPEED * math.sqrt(2.0))) / limit - math.sqrt(1.5)) < 1e-12
    v = released(45, (1, 0, 0), 1.0, make, precision).step(limit * 1.05)
    assert v is not None and v["quantity"] == "Courant number"
    assert abs(v["after"] - 1.05) < 1e-9
    assert released(45, (1, 0, 0), 1.0, make, precision).step(limit) is None


def test_a_released_mode_tracks_the_cosine_and_converges_at_second_order():  # :99-130
    check_second_order()


def test_the_courant_limit_is_the_diagonal_of_a_cube():  # :186-237
    check_courant()


def test_collapsing_an_axis_reduces_to_the_lower_dimension():  # :239-282
    flat = hall(45, depth=0.0)
    assert flat.nodes[2] == 1
    nx, ny, _ = flat.nodes
    lx, ly = (nx - 1) * flat.dx, (ny - 1) * flat.dx
    want = SPEED / 2.0 * math.sqrt((1.0 / lx) ** 2 + (1.0 / ly) ** 2)
    assert abs(mode_frequency(flat, (1, 1, 0)) - want) < 1e-9
    flat.release_mode((1, 1, 0), 1.0)
    trace = peak_trace(flat, flat.max_stable_dt() * 0.9, 400)
    assert min(p for _, p in trace) < 0.2
    assert max(p for _, p in trace) <= 1.0 + 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_hall_closed_forms(precision):
    from pantometry_b200.domains import Hall

    got = check_second_order(Hall, precision)
    if precision == "f64":  # the same departures as the oracle's, to the bit
        want = check_second_order()
        assert got == want
    check_courant(Hall, precision)
