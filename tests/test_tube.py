"""`Tube`, the one-dimensional acoustic domain (crates/pantometry-acoustic/src/lib.rs:107-560).

The oracle is pinned by the reference's own known-answer tests (lib.rs:577-991): one step from
rest is the three-point Laplacian with half-width ends, an absorbing end halves the step limit,
a pulse travels at the speed of sound, the fundamental inverts in half a period and returns in one,
a closed tube keeps its energy to 1e-9 over 2000 steps, a matched end drains the tube and publishes
what it took to 2e-3, the 1 m, 201-cell tube's limit is 14.58 µs and it runs audited at 1e-9.
The GPU forms are checked against the oracle: plain f64 bit for bit with the books within 1e-12,
FP32 within f32 bounds, both draining through a matched end as the reference does.
"""
import math

import numpy as np
import pytest

import oracle

RHO, C_AIR = 1.204, 343.0


def air_tube(cells):
    """`Tube::of_air("tube", 1 m, cells, 1e-4 m²)` (lib.rs:572-574, 196-205)."""
    return oracle.Tube(1.0, cells, 1e-4)


def profile(t, f):
    return f(np.arange(t.n) * t.dx)


def test_one_step_from_rest_is_the_three_point_laplacian():  # lib.rs:577-610
    n = 33
    t = air_tube(n)
    t.release(profile(t, lambda x: np.cos(math.pi * x / 1.0)))
    dx, c = t.dx, C_AIR
    h = t.max_stable_dt() * 0.7
    before = t.fields()["p"].copy()
    assert t.step(h) is None
    after = t.fields()["p"]
    scale = np.abs(before).max() / (dx * dx)
    for i in range(n):
        left = before[1] if i == 0 else before[i - 1]
        right = before[n - 2] if i + 1 == n else before[i + 1]
        expected = (left - 2.0 * before[i] + right) / (dx * dx)
        implied = (after[i] - before[i]) / (0.5 * h * h * c * c)
        assert abs(implied - expected) < scale * 1e-12, i


def test_an_absorbing_end_tightens_the_step_and_a_closed_one_does_not():  # lib.rs:620-645
    closed = air_tube(101)
    wave = closed.max_stable_dt()
    assert abs(wave - closed.dx / C_AIR) < 1e-15
    z = RHO * C_AIR
    matched = air_tube(101).set_ends(("closed", 0.0), ("matched", z))
    assert abs(matched.max_stable_dt() / (wave / 2.0) - 1.0) < 1e-12
    stiff = air_tube(101).set_ends(("closed", 0.0), ("matched", z * 4.0))
    assert abs(stiff.max_stable_dt() - wave) < 1e-15
    opened = air_tube(101).set_ends(("open", 0.0), ("closed", 0.0))
    assert abs(opened.max_stable_dt() - wave / 2.0) < 1e-15


def test_a_pulse_travels_at_the_speed_of_sound():  # lib.rs:727-776
    cells = 401
    t = oracle.Tube(4.0, cells, 1e-4)
    t.release(profile(t, lambda x: 100.0 * np.exp(-(((x - 1.0) / 0.05) ** 2))))
    dt = t.max_stable_dt()
    dx = 4.0 / (cells - 1)
    steps = round(0.005 / dt)
    assert t.step(dt, steps) is None
    p = t.fields()["p"]
    start_cell = round(1.0 / dx)
    best_at = start_cell + 5 + int(np.argmax(p[start_cell + 5:]))
    distance = (best_at - start_cell) * dx
    assert abs(distance / (C_AIR * dt * steps) - 1.0) < 0.02
    assert p[best_at] > 30.0


def test_the_fundamental_oscillates_at_its_predicted_period():  # lib.rs:817-857
    t = air_tube(201)
    t.release(profile(t, lambda x: 100.0 * np.cos(math.pi / 1.0 * x)))
    period = 1.0 / (C_AIR / 2.0)
    dt = t.max_stable_dt()
    steps = round(period / dt)
    start = t.fields()["p"][0]
    assert t.step(dt, steps // 2) is None
    assert t.fields()["p"][0] < -0.9 * start
    assert t.step(dt, steps - steps // 2) is None
    assert abs(t.fields()["p"][0] / start - 1.0) < 0.05


def gaussian(t, centre, width, amp):
    t.release(profile(t, lambda x: amp * np.exp(-(((x - centre) / width) ** 2))))
    return t


def test_a_closed_tube_keeps_its_energy_to_itself():  # lib.rs:859-887
    t = gaussian(air_tube(201), 0.5, 0.08, 200.0)
    start = t.ledger()["total"]
    assert start > 0.0
    assert t.step(t.max_stable_dt(), 2000) is None
    assert t.ledger()["radiated"] == 0.0
    assert abs(t.ledger()["total"] / start - 1.0) < 1e-9


def test_a_matched_end_absorbs_and_publishes_what_it_took():  # lib.rs:889-936
    t = gaussian(air_tube(201).set_ends(("closed", 0.0), ("matched", RHO * C_AIR)), 0.3, 0.05, 150.0)
    start = t.ledger()["total"]
    assert t.step(t.max_stable_dt(), 3000) is None
    collected = t.ledger()["radiated"]
    assert collected > 0.0
    left = t.ledger()["total"]
    assert abs(collected / (start - left) - 1.0) < 2e-3
    assert left < start * 0.01


def test_the_domain_runs_audited():  # lib.rs:938-966
    t = gaussian(air_tube(201), 0.5, 0.08, 200.0)
    assert abs(t.max_stable_dt() * 1e6 - 14.58) < 0.05
    assert t.advance(t.max_stable_dt(), 69 * 21, tol=1e-9) is None


def test_degenerate_tubes_are_handled():  # lib.rs:968-991
    assert air_tube(1).n == 3
    frozen = oracle.Tube(1.0, 11, 1e-4, RHO, 0.0)
    assert not math.isfinite(frozen.max_stable_dt())
    frozen.release(np.full(11, 5.0))
    assert frozen.step(1.0) is None
    assert np.array_equal(frozen.fields()["p"], np.full(11, 5.0))


# ------------------------------------------------------------------------------------------
# The GPU forms against the oracle
# ------------------------------------------------------------------------------------------
ENDS = {
    "closed": (("closed", 0.0), ("closed", 0.0)),
    "matched": (("closed", 0.0), ("matched", 0.0)),
    "open_stiff": (("open", 0.0), ("matched", 3.0 * RHO * C_AIR)),
}


def tube_pair(cells, ends, precision="f64", centre=0.3):
    from pantometry_b200.domains import Tube

    o = air_tube(cells).set_ends(*ENDS[ends])
    g = Tube(1.0, cells, 1e-4, precision=precision).set_ends(*ENDS[ends])
    assert g.n == o.n and g.dx == o.dx
    p = profile(o, lambda x: 150.0 * np.exp(-(((x - centre) / 0.05) ** 2)))
    o.release(p)
    g.release(p)
    return o, g


def assert_bitexact(name, got, want):
    bad = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
    assert bad.size == 0, f"{name}: {bad.size} values differ, first at {bad[0]}: {got[bad[0]]!r} vs {want[bad[0]]!r}"


@pytest.mark.gpu
@pytest.mark.parametrize("ends", list(ENDS))
@pytest.mark.parametrize("cells", [201, 1000])
def test_tube_plain_bitexact(ends, cells):
    o, g = tube_pair(cells, ends)
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-9 if ends == "closed" else -1.0)
    assert o.step(dt, 1) is None and g.step(dt, 1) is None  # the half-step start
    assert o.step(dt, 300) is None and g.step(dt, 300) is None  # graph runs
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "v"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]
    assert abs(lg["parts"][1] - lo["radiated"]) <= 1e-12 * max(lo["radiated"], lo["scale"])


@pytest.mark.gpu
def test_tube_refusal_and_checkpoint_match():
    o, g = tube_pair(101, "matched")
    limit = o.max_stable_dt()
    vo, vg = o.step(limit * 2.5), g.step(limit * 2.5)  # past dx/c as well
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert vg[key] == vo[key], key
    dt = 0.8 * limit
    assert o.step(dt, 10) is None and g.step(dt, 10) is None
    o.checkpoint()
    g.checkpoint()
    assert o.step(dt, 80) is None and g.step(dt, 80) is None
    o.restore()
    g.restore()
    assert o.step(dt, 7) is None and g.step(dt, 7) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "v"):
        assert_bitexact(k, fg[k], fo[k])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_tube_matched_end_drains_on_the_gpu(precision):
    """lib.rs:889-936 on the GPU: the matched end takes the pulse and publishes what it took."""
    o, g = tube_pair(201, "matched", precision=precision)
    start = g.ledger()["total"]
    assert g.step(g.max_stable_dt(), 3000) is None
    collected = g.ledger()["parts"][1]
    left = g.ledger()["total"]
    assert collected > 0.0
    assert abs(collected / (start - left) - 1.0) < 2e-3
    assert left < start * 0.01


@pytest.mark.gpu
def test_tube_f32_within_bounds_and_audited():
    o, g = tube_pair(2001, "closed", precision="f32")
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-5)
    assert o.step(dt, 400) is None
    assert g.step(dt, 400) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "v"):
        scale = float(np.abs(fo[k]).max())
        assert np.abs(fg[k] - fo[k]).max() < 1e-4 * scale, k
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-5 * lo["scale"]
