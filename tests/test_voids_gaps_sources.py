"""Void cells, the radiative gaps across them, and heat that has a place.

Restated from the reference's own tests: crates/pantometry-thermal/tests/a_gap_that_radiates.rs
(one step is the parallel-plate closed form, a pair conserves to 1e-12 and settles at the mean, a
wider gap between mirrored sides carries the same, a hot pair gets a shorter limit and does not
overshoot), a_grid_with_nothing_in_it.rs (void breaks the path where a poor conductor only slows
it, mirrors across a gap carry nothing, void takes no share of the bus, a block of nothing is no
division by zero) and a_block_that_generates.rs (a source leaves the books balanced and makes a
hot spot, void generates nothing, a constant source leaves the limit alone, a bar between a source
and a film drops P·L/(kA)). The oracle carries the figures; the GPU's plain f64 form reproduces
the oracle bit for bit with void, gaps (the state-dependent limit included) and sources, and the
FP32 form tracks it with void and sources (gaps are refused there, as radiating films are).
"""
import math

import numpy as np
import pytest

import oracle

SIGMA = 5.670374419e-8
# Substance::copper and Substance::pla (crates/pantometry-core/src/substance.rs:462-476, 558-567)
COPPER = dict(density=8.96 * 1e3, conductivity=401.0, specific_heat=385.0, emissivity=0.04)
PLA = dict(density=1.24 * 1e3, conductivity=0.13, specific_heat=1800.0, emissivity=0.90)
GLASS = dict(density=2.51 * 1e3, conductivity=1.114, specific_heat=858.0, emissivity=0.90)


def celsius(c):
    return c + 273.15


def block(counts, dx, sub, initial_c, gpu=False, precision="f64", emissivity=None):
    eps = sub["emissivity"] if emissivity is None else emissivity
    if gpu:
        from pantometry_b200.domains import Solid3D

        return Solid3D(counts, dx, sub["density"], sub["conductivity"], sub["specific_heat"], celsius(initial_c),
                       emissivity=eps, precision=precision)
    return oracle.Heat(counts, dx, sub["density"], sub["conductivity"], sub["specific_heat"], celsius(initial_c),
                       emissivity=eps)


def set_cell(b, c, kelvin):
    t = b.cells
    t[c] = kelvin
    b.cells = t


def plates(gap, emissivity, hot_c, cold_c, gpu=False):
    """a_gap_that_radiates.rs:21-35: two 5 mm copper cells `gap` void cells apart along z."""
    n = 2 + gap
    b = block((1, 1, n), 5e-3, COPPER, cold_c, gpu=gpu, emissivity=emissivity)
    set_cell(b, 0, celsius(hot_c))
    mask = np.zeros(n, dtype=np.uint8)
    mask[1:n - 1] = 1
    return b.empty(mask)


# ------------------------------------------------------------------------------ the oracle


def test_one_step_moves_what_the_parallel_plate_form_says():
    """a_gap_that_radiates.rs:47-71."""
    eps = 0.8
    b = plates(1, eps, 500.0, 20.0)
    hot0, cold0 = b.cells[0], b.cells[2]
    cap = b.coefficients()["capacity"][0]
    dt = 1e-4
    assert b.step(dt, 1) is None
    moved = abs(cold0 - b.cells[2]) * cap
    area = 5e-3 * 5e-3
    expect = SIGMA * area * (hot0 ** 4 - cold0 ** 4) / (2.0 / eps - 1.0) * dt
    assert abs(moved - expect) / expect < 1e-9
    a, bb, g = b.gaps()
    assert list(a) == [0] and list(bb) == [2]
    assert g[0] == SIGMA * area / (1.0 / eps + 1.0 / eps - 1.0)


def test_a_gap_conserves_exactly():
    """a_gap_that_radiates.rs:78-100."""
    b = plates(1, 0.9, 600.0, 20.0)
    opening = b.ledger()["total"]
    dt = b.max_stable_dt()
    assert b.step(dt, 5000) is None
    closing = b.ledger()["total"]
    assert b.cells[2] > celsius(30.0)
    assert abs(closing - opening) / max(abs(opening), 1.0) < 1e-12


def test_an_isolated_pair_settles_at_the_mean():
    """a_gap_that_radiates.rs:107-128."""
    b = plates(1, 0.9, 400.0, 0.0)
    dt = b.max_stable_dt()
    assert b.step(dt, 400_000) is None
    hot, cold = b.cells[0], b.cells[2]
    mean = 0.5 * (celsius(400.0) + celsius(0.0))
    assert abs(hot - cold) < 1.0
    assert abs(0.5 * (hot + cold) - mean) < 1e-6


def test_a_wide_gap_carries_the_same_because_the_sides_are_mirrors():
    """a_gap_that_radiates.rs:152-170 (the exchange part; the open-gap view factor is a report,
    not part of the step)."""
    def step_once(gap):
        b = plates(gap, 0.8, 500.0, 20.0)
        before = b.cells[1 + gap]
        assert b.step(1e-4, 1) is None
        return b.cells[1 + gap] - before

    narrow, wide = step_once(1), step_once(5)
    assert abs(narrow - wide) / narrow < 1e-12


def test_a_hot_pair_gets_a_shorter_limit_and_does_not_overshoot():
    """a_gap_that_radiates.rs:200-225."""
    cool = plates(1, 0.9, 40.0, 20.0).max_stable_dt()
    hot = plates(1, 0.9, 1200.0, 20.0).max_stable_dt()
    assert hot < cool
    b = plates(1, 0.9, 1200.0, 20.0)
    dt = b.max_stable_dt()
    for _ in range(200):
        assert b.step(dt, 1) is None
        assert b.cells[0] >= b.cells[2]


def bar(n, hot_cells, gpu=False, emissivity=None):
    """a_grid_with_nothing_in_it.rs:16-28: copper, 5 mm cells along z, the first cells at 300 C."""
    b = block((1, 1, n), 5e-3, COPPER, 20.0, gpu=gpu, emissivity=emissivity)
    t = b.cells
    t[:hot_cells] = celsius(300.0)
    b.cells = t
    return b


def march(b, steps):
    dt = b.max_stable_dt()
    assert b.step(dt, steps) is None


def test_void_breaks_the_path_and_a_poor_conductor_only_slows_it():
    """a_grid_with_nothing_in_it.rs:52-89."""
    middle = (np.arange(5) == 2).astype(np.uint8)
    solid = bar(5, 2)
    march(solid, 4000)
    insulated = bar(5, 2)
    insulated.fill(middle, PLA["density"], PLA["conductivity"], PLA["specific_heat"], PLA["emissivity"])
    march(insulated, 4000)
    gapped = bar(5, 2).empty(middle)
    march(gapped, 4000)
    start = celsius(20.0)
    copper, plastic, nothing = solid.cells[4], insulated.cells[4], gapped.cells[4]
    assert copper > start + 50.0
    assert plastic > start + 1.0
    assert nothing > start
    assert plastic < copper and nothing < plastic


def test_a_gap_between_mirrors_carries_nothing():
    """a_grid_with_nothing_in_it.rs:97-122."""
    b = bar(5, 2, emissivity=0.0).empty((np.arange(5) == 2).astype(np.uint8))
    assert len(b.gaps()[0]) == 0
    march(b, 4000)
    assert abs(b.cells[4] - celsius(20.0)) < 1e-9


def test_void_takes_no_share_of_the_bus():
    """a_grid_with_nothing_in_it.rs:165-203."""
    def gained(void):
        b = block((4, 1, 1), 5e-3, COPPER, 20.0)
        mask = (np.arange(4) >= 2).astype(np.uint8)
        if void:
            b.empty(mask)
        opening = b.ledger()["total"]
        b.absorb(1000.0)
        assert b.step(1e-6, 1) is None
        keep = ~mask.astype(bool) if void else np.ones(4, dtype=bool)
        return b.ledger()["total"] - opening, b.cells[keep].mean() - celsius(20.0)

    g_whole, rise_whole = gained(False)
    g_half, rise_half = gained(True)
    assert abs(g_whole - 1000.0) < 1e-6 and abs(g_half - 1000.0) < 1e-6
    assert abs(rise_half / rise_whole - 2.0) < 1e-9


def test_a_block_of_nothing_is_not_a_division_by_zero():
    """a_grid_with_nothing_in_it.rs:207-226."""
    b = block((2, 2, 2), 5e-3, COPPER, 20.0).empty(np.ones(8, dtype=np.uint8))
    assert math.isinf(b.max_stable_dt())
    assert b.ledger()["total"] == 0.0
    assert b.step(1.0, 1) is None


def test_a_source_leaves_the_books_balanced():
    """a_block_that_generates.rs:204-256."""
    b = block((3, 3, 3), 5e-3, COPPER, 20.0)
    centre = np.zeros(27, dtype=np.uint8)
    centre[13] = 1
    b.dissipating(30.0, centre)
    opening = b.ledger()["total"]
    hot_spot = 0.0
    for n in range(2000):
        assert b.step(b.max_stable_dt(), 1) is None
        if n == 20:
            hot_spot = b.cells[13] - b.cells[0]
    closing = b.ledger()["total"]
    assert b.generated_energy() > 100.0
    assert abs(closing - opening) / b.generated_energy() < 1e-12
    assert hot_spot > 1.0


def test_nothing_generates_nothing():
    """a_block_that_generates.rs:263-292."""
    half = (np.arange(4) >= 2).astype(np.uint8)
    b = block((4, 1, 1), 5e-3, COPPER, 20.0).empty(half)
    b.dissipating(10.0, np.ones(4, dtype=np.uint8))
    assert abs(b.generated_power() - 10.0) < 1e-12
    e = block((4, 1, 1), 5e-3, COPPER, 20.0).empty(half)
    e.dissipating(10.0, half)
    assert e.generated_power() == 0.0


def test_a_hard_source_is_stepped_no_shorter_than_a_gentle_one():
    """a_block_that_generates.rs:302-324: a constant source has no feedback on the limit."""
    def limit(watts):
        b = block((3, 3, 3), 5e-3, COPPER, 20.0)
        centre = np.zeros(27, dtype=np.uint8)
        centre[13] = 1
        return b.dissipating(watts, centre).max_stable_dt()

    assert abs(limit(1.0) - limit(1000.0)) < 1e-15


def test_a_source_at_one_end_and_a_sink_at_the_other_makes_the_gradient():
    """a_block_that_generates.rs:164-197, settled as `settle` settles (a_block_that_generates.rs:63-90):
    the limit taken afresh every step, windows of a second until the mean moves under 1 µK/s."""
    watts, n, dx = 5.0, 12, 4e-3
    face = dx * dx
    b = block((n, 1, 1), dx, COPPER, 20.0)
    b.dissipating(watts, (np.arange(n) == 0).astype(np.uint8))
    b.losing_from(1, celsius(20.0), 5000.0, face)
    previous = b.cells.mean()
    for rnd in range(4000):
        window = 0.0
        while window < 1.0:
            dt = b.max_stable_dt()
            assert b.step(dt, 1) is None
            window += dt
        now = b.cells.mean()
        if rnd > 0 and abs(now - previous) / window < 1e-6:
            break
        previous = now
    else:
        raise AssertionError("it never settled")
    drop = b.cells[0] - b.cells[n - 1]
    closed = watts * ((n - 1) * dx) / (COPPER["conductivity"] * face)
    assert abs(drop / closed - 1.0) < 1e-3


# ------------------------------------------------------------------------------ the GPU


def assembly(counts, dx, gpu, precision="f64", gaps=True, seed=3):
    """Copper with a borosilicate region, a void slot across the block and scattered void cells,
    two films (one radiating when `gaps`), 20 W in a corner region, a 40 K spread."""
    nx, ny, nz = counts
    rng = np.random.default_rng(seed)
    k, j, i = np.indices((nz, ny, nx)).reshape(3, -1)
    eps = None if gaps else 0.0
    b = block(counts, dx, COPPER, 20.0, gpu=gpu, precision=precision, emissivity=eps)
    glass = ((i >= nx // 2) & (k < nz // 2)).astype(np.uint8)
    b.fill(glass, GLASS["density"], GLASS["conductivity"], GLASS["specific_heat"], GLASS["emissivity"] if gaps else 0.0)
    void = ((i == nx // 3) & (j > 0)) | ((k == 2 * nz // 3) & (i > 1) & (i < nx - 2)) | (rng.random(i.size) < 0.04)
    b.empty(void.astype(np.uint8))
    b.losing_from(0, celsius(15.0), 40.0, (ny * dx) * (nz * dx))
    b.losing_from(5, celsius(25.0), 300.0, (nx * dx) * (ny * dx))
    b.dissipating(20.0, ((i < 3) & (j < 3) & (k < 3)).astype(np.uint8))
    b.cells = celsius(20.0) + 40.0 * np.random.default_rng(seed + 1).random(i.size)
    return b, void


@pytest.mark.gpu
def test_gpu_plates_match_the_oracle_bit_for_bit():
    o, g = plates(1, 0.9, 600.0, 20.0), plates(1, 0.9, 600.0, 20.0, gpu=True)
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = o.max_stable_dt()
    assert o.step(dt, 5000) is None
    assert g.step(dt, 5000) is None
    np.testing.assert_array_equal(g.cells, o.cells)
    assert g.max_stable_dt() == o.max_stable_dt()  # the state's own limit, gathered on the device
    lo, lg = o.ledger(), g.ledger()
    bound = 1e-12 * max(abs(lo["total"]), 1.0)
    assert abs(lg["total"] - lo["total"]) < bound
    assert abs(lg["parts"][0] - lo["stored"]) < bound


@pytest.mark.gpu
def test_gpu_hot_pair_steps_at_its_own_limit_and_refuses_past_it():
    o, g = plates(1, 0.9, 1200.0, 20.0), plates(1, 0.9, 1200.0, 20.0, gpu=True)
    for _ in range(50):
        dt = o.max_stable_dt()
        assert g.max_stable_dt() == dt
        assert o.step(dt, 1) is None
        assert g.step(dt, 1) is None
    np.testing.assert_array_equal(g.cells, o.cells)
    # the same step size carried on: the pair cools, its limit opens, and both take it
    dt = o.max_stable_dt()
    assert o.step(dt, 300) is None
    assert g.step(dt, 300) is None
    np.testing.assert_array_equal(g.cells, o.cells)
    # past the limit: refused before anything moves, on the host and on the device alike
    v = g.step(1.5 * g.max_stable_dt(), 1)
    assert v is not None and v["quantity"] == "Fourier number"
    np.testing.assert_array_equal(g.cells, o.cells)


@pytest.mark.gpu
@pytest.mark.parametrize("counts", [(11, 7, 6), (34, 21, 17)])
def test_gpu_assembly_with_void_gaps_and_sources_is_bit_exact(counts):
    dx = 2e-3
    o, void = assembly(counts, dx, gpu=False)
    g, _ = assembly(counts, dx, gpu=True)
    ao, bo, co = o.gaps()
    ag, bg, cg = g.gaps()
    assert len(ao) > 10
    np.testing.assert_array_equal(ag, ao)
    np.testing.assert_array_equal(bg, bo)
    np.testing.assert_array_equal(cg, co)
    assert g.generated_power() == o.generated_power()
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.8 * o.max_stable_dt()
    g.set_tolerance(1e-9)
    for w in (o, g):
        assert w.step(dt, 40) is None
    np.testing.assert_array_equal(g.cells, o.cells)
    for w in (o, g):
        assert w.step(dt, 150) is None  # graph runs of many steps
    np.testing.assert_array_equal(g.cells, o.cells)
    assert g.max_stable_dt() == o.max_stable_dt()
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-10 * lo["scale"]
    assert abs(g.generated_energy() - o.generated_energy()) < 1e-12 * o.generated_energy()
    # placeless heat skips the void on both
    for w in (o, g):
        w.absorb(3.0)
        assert w.step(dt, 1) is None
    np.testing.assert_array_equal(g.cells, o.cells)
    # a checkpoint and a restore put back the generated joules too
    g.checkpoint()
    before = g.generated_energy()
    assert g.step(dt, 10) is None
    g.restore()
    assert g.generated_energy() == before
    np.testing.assert_array_equal(g.cells, o.cells)


@pytest.mark.gpu
def test_gpu_void_breaks_the_path_as_the_oracle_does():
    middle = (np.arange(5) == 2).astype(np.uint8)
    o, g = bar(5, 2).empty(middle), bar(5, 2, gpu=True).empty(middle)
    dt = o.max_stable_dt()
    assert g.max_stable_dt() == dt
    assert o.step(dt, 4000) is None
    assert g.step(dt, 4000) is None
    np.testing.assert_array_equal(g.cells, o.cells)


@pytest.mark.gpu
def test_gpu_block_of_nothing():
    g = block((2, 2, 2), 5e-3, COPPER, 20.0, gpu=True).empty(np.ones(8, dtype=np.uint8))
    assert math.isinf(g.max_stable_dt())
    assert g.ledger()["total"] == 0.0
    before = g.cells
    assert g.step(1.0, 3) is None
    np.testing.assert_array_equal(g.cells, before)


@pytest.mark.gpu
def test_gpu_source_books_and_hot_spot():
    o, g = block((3, 3, 3), 5e-3, COPPER, 20.0), block((3, 3, 3), 5e-3, COPPER, 20.0, gpu=True)
    centre = np.zeros(27, dtype=np.uint8)
    centre[13] = 1
    for w in (o, g):
        w.dissipating(30.0, centre)
    g.set_tolerance(1e-12)
    opening = g.ledger()["total"]
    dt = o.max_stable_dt()
    assert g.max_stable_dt() == dt
    for w in (o, g):
        assert w.step(dt, 2000) is None
    np.testing.assert_array_equal(g.cells, o.cells)
    assert g.generated_energy() > 100.0
    assert abs(g.ledger()["total"] - opening) / g.generated_energy() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("counts", [(12, 7, 5), (40, 24, 18)])
def test_gpu_f32_void_and_sources_track_the_oracle(counts):
    """The FP32 form with void and sources, films that do not radiate: within 1e-4 K on a 40 K
    spread and the books within 1e-6 of the ledger's scale, audited every step."""
    dx = 2e-3
    o, void = assembly(counts, dx, gpu=False, gaps=False)
    g, _ = assembly(counts, dx, gpu=True, precision="f32", gaps=False)
    assert len(o.gaps()[0]) == 0
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.8 * o.max_stable_dt()
    g.set_tolerance(1e-6)
    assert o.step(dt, 150) is None
    assert g.step(dt, 150) is None
    keep = ~void
    assert np.abs(g.cells[keep] - o.cells[keep]).max() < 1e-4
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-6 * lo["scale"]
    assert abs(g.generated_energy() - o.generated_energy()) < 1e-9 * o.generated_energy()


@pytest.mark.gpu
def test_gpu_f32_refuses_radiative_gaps():
    from pantometry_b200 import _native as N

    g = block((1, 1, 3), 5e-3, COPPER, 20.0, gpu=True, precision="f32", emissivity=0.9)
    g.empty(np.array([0, 1, 0], dtype=np.uint8))
    with pytest.raises(N.NativeError, match="plain f64"):
        g.step(1e-4, 1)
