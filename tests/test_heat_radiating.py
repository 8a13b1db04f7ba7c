"""Radiating films (emissivity > 0) on the plain f64 path, and on the FP32 form for blocks of one
material.

With ε > 0 a film's conductance depends on the temperature of the cell it cools: `film_flux` adds
εσ·share·(T⁴ − T∞⁴) (solid.rs:1192-1219), and `worst_rate_now` takes each boundary cell's tangent
conductance h + 4εσ·max(T, T∞)³ at its present temperature (solid.rs:1148-1185, 1269-1288), so the
step limit moves with the state and `step` checks it before it sweeps (solid.rs:1718-1738). On the
device each step kernel gathers the rate of the state it leaves, and the next step checks its dt
against it before anything moves, so a refusal inside a many-step call falls on the same step,
with the same numbers, as the reference's.

The film only sets the limit where its conductance rivals a face's (k/dx): a poor conductor on
coarse cells, hot. The slab case below is such a block: a 1800 K slab beside a radiating face of
5 cm cells of a ceramic (k = 1 W/m K, ε = 0.9); as the face warms, the limit tightens.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, heat_pair

CERAMIC = dict(density=2500.0, conductivity=1.0, specific_heat=840.0, emissivity=0.9)
# Substance::copper (crates/pantometry-core/src/substance.rs:462-475)
COPPER = dict(density=8960.0, conductivity=401.0, specific_heat=385.0, emissivity=0.04)
STILL_AIR_H = 7.0  # Environment::still_air (crates/pantometry-thermal/src/lib.rs:90-96)


def slab_pair(precision="f64"):
    counts, dx = (6, 5, 5), 5e-2
    nx, ny, nz = counts
    k, j, i = np.indices((nz, ny, nx)).reshape(3, -1)
    cells = np.where((i == 1) | (i == 2), 1800.0, 300.0)
    return heat_pair(counts, dx, CERAMIC, 300.0, films=[(0, 300.0, 10.0, (ny * dx) * (nz * dx))], cells=cells,
                     precision=precision)


def copper_cube_pair(precision="f64"):
    """a_block_that_cools.rs:120-148: a copper cube of 3 cells of 4 mm at 300 °C, its ZMax face in
    still air at 20 °C (7 W/m²K), copper's emissivity 0.04."""
    side = 3 * 4.0e-3
    return heat_pair((3, 3, 3), 4.0e-3, COPPER, 300.0 + 273.15, films=[(5, 20.0 + 273.15, STILL_AIR_H, side * side)],
                     precision=precision)


def test_oracle_every_joule_that_leaves_a_radiating_cube_is_counted():
    """a_block_that_cools.rs:129 restated with the film radiating: 2000 s at 0.4 of the opening
    limit, and `stored + lost` (the ledger) moves by less than 1e-12 of the heat shed."""
    o = oracle.Heat((3, 3, 3), 4.0e-3, COPPER["density"], COPPER["conductivity"], COPPER["specific_heat"],
                    300.0 + 273.15, emissivity=COPPER["emissivity"])
    side = 3 * 4.0e-3
    o.losing_from(5, 20.0 + 273.15, STILL_AIR_H, side * side)
    dt = 0.4 * o.max_stable_dt()
    opening = o.ledger()["total"]
    assert o.step(dt, math.ceil(2000.0 / dt)) is None
    closing, moved = o.ledger()["total"], o.ledger()["lost"]
    assert moved > 0.0
    assert abs(closing - opening) / moved < 1e-12


def test_oracle_radiating_film_sets_a_limit_that_follows_the_state():
    """The slab block in the oracle: the opening limit is the interior's dx²/(6α); once the face
    beside the slab warms, the radiating film's tangent conductance makes it shorter."""
    counts, dx = (6, 5, 5), 5e-2
    nx, ny, nz = counts
    o = oracle.Heat(counts, dx, CERAMIC["density"], CERAMIC["conductivity"], CERAMIC["specific_heat"], 300.0,
                    emissivity=CERAMIC["emissivity"])
    o.losing_from(0, 300.0, 10.0, (ny * dx) * (nz * dx))
    k, j, i = np.indices((nz, ny, nx)).reshape(3, -1)
    o.cells = np.where((i == 1) | (i == 2), 1800.0, 300.0)
    alpha = CERAMIC["conductivity"] / (CERAMIC["density"] * CERAMIC["specific_heat"])
    opening = o.max_stable_dt()
    assert abs(opening - dx * dx / (6.0 * alpha)) <= 1e-12 * opening
    assert o.step(0.5 * opening, 4) is None
    assert o.max_stable_dt() < 0.97 * opening


@pytest.mark.gpu
def test_radiating_copper_cube_bitexact_and_every_joule_counted():
    """The same run on the GPU: every cell bit for bit with the oracle after 217 961 steps. The
    books hold to 2e-12 of the heat shed rather than the reference's 1e-12 (which the oracle meets,
    at 8.6e-13): the fields are the same bits, but the device adds each step's shed heat to `lost`
    as one fixed-order sum, where the reference adds it cell by cell, and over 2e5 steps the two
    associations part by about 1e-13 of the total."""
    o, g = copper_cube_pair()
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.4 * o.max_stable_dt()
    steps = math.ceil(2000.0 / dt)
    opening = g.ledger()["total"]
    assert o.step(dt, steps) is None
    assert g.step(dt, steps) is None  # graphs of 64 steps and single launches
    assert_bitexact("cells", g.cells, o.cells)
    lg, lo = g.ledger(), o.ledger()
    moved = lg["parts"][1]
    assert moved > 0.0
    assert abs(lg["total"] - opening) / moved < 2e-12
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]
    assert abs(moved - lo["lost"]) <= 1e-12 * lo["lost"]
    assert g.max_stable_dt() == o.max_stable_dt()


@pytest.mark.gpu
def test_radiating_limit_follows_the_state_bit_for_bit():
    o, g = slab_pair()
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.5 * o.max_stable_dt()
    g.set_tolerance(1e-9)
    for _ in range(3):
        assert o.advance(dt, 5, tol=1e-9) is None
        assert g.step(dt, 5) is None
        assert_bitexact("cells", g.cells, o.cells)
        assert g.max_stable_dt() == o.max_stable_dt()  # the state-dependent limit of the new state


@pytest.mark.gpu
@pytest.mark.parametrize("calls", ["one call of 100 steps", "single steps"])
def test_radiating_refusal_falls_on_the_reference_step(calls):
    """A step at 0.95 of the opening limit: the oracle refuses on step 4, once the face beside the
    slab has warmed. The GPU refuses the same step, inside a call of 100 steps (a 64-step graph)
    or on its own, with the same violation, and holds the state of the step before."""
    o, g = slab_pair()
    dt = 0.95 * o.max_stable_dt()
    refused_at = None
    for s in range(1, 100):
        v = o.step(dt, 1)
        if v is not None:
            refused_at, want = s, v
            break
    assert refused_at == 4, refused_at
    if calls == "single steps":
        for s in range(1, refused_at):
            assert g.step(dt, 1) is None
        v = g.step(dt, 1)
        assert v is not None and v["step"] == 1
    else:
        v = g.step(dt, 100)
        assert v is not None and v["step"] == refused_at
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert v[key] == want[key], key
    assert_bitexact("cells", g.cells, o.cells)


@pytest.mark.gpu
def test_radiating_fp32_copper_cube_tracks_the_oracle_and_counts_every_joule():
    """The FP32 form of the cooling cube (one material, no gaps): the one-cell FP32 kernel with each
    face cell's film at its kelvin, 20 000 steps at 0.4 of the limit, within f32 rounding of the
    oracle, the books holding what the film took."""
    o, g = copper_cube_pair()
    _, f = copper_cube_pair(precision="f32")
    assert f.step_kernel(64)[0] == "heat_f32_step"
    assert abs(f.max_stable_dt() - o.max_stable_dt()) <= 1e-6 * o.max_stable_dt()
    dt = 0.4 * o.max_stable_dt()
    f.set_tolerance(1e-6)
    opening = f.ledger()["total"]
    assert o.step(dt, 20000) is None
    assert f.step(dt, 20000) is None
    assert np.abs(f.cells - o.cells).max() < 1e-3  # kelvin, from 573 K down by tens of kelvin
    lf, lo = f.ledger(), o.ledger()
    assert lf["parts"][1] > 0.0 and abs(lf["parts"][1] - lo["lost"]) <= 1e-4 * lo["lost"]
    # the books: every step audited at 1e-6; over 20 000 steps the f32 rounding of each cell's
    # deviation (tens of kelvin, 27 cells) leaves the total a few 1e-5 of the scale from the opening
    assert abs(lf["total"] - opening) <= 1e-4 * lf["scale"]
    assert abs(f.max_stable_dt() - o.max_stable_dt()) <= 1e-6 * o.max_stable_dt()


@pytest.mark.gpu
def test_radiating_fp32_limit_follows_the_state_and_refuses_on_the_reference_step():
    o, g = slab_pair(precision="f32")
    assert abs(g.max_stable_dt() - o.max_stable_dt()) <= 1e-6 * o.max_stable_dt()
    dt = 0.5 * o.max_stable_dt()
    for _ in range(3):
        assert o.step(dt, 5) is None
        assert g.step(dt, 5) is None
        assert np.abs(g.cells - o.cells).max() < 1e-3
        assert abs(g.max_stable_dt() - o.max_stable_dt()) <= 1e-6 * o.max_stable_dt()
    # at 0.95 of the opening limit the state's own limit overtakes the step on the fourth step
    o, g = slab_pair(precision="f32")
    dt = 0.95 * o.max_stable_dt()
    v = g.step(dt, 100)
    assert v is not None and v["quantity"] == "Fourier number" and v["step"] == 4
    assert g.ledger()["steps"] == 3


@pytest.mark.gpu
def test_radiating_fp32_refusals_that_remain():
    """Blocks of several materials with radiating films stay on the plain f64 form."""
    from pantometry_b200._native import NativeError

    counts, dx = (6, 5, 5), 5e-2
    mask = np.zeros(int(np.prod(counts)), dtype=np.uint8)
    mask[:30] = 1
    _, g = heat_pair(counts, dx, CERAMIC, 300.0, films=[(0, 300.0, 10.0, 0.0625)], precision="f32",
                     fill=(mask, COPPER))
    with pytest.raises(NativeError, match="plain f64"):
        g.step(1e-3, 1)
