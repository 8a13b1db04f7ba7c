"""`Bar1D`, explicit conduction along an insulated bar (crates/pantometry-thermal/src/lib.rs:425-660).

The oracle is pinned by the reference's own tests (lib.rs:1179-1360): aluminium on a millimetre
grid has a 7.2 ms limit at Fourier number ½ and refuses past it; glass and aluminium differ by
more than 100× in step; insulated conduction conserves the heat to 1e-12 and flattens a hot spot
tenfold in 500 steps; the same joules handed in lumped or per cell land in different places but
are the same amount. The heat a step takes from the bus is handed in by the caller (`absorb`,
`deposit`). The GPU forms are checked against the oracle: plain f64 bit for bit with the books
within 1e-12, FP32 within f32 bounds, both audited against the heat they took.
"""
import math

import numpy as np
import pytest

import oracle

C0 = 273.15
# substance.rs:362-369 and 336-343 (g/cm³ → kg/m³)
ALUMINIUM = (2.70 * 1000.0, 167.0, 896.0)
GLASS = (2.51 * 1000.0, 1.114, 858.0)


def bar(cells=21, sub=ALUMINIUM, dx=1e-3, initial=C0 + 20.0):
    return oracle.Bar(cells, dx, 1e-4, *sub, initial)


def test_explicit_conduction_refuses_an_unstable_step():  # lib.rs:1179-1204
    b = bar(20)
    limit = b.max_stable_dt()
    assert abs(limit * 1e3 - 7.2) < 0.2
    assert abs(b.fourier_number(limit) - 0.5) < 1e-12
    assert b.step(limit) is None
    v = b.step(limit * 1.5)
    assert v is not None and v["quantity"] == "Fourier number" and v["after"] > 0.5


def test_two_materials_on_one_grid_need_different_steps():  # lib.rs:1209-1230
    glass, metal = bar(10, GLASS).max_stable_dt(), bar(10, ALUMINIUM).max_stable_dt()
    assert abs(glass - 0.967) < 0.02 and abs(metal - 0.0072) < 0.001 and glass / metal > 100.0


def test_conduction_conserves_heat_and_flattens_a_gradient():  # lib.rs:1233-1268
    b = bar(21)
    t = b.cells
    t[10] = C0 + 60.0
    b.cells = t
    before = b.cells
    assert b.step(b.max_stable_dt() * 0.9, 500) is None
    after = b.cells
    assert abs(after.sum() / before.sum() - 1.0) < 1e-12
    assert np.ptp(after) < np.ptp(before) / 10.0
    assert after.mean() - C0 > 21.0


def test_heat_arrives_where_it_is_handed_in():  # lib.rs:1278-1345
    joules = 2.0
    lumped = bar(21)
    lumped.absorb(joules)
    assert lumped.step(1e-4) is None
    resolved = bar(21)
    spot = np.zeros(21)
    spot[10] = joules
    resolved.deposit(spot)
    assert resolved.step(1e-4) is None
    assert abs(resolved.ledger()["absorbed"] - lumped.ledger()["absorbed"]) < 1e-15
    lt, rt = lumped.cells - C0, resolved.cells - C0
    assert lt[0] > lt[10] + 1.0 and abs(lt[10] - 20.0) < 1e-9
    assert rt[10] > rt[0] + 1.0


def test_an_audited_bar_books_what_it_took():
    b = bar(41)
    t = b.cells
    t[5:9] = C0 + 45.0
    b.cells = t
    b.absorb(0.5)
    assert b.advance(b.max_stable_dt() * 0.9, 300, tol=1e-9) is None


# ------------------------------------------------------------------------------------------
# The GPU forms against the oracle
# ------------------------------------------------------------------------------------------
def bar_pair(cells, precision="f64"):
    from pantometry_b200.domains import Bar

    o = bar(cells)
    g = Bar(cells, 1e-3, 1e-4, *ALUMINIUM, C0 + 20.0, precision=precision)
    t = C0 + 20.0 + 30.0 * np.exp(-(((np.arange(cells) - cells / 3.0) / (cells / 10.0)) ** 2))
    o.cells = t
    g.cells = t
    return o, g


def assert_bitexact(got, want):
    bad = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
    assert bad.size == 0, f"{bad.size} cells differ, first at {bad[0]}: {got[bad[0]]!r} vs {want[bad[0]]!r}"


@pytest.mark.gpu
@pytest.mark.parametrize("cells", [2, 21, 1000])
def test_bar_plain_bitexact_with_heat_handed_in(cells):
    o, g = bar_pair(cells)
    dt = 0.9 * o.max_stable_dt()
    assert g.max_stable_dt() == o.max_stable_dt()
    g.set_tolerance(1e-9)
    assert o.advance(dt, 70, tol=1e-9) is None and g.step(dt, 70) is None  # a graph run
    for d in (o, g):
        d.absorb(0.3)
        d.deposit(np.linspace(0.0, 0.01, cells))
    assert o.advance(dt, 1, tol=1e-9) is None and g.step(dt, 1) is None
    assert o.advance(dt, 5, tol=1e-9) is None and g.step(dt, 5) is None
    assert_bitexact(g.cells, o.cells)
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * max(lo["scale"], lo["absorbed"])
    assert lg["parts"][1] == pytest.approx(lo["absorbed"], rel=1e-15)


@pytest.mark.gpu
def test_bar_refusal_and_checkpoint_match():
    o, g = bar_pair(21)
    vo, vg = o.step(o.max_stable_dt() * 1.5), g.step(g.max_stable_dt() * 1.5)
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert vg[key] == vo[key], key
    dt = 0.8 * o.max_stable_dt()
    assert o.step(dt, 5) is None and g.step(dt, 5) is None
    o.checkpoint()
    g.checkpoint()
    assert o.step(dt, 70) is None and g.step(dt, 70) is None
    o.restore()
    g.restore()
    assert o.step(dt, 3) is None and g.step(dt, 3) is None
    assert_bitexact(g.cells, o.cells)


@pytest.mark.gpu
def test_bar_f32_within_bounds_and_audited():
    o, g = bar_pair(4001, precision="f32")
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-6)
    o.absorb(1.0)
    g.absorb(1.0)
    assert o.step(dt, 500) is None
    assert g.step(dt, 500) is None
    assert np.abs(g.cells - o.cells).max() < 1e-4  # kelvin, on a 30 K spot
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-6 * max(lo["scale"], lo["absorbed"])
    assert math.isclose(lg["parts"][1], lo["absorbed"], rel_tol=1e-12)
