"""Radiating films at the edge of the state-dependent limit, restating the reference's
crates/pantometry-thermal/tests/a_cold_cell_and_a_bus_slug.rs:
  * a glass cell colder than its enclosure, stepped at exactly the limit it reports, warms toward
    the enclosure and does not pass it (:6-44);
  * a slug of placeless heat (900 K of rise) on a PLA block whose every face radiates is taken by
    the next step after that step's stability refusal, checked against the state before the rise
    (solid.rs:1718-1765), and sheds no cell below the air (:46-97; "surface loss ratio" appears
    nowhere in the reference's source, so the step is taken);
  * a hot glass block under still air keeps its books to 1e-12 of what it shed over 200 steps at
    the opening limit (:99-130).
Borosilicate (substance.rs:336-347) and PLA (substance.rs:558-567) keep their catalogue
emissivities of 0.90. The device's plain f64 form reproduces the oracle bit for bit; its FP32 form
passes the same bounds.
"""
import numpy as np
import pytest

import oracle
from pantometry_b200.scenes import BOROSILICATE_CROWN as GLASS

PLA = dict(density=1.24e3, conductivity=0.13, specific_heat=1800.0, emissivity=0.90)
C20, C400, C700 = 20.0 + 273.15, 400.0 + 273.15, 700.0 + 273.15
FACES = ("XMin", "XMax", "YMin", "YMax", "ZMin", "ZMax")


def block(sub, counts, dx, initial, make=None, precision="f64"):
    if make is None:
        return oracle.Heat(counts, dx, sub["density"], sub["conductivity"], sub["specific_heat"], initial,
                           emissivity=sub["emissivity"])
    return make(counts, dx, sub["density"], sub["conductivity"], sub["specific_heat"], initial,
                emissivity=sub["emissivity"], precision=precision)


def cold_cell(make=None, precision="f64"):
    """:7-22: one 20 mm glass cell at 20 °C, its top face seeing a 700 °C enclosure with no
    convection."""
    b = block(GLASS, (1, 1, 1), 20e-3, C20, make, precision)
    b.losing_from("ZMax", C700, 0.0, 20.0e-3 * 20.0e-3)
    return b


def pla_part(make=None, precision="f64"):
    """:48-67: a 4×4×4 PLA part of 5 mm cells, every face radiating to 20 °C air, no convection."""
    side = 4.0 * 5.0e-3
    b = block(PLA, (4, 4, 4), 5e-3, C20, make, precision)
    for f in FACES:
        b.losing_from(f, C20, 0.0, side * side)
    return b


def hot_glass(make=None, precision="f64"):
    """:101-112: a 2×2×2 glass block of 10 mm cells at 400 °C under still air on its top face
    (Environment::still_air, lib.rs:90-96: h = 7 W/m²K)."""
    b = block(GLASS, (2, 2, 2), 10e-3, C400, make, precision)
    b.losing_from("ZMax", C20, 7.0, 4.0e-4)
    return b


def slug_joules():
    """:68-69: 900 times the part's heat capacity, published on the bus."""
    return 900.0 * oracle_capacity()


def oracle_capacity():
    return float(pla_part().coefficients()["capacity"].sum())


def check_cold_cell(b, tol=1e-9):
    limit = b.max_stable_dt()
    assert b.step(limit) is None, "the reported limit must be a step this domain can take"
    after = float(b.cells[0])
    assert C20 - tol < after <= C700, after


def check_slug(b, floor_tol=1e-6):
    limit = b.max_stable_dt()
    b.absorb(slug_joules())
    assert b.max_stable_dt() == limit  # the heat is still on the bus
    assert b.step(limit) is None
    assert float(b.cells.min()) >= C20 - floor_tol


def check_books(b, tol):
    opening = b.ledger()["total"]
    dt = b.max_stable_dt()
    assert b.step(dt, 200) is None
    led = b.ledger()
    moved = led["lost"] if "lost" in led else led["parts"][1]
    assert moved > 0.0
    assert abs(led["total"] - opening) / moved < tol


def test_a_cell_colder_than_its_surroundings_is_not_overdriven():  # :6-44
    check_cold_cell(cold_cell())


def test_a_bus_slug_cannot_shed_a_cell_past_ambient():  # :46-97
    check_slug(pla_part())


def test_a_refused_step_leaves_the_slug_on_the_bus():
    """solid.rs:1718-1765: the refusal comes before the bus share is taken, so a step refused for
    its Fourier number changes nothing and the next one takes the slug."""
    b = pla_part()
    limit = b.max_stable_dt()
    before = b.cells.copy()
    b.absorb(slug_joules())
    assert b.step(limit * 1.01)["quantity"] == "Fourier number"
    assert np.array_equal(b.cells, before)
    assert b.step(limit) is None
    assert float(b.cells.mean()) > C20 + 100.0


def test_the_books_balance_at_the_limit():  # :99-130
    check_books(hot_glass(), 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_films_at_the_limit(precision):
    from pantometry_b200.domains import Solid3D

    f64 = precision == "f64"
    if f64:  # one cell: the plain form's one-cell-a-thread kernel
        o, g = cold_cell(), cold_cell(Solid3D)
        assert g.max_stable_dt() == o.max_stable_dt()
        check_cold_cell(o)
        check_cold_cell(g)
        assert np.array_equal(g.cells, o.cells)
    o, g = pla_part(), pla_part(Solid3D, precision)
    check_slug(o)
    check_slug(g, 1e-6 if f64 else 1e-3)
    if f64:
        assert np.array_equal(g.cells, o.cells)
    else:
        assert np.abs(g.cells - o.cells).max() < 1e-3  # kelvin, from f32 deviations of ~900 K
    o, g = hot_glass(), hot_glass(Solid3D, precision)
    check_books(o, 1e-12)
    check_books(g, 1e-12 if f64 else 1e-4)
    if f64:
        assert np.array_equal(g.cells, o.cells)
