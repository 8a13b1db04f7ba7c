"""The cooled boundary's order of accuracy (crates/pantometry-thermal/tests/the_cooled_boundary_order.rs):
a glass slab of n cells in a column, insulated but for a convective film on its top face, settles
into its slowest mode, whose decay rate has the closed form α·λ²/L² with λ·tan λ = Bi. The film's
series-with-the-half-cell conductance (solid.rs:110-122, 1192-1219) makes that rate converge at
second order: each doubling of n cuts the error by more than 3.4, at Bi = 1.7 and at Bi = 17, and
the finest of 4 to 32 cells is within 5e-3. The device's plain f64 slab steps bit for bit with the
oracle's.
"""
import math

import numpy as np
import pytest

import oracle
from pantometry_b200.scenes import BOROSILICATE_CROWN as GLASS  # substance.rs:336-347

LENGTH = 0.048
TOP = 120.0 + 273.15  # Temperature::celsius (crates/pantometry-units/src/lib.rs:729-731)
AMBIENT = 20.0 + 273.15


def slab(cells, h, make=None):
    """the_cooled_boundary_order.rs:22-45: borosilicate with its emissivity zeroed, (1, 1, cells),
    a film of h on ZMax over one cell's face."""
    dx = LENGTH / cells
    g = GLASS
    if make is None:
        b = oracle.Heat((1, 1, cells), dx, g["density"], g["conductivity"], g["specific_heat"], TOP, emissivity=0.0)
    else:
        b = make((1, 1, cells), dx, g["density"], g["conductivity"], g["specific_heat"], TOP)
    b.losing_from("ZMax", AMBIENT, h, dx * dx)
    return b


def measured_rate(cells, h):
    """the_cooled_boundary_order.rs:47-79: settle 40·n² steps at a fifth of the limit, then the
    relative fall of Σ(T − T_amb) over one more step, per second."""
    block = slab(cells, h)
    dt = block.max_stable_dt() * 0.2
    assert block.step(dt, 40 * cells * cells) is None
    before = float(np.sum(block.cells - AMBIENT))
    assert block.step(dt) is None
    after = float(np.sum(block.cells - AMBIENT))
    return (1.0 - after / before) / dt


def exact_rate(h):
    """the_cooled_boundary_order.rs:81-106: α·λ²/L², λ the first root of λ·tan λ = Bi by bisection."""
    k = GLASS["conductivity"]
    alpha = k / GLASS["density"] / GLASS["specific_heat"]
    bi = h * LENGTH / k
    lo, hi = 1e-12, math.pi / 2 - 1e-12
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid * math.tan(mid) < bi:
            lo = mid
        else:
            hi = mid
    lam = 0.5 * (lo + hi)
    return alpha * lam * lam / (LENGTH * LENGTH)


def errors_for(h):
    exact = exact_rate(h)
    errors = [abs(measured_rate(n, h) - exact) / exact for n in (4, 8, 16, 32)]
    return errors, [errors[i] / errors[i + 1] for i in range(3)]


def test_the_cooled_boundary_converges_at_second_order():  # the_cooled_boundary_order.rs:108-131
    errors, ratios = errors_for(40.0)
    assert all(r > 3.4 for r in ratios), (errors, ratios)
    assert errors[3] < 5e-3, errors


def test_a_stiff_film_converges_at_second_order_as_well():  # the_cooled_boundary_order.rs:133-150
    errors, ratios = errors_for(400.0)
    assert all(r > 3.4 for r in ratios), (errors, ratios)


@pytest.mark.gpu
def test_device_slab_matches_the_oracle():
    """The 16-cell slab at Bi = 17 for 2000 steps: plain f64 bit for bit with the oracle."""
    from pantometry_b200.domains import Solid3D

    o = slab(16, 400.0)
    g = slab(16, 400.0, make=Solid3D)
    dt = o.max_stable_dt() * 0.2
    assert g.max_stable_dt() * 0.2 == dt
    assert o.step(dt, 2000) is None and g.step(dt, 2000) is None
    assert np.array_equal(g.cells.view(np.uint64), o.cells.view(np.uint64))
