"""Filled (multi-material) blocks against the reference's own known answers.

Restated from crates/pantometry-thermal/tests/a_layered_wall.rs and a_composite.rs: a wall of
aluminium then borosilicate has exactly the series resistance of its layers at every resolution
(the harmonic face mean makes it an equality), a one-cell laminate is exactly the Reuss bound, the
marched steady state carries ΔT/R and puts the interface where the layers say, a two-material
block conserves its heat to `steps × ε`, and placeless heat leaves it uniform. The oracle carries
the figures; the GPU's plain f64 form reproduces the oracle's filled walls bit for bit.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import assert_bitexact

# Substance::aluminium_6061 and Substance::borosilicate_crown (crates/pantometry-core/src/substance.rs)
ALU = dict(density=2700.0, conductivity=167.0, specific_heat=896.0, emissivity=0.09)
GLASS = dict(density=2510.0, conductivity=1.114, specific_heat=858.0, emissivity=0.90)
T20 = 20.0 + 273.15
DX = 1e-3


def wall(cells, gpu=False, precision="f64"):
    """a_layered_wall.rs:43-54: `cells` millimetre cubes along z, aluminium, then borosilicate
    from the middle on."""
    mask = (np.arange(cells) >= cells // 2).astype(np.uint8)
    if gpu:
        from pantometry_b200.domains import Solid3D

        w = Solid3D((1, 1, cells), DX, ALU["density"], ALU["conductivity"], ALU["specific_heat"], T20,
                    emissivity=ALU["emissivity"], precision=precision)
    else:
        w = oracle.Heat((1, 1, cells), DX, ALU["density"], ALU["conductivity"], ALU["specific_heat"], T20,
                        emissivity=ALU["emissivity"])
    w.fill(mask, GLASS["density"], GLASS["conductivity"], GLASS["specific_heat"], GLASS["emissivity"])
    return w


def chain(w):
    """Σ 1/G over the faces from the first cell centre to the last (face_conductance = k_face·dx,
    solid.rs:564-581)."""
    kz = w.coefficients()["kz"]
    nz = w.counts[2]
    total = 0.0
    for k in range(1, nz):
        total += 1.0 / (kz[k] * DX)
    return total


def test_a_layered_wall_has_exactly_the_series_resistance_of_its_layers():
    """a_layered_wall.rs:137-160."""
    area = DX * DX
    for cells in (12, 24, 48, 96):
        half = cells // 2
        closed = (half - 0.5) * DX / (ALU["conductivity"] * area) + (cells - half - 0.5) * DX / (GLASS["conductivity"] * area)
        off = abs(chain(wall(cells)) / closed - 1.0)
        assert off < 1e-14, (cells, off)


def test_arithmetic_averaging_is_first_order_in_exactly_one_face():
    """a_layered_wall.rs:172-233: err·(n−1) is one number, 2(1/H − 1/A)/(1/k_a + 1/k_g)."""
    ka, kg = ALU["conductivity"], GLASS["conductivity"]
    area = DX * DX
    errors = []
    for cells in (12, 24, 48, 96):
        half = cells // 2
        closed = (half - 0.5) * DX / (ka * area) + (cells - half - 0.5) * DX / (kg * area)
        per = lambda k: DX / (k * area)  # noqa: E731
        arithmetic = (half - 1.0) * per(ka) + (cells - half - 1.0) * per(kg) + per(0.5 * (ka + kg))
        errors.append(abs(arithmetic / closed - 1.0))
    harmonic = 2.0 * ka * kg / (ka + kg)
    want = 2.0 * (1.0 / harmonic - 2.0 / (ka + kg)) / (1.0 / ka + 1.0 / kg)
    assert errors[0] > 0.08 and errors[3] > 0.005
    for n, e in zip((12, 24, 48, 96), errors):
        assert abs(e * (n - 1.0) / want - 1.0) < 1e-12


def test_a_laminate_across_its_layers_is_exactly_the_reuss_bound():
    """a_composite.rs:115-160: every other cell borosilicate, so every face is an interface."""
    reuss = 1.0 / (0.5 / ALU["conductivity"] + 0.5 / GLASS["conductivity"])
    for cells in (8, 16, 32, 64):
        w = oracle.Heat((1, 1, cells), DX, ALU["density"], ALU["conductivity"], ALU["specific_heat"], T20)
        w.fill((np.arange(cells) % 2 == 1).astype(np.uint8), GLASS["density"], GLASS["conductivity"],
               GLASS["specific_heat"], GLASS["emissivity"])
        measured = (cells - 1) / (chain(w) * 1 * DX)
        assert abs(measured / reuss - 1.0) < 1e-15, (cells, measured, reuss)
        # a_composite.rs:501-540: the resolved capacity is the cells' own ρc V
        cap = w.coefficients()["capacity"].sum()
        want = sum((GLASS if k % 2 else ALU)["density"] * DX ** 3 * (GLASS if k % 2 else ALU)["specific_heat"]
                   for k in range(cells))
        assert abs(cap / want - 1.0) < 1e-14


def clamped_march(w, steps, dt, hot, cold):
    """Both end cells held every step (set_temperature at 0 and at the last cell)."""
    for _ in range(steps):
        t = w.cells
        t[0], t[-1] = hot, cold
        w.cells = t
        assert w.step(dt, 1) is None
    t = w.cells
    t[0], t[-1] = hot, cold
    w.cells = t


def test_the_swept_steady_state_lands_on_the_layers_resistance():
    """a_layered_wall.rs:248-346: 400 s of a 24-cell wall clamped at 90 °C and 20 °C."""
    cells = 24
    w = wall(cells)
    hot, cold = 90.0 + 273.15, 20.0 + 273.15
    closed = chain(w)
    dt = 0.9 * w.max_stable_dt()
    clamped_march(w, int(400.0 / dt), dt, hot, cold)
    kz, t = w.coefficients()["kz"], w.cells
    drop = hot - cold
    want = drop / closed
    flux = kz[6] * DX * (t[5] - t[6])
    assert abs(flux / want - 1.0) < 1e-4
    running, worst = 0.0, 0.0
    for k in range(1, cells):
        running += 1.0 / (kz[k] * DX)
        worst = max(worst, abs(t[k] - (hot - want * running)))
    assert worst < 1e-4
    alu_path = (cells / 2.0 - 0.5) * 1e-3 / (ALU["conductivity"] * 1e-6)
    interface = hot - want * alu_path
    held = (hot - interface) / drop
    share = GLASS["conductivity"] / (GLASS["conductivity"] + ALU["conductivity"])
    assert abs(held - share) < 1e-9
    half_glass = 0.5e-3 / (GLASS["conductivity"] * 1e-6) * want
    assert half_glass / (hot - interface) > 6.0


def deposit_first_cell(w, joules, capacity):
    t = w.cells
    t[0] = t[0] + joules / capacity  # `deposit`: add_kelvin(c, J / C_c) (solid.rs:1346-1375)
    w.cells = t


def test_a_two_material_block_conserves_exactly():
    """a_layered_wall.rs:361-414: 30 J into the first aluminium cell of a 24-cell wall, 4000
    steps at 0.9 of the limit, and the books hold to 4000·ε."""
    w = wall(24)
    cap = w.coefficients()["capacity"]
    deposit_first_cell(w, 30.0, cap[0])
    opening = w.ledger()["total"]
    assert abs(opening - 30.0) < 1e-12 * 30.0
    dt = 0.9 * w.max_stable_dt()
    assert w.step(dt, 4000) is None
    closing = w.ledger()["total"]
    assert abs(closing - 30.0) < 4000 * np.finfo(float).eps * 30.0
    t = w.cells
    assert t[20] > t[23] + 1e-9
    want = 12.0 * 1e-9 * (2700.0 * 896.0 + 2510.0 * 858.0)
    assert abs(cap.sum() / want - 1.0) < 1e-12


@pytest.mark.gpu
def test_gpu_filled_wall_conserves_and_matches_the_oracle_bit_for_bit():
    o, g = wall(24), wall(24, gpu=True)
    cap = o.coefficients()["capacity"]
    for w in (o, g):
        deposit_first_cell(w, 30.0, cap[0])
    dt = 0.9 * o.max_stable_dt()
    assert g.max_stable_dt() == o.max_stable_dt()
    assert o.step(dt, 4000) is None
    assert g.step(dt, 4000) is None
    assert_bitexact("cells", g.cells, o.cells)
    assert abs(g.ledger()["total"] - 30.0) < 4000 * np.finfo(float).eps * 30.0


@pytest.mark.gpu
def test_gpu_clamped_wall_matches_the_oracle_bit_for_bit():
    """The first 3000 steps of the clamped march on the GPU, every clamp an upload of the wall."""
    o, g = wall(24), wall(24, gpu=True)
    dt = 0.9 * o.max_stable_dt()
    for w in (o, g):
        clamped_march(w, 3000, dt, 90.0 + 273.15, 20.0 + 273.15)
    assert_bitexact("cells", g.cells, o.cells)


@pytest.mark.gpu
def test_gpu_placeless_heat_leaves_a_two_material_block_uniform():
    """a_layered_wall.rs:421-446: 12 J off the plain channel is a uniform rise of J over the whole
    block's capacity (`pm_heat_absorb`)."""
    o, g = wall(24), wall(24, gpu=True)
    g.absorb(12.0)
    assert g.step(1e-6, 1) is None
    t = g.cells
    assert np.all(np.abs(t - t[0]) < 1e-12)
    rise = t[0] - T20
    want = 12.0 / o.coefficients()["capacity"].sum()
    assert abs(rise / want - 1.0) < 1e-12
