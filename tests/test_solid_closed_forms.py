"""More of `Solid3D`'s closed forms, restating crates/pantometry-thermal/tests/solid_closed_forms.rs
on the oracle (the eigen-decay, axis, conservation and limit tests are restated with the other pins):
  * placeless heat off the bus leaves the block uniform, risen by J over the block's capacity
    (:254-294);
  * a hot spot spreads the same way along all six arms, to 1e-12 of its rise, and the diagonal sits
    between the air and an arm (:296-339);
  * a block one cell thick is a bar: its mode's amplification is 1 + F·λ with λ = −4 sin²(π/2n),
    and 30 steps give the amplitude to 1e-12 (:341-371);
  * the field reads each cell back at its centre and stays inside the block's range outside it
    (:373-416);
  * at the reported limit the sharpest mode is marginal and oscillatory (amplification in
    [−1, −0.5)) and holds over 60 steps; at three times it diverges and is refused (:503-541).
The device's placeless heat, deposits and plain stencil are checked against the oracle bit for bit
elsewhere (`test_layered_wall.py`, `test_voids_gaps_sources.py`, `test_gpu_parity.py`).
"""
import math

import numpy as np

import oracle
from pantometry_b200.scenes import ALUMINIUM_6061 as AL  # substance.rs:362-373

C20 = 20.0 + 273.15


def block(counts, dx_mm):
    """solid_closed_forms.rs:13-21: aluminium 6061 at 20 °C in cubes of dx_mm."""
    return oracle.Heat(counts, dx_mm * 1e-3, AL["density"], AL["conductivity"], AL["specific_heat"], C20,
                       emissivity=AL["emissivity"])


def test_placeless_heat_leaves_the_block_uniform():  # :254-294
    b = block((4, 3, 2), 3.0)
    b.absorb(12.0)
    assert b.step(1e-5) is None
    t = b.cells
    assert np.all(np.abs(t - t[0]) < 1e-12)
    volume = 4 * 3 * 2 * (3e-3) ** 3
    capacity = (AL["density"] * volume) * AL["specific_heat"]  # Substance::heat_capacity (substance.rs:219-222)
    assert abs((t[0] - C20) - 12.0 / capacity) < 1e-12


def test_a_hot_spot_spreads_the_same_way_along_every_axis():  # :296-339
    b = block((9, 9, 9), 1.0)
    t = b.cells
    c = 4 + 9 * (4 + 9 * 4)
    t[c] += 2.0 / b.coefficients()["capacity"][c]  # deposit: add_kelvin(c, J/C) (solid.rs:1368-1375)
    b.cells = t
    assert b.step(2e-6, 5) is None
    g = b.cells.reshape(9, 9, 9)
    arms = [g[4, 4, 3], g[4, 4, 5], g[4, 3, 4], g[4, 5, 4], g[3, 4, 4], g[5, 4, 4]]
    for arm in arms:
        assert arm > C20 + 1e-6
        assert abs(arm - arms[0]) < 1e-12 * (arms[0] - C20)
    corner = g[4, 3, 3]
    assert C20 < corner < arms[0]


def test_one_cell_thick_reduces_to_a_bar():  # :341-371
    n = 12
    b = block((n, 1, 1), 2.0)
    b.release_mode((1, 0, 0), C20, 5.0)
    dt = 2e-5
    alpha = AL["conductivity"] / (AL["density"] * AL["specific_heat"])
    f = alpha * dt / (2e-3 * 2e-3)  # Solid3D::fourier_number (solid.rs:1423-1428)
    lam = -4.0 * math.sin(math.pi / (2.0 * n)) ** 2
    per_step = 1.0 + f * lam
    assert abs(b.mode_amplification((1, 0, 0), dt) - per_step) < 1e-15
    assert b.step(dt, 30) is None
    assert abs(b.mode_amplitude((1, 0, 0)) - 5.0 * per_step ** 30) < 1e-12 * 5.0


def test_the_field_reads_back_the_cells_and_clamps_at_the_faces():  # :373-416
    b = block((5, 4, 3), 2.0)
    b.release_mode((1, 1, 1), C20, 10.0)
    t = b.cells
    dx = 2e-3
    got = b.sample((0.5 * dx, 0.5 * dx, 0.5 * dx), (4.5 * dx, 3.5 * dx, 2.5 * dx), (5, 4, 3))
    assert np.abs(got - t).max() < 1e-9  # each cell centre reads its cell
    for p in ((-1.0, 0.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.0, -1.0), (1.0, 1.0, 1.0)):
        v = b.sample(p, p, (1, 1, 1))[0]
        assert t.min() - 1e-9 <= v <= t.max() + 1e-9


def test_the_limit_is_where_the_sharpest_mode_stops_growing():  # :503-541
    n = 5
    sharpest = (n - 1, n - 1, n - 1)
    b = block((n, n, n), 2.0)
    b.release_mode(sharpest, C20, 1.0)
    limit = b.max_stable_dt()
    assert b.step(limit, 60) is None
    assert abs(b.mode_amplitude(sharpest)) <= 1.0 + 1e-9
    per_step = block((n, n, n), 2.0).mode_amplification(sharpest, limit)
    assert -1.0 <= per_step < -0.5  # marginal and oscillatory
    runaway = block((n, n, n), 2.0).mode_amplification(sharpest, 3.0 * limit)
    assert abs(runaway) > 1.0 and abs(runaway) ** 60 > 1e6
    assert block((n, n, n), 2.0).step(3.0 * limit)["quantity"] == "Fourier number"
