"""The wide `Solid3D` steps against one cell per thread on the same block: four adjacent cells of a
row per thread in the FP32 form (heat_f32_quad_step, rows of a multiple of 4 cells) and two in the
plain f64 form (heat_plain_pair_step, even rows), both for blocks of one material. Each does
`Solid3D::step`'s arithmetic (crates/pantometry-thermal/src/solid.rs:1773-1826) in the same order and
roundings as the one-cell kernel, so the fields agree bit for bit under insulated faces, Dirichlet
films (h = +inf) and films of finite h on some faces; the books, summed in another order, agree to
1e-12 of the ledger's scale. The plain form is also bit for bit with the oracle, the FP32 form
within its bounds, both audited every step.
"""
import numpy as np
import pytest

from helpers import dirichlet_films, heat_pair

pytestmark = pytest.mark.gpu

ALUMINIUM = dict(density=2700.0, conductivity=167.0, specific_heat=896.0, emissivity=0.0)


def films_of(kind, counts, dx):
    nx, ny, nz = counts
    areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
    if kind == "insulated":
        return []
    if kind == "dirichlet":
        return dirichlet_films(counts, dx, 300.0)
    return [(0, 280.0, 50.0, areas[0]), (1, 320.0, 2000.0, areas[1]), (3, 290.0, 10.0, areas[3]),
            (4, 310.0, 500.0, areas[4])]


@pytest.mark.parametrize("counts", [(4, 3, 5), (8, 8, 8), (64, 20, 17), (100, 9, 33), (6, 7, 4)])
@pytest.mark.parametrize("kind", ["insulated", "dirichlet", "finite"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_wide_and_single_cells_agree(counts, kind, precision):
    dx = 1e-3
    cells = 300.0 + 30.0 * np.random.default_rng(sum(counts)).random(int(np.prod(counts)))
    films = films_of(kind, counts, dx)
    runs = []
    for per_thread in (4 if precision == "f32" else 2, 1):
        o, g = heat_pair(counts, dx, ALUMINIUM, 300.0, films, cells, precision=precision)
        g.set_cells_per_thread(per_thread)
        g.set_tolerance(1e-6 if precision == "f32" else 1e-9)
        dt = 0.9 * g.max_stable_dt()
        assert g.step(dt, 70) is None  # a captured graph of 64, then six single launches
        runs.append((g.cells, g.ledger()))
    assert o.step(dt, 70) is None
    (wide, lw), (single, ls) = runs
    bad = np.flatnonzero(wide.view(np.uint64) != single.view(np.uint64))
    assert bad.size == 0, f"{bad.size} cells differ, first at {bad[0]}"
    assert abs(lw["total"] - ls["total"]) <= 1e-12 * max(ls["scale"], 1e-300)
    if precision == "f64":  # the plain form is the reference's arithmetic: bit for bit with the oracle
        assert np.array_equal(wide.view(np.uint64), o.cells.view(np.uint64))
        lo = o.ledger()
        assert abs(lw["total"] - lo["total"]) <= 1e-12 * max(lo["scale"], 1e-300)
    else:
        assert np.abs(wide - o.cells).max() < 1e-4  # kelvin, on a 30 K spread


def test_cells_per_thread_is_one_or_a_width_of_the_form():
    _, g = heat_pair((8, 4, 4), 1e-3, ALUMINIUM, 300.0, precision="f32")
    with pytest.raises(Exception):
        g.set_cells_per_thread(2)
    g.set_cells_per_thread(1)
    g.set_cells_per_thread(4)
    _, g = heat_pair((8, 4, 4), 1e-3, ALUMINIUM, 300.0, precision="f64")
    with pytest.raises(Exception):
        g.set_cells_per_thread(3)
    g.set_cells_per_thread(1)
    g.set_cells_per_thread(2)
    g.set_cells_per_thread(4)


def test_step_kernel_names_each_form():
    """pm_heat_step_kernel names the kernel a call would run and its launches, running nothing."""
    from helpers import dirichlet_films

    counts, dx = (64, 20, 17), 1e-3
    _, g = heat_pair(counts, dx, ALUMINIUM, 300.0, dirichlet_films(counts, dx, 300.0))
    assert g.step_kernel(1) == ("heat_plain_quad_step", 1)
    name, launches = g.step_kernel(2500)  # a small block: many steps a cooperative launch
    assert name.startswith("heat_plain_pair_steps") and launches == 3
    g.set_cells_per_thread(2)
    assert g.step_kernel(1) == ("heat_plain_pair_step", 1)
    g.set_cells_per_thread(1)
    assert g.step_kernel(1) == ("heat_plain_step", 1)
    _, h = heat_pair((63, 20, 17), dx, ALUMINIUM, 300.0)
    assert h.step_kernel(5) == ("heat_plain_step", 5)  # odd rows: one cell per thread
    _, f = heat_pair(counts, dx, ALUMINIUM, 300.0, precision="f32")
    assert f.step_kernel(1) == ("heat_tma_step (TMA-staged)", 1)
    assert f.step_kernel(0) == ("none", 0)


@pytest.mark.parametrize("counts", [(64, 20, 17), (100, 9, 33), (8, 8, 8), (4, 3, 5)])
@pytest.mark.parametrize("kind", ["insulated", "dirichlet", "finite"])
def test_plain_four_two_and_one_cells_agree_with_the_oracle(counts, kind):
    """Four cells of a row per thread in plain f64 (heat_plain_quad_step), one step a call (a call of
    more steps on a block this small takes the many-step cooperative kernel): bit for bit with the
    pair and one-cell forms and the oracle, books within 1e-12 of the oracle's scale."""
    dx = 1e-3
    cells = 300.0 + 30.0 * np.random.default_rng(sum(counts) + 1).random(int(np.prod(counts)))
    films = films_of(kind, counts, dx)
    runs = []
    for per_thread in (4, 2, 1):
        o, g = heat_pair(counts, dx, ALUMINIUM, 300.0, films, cells)
        g.set_cells_per_thread(per_thread)
        g.set_tolerance(1e-9)
        dt = 0.9 * g.max_stable_dt()
        for _ in range(20):
            assert g.step(dt, 1) is None
        runs.append((g.cells, g.ledger()))
    assert o.step(dt, 20) is None
    lo = o.ledger()
    for cells_now, led in runs:
        assert np.array_equal(cells_now.view(np.uint64), o.cells.view(np.uint64))
        assert abs(led["total"] - lo["total"]) <= 1e-12 * max(lo["scale"], 1e-300)


def test_plain_four_cells_many_steps_past_the_cooperative_size():
    """256 × 128 × 129 cells (just over 2^22): a call of 70 steps runs heat_plain_quad_step (a
    64-step graph and six single launches), bit for bit with the oracle."""
    counts, dx = (256, 128, 129), 1e-3
    cells = 300.0 + 30.0 * np.random.default_rng(3).random(int(np.prod(counts)))
    o, g = heat_pair(counts, dx, ALUMINIUM, 300.0, films_of("dirichlet", counts, dx), cells)
    assert g.step_kernel(70) == ("heat_plain_quad_step", 70)
    g.set_tolerance(1e-9)
    dt = 0.9 * g.max_stable_dt()
    assert g.step(dt, 70) is None
    assert o.step(dt, 70) is None
    assert np.array_equal(g.cells.view(np.uint64), o.cells.view(np.uint64))
    lg, lo = g.ledger(), o.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * max(lo["scale"], 1e-300)
