"""Batched Solid3D ensembles (`pm_ensemble_*`) against the oracle, block by block.

The reference runs an ensemble as independent `Solid3D` samples (`Ensemble::run`,
crates/pantometry-core/src/ensemble.rs:102-140), so each block of a GPU ensemble must be exactly
what the oracle's `Solid3D` gives for that block alone:
  * plain f64 — every cell bit-exact after a run that replays a graph and single launches, under
    every brick shape; ledgers within 1e-12 of the scale;
  * f32 — within the single-block f32 bound (20·1e-7·√steps of the 50 K amplitude) and equal to
    the single-block f32 handle to f32 rounding; books drift below 1e-6.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import heat_pair
from pantometry_b200 import workloads as W

STEPS = 70  # one graph of 64 steps, then six single launches


def small_grids(count=9, seed=0x5EED, lo=3, hi=21):
    """Uneven blocks of lo..hi (3..21) cells per axis with the benchmark's draws; films cycle
    through insulated, Dirichlet (h = +inf) and a finite h, so all three film paths are covered."""
    from pantometry_b200.domains import Ensemble

    cfg = W.heat_ensemble(count=count, seed=seed, lo=lo, hi=hi)
    grids = []
    for g, src in enumerate(cfg["grids"]):
        grids.append({"counts": src["counts"], "dx": src["dx"], "substance": src["substance"],
                      "initial": src["initial"], "convection": (0.0, math.inf, 2.0e3)[g % 3]})
    for g, limit in zip(grids, Ensemble.max_stable_dt(grids)):
        g["dt"] = 0.9 * limit
    cells = [W.ensemble_cells(src) for src in cfg["grids"]]
    return grids, cells


def oracle_block(g):
    nx, ny, nz = g["counts"]
    dx, s = g["dx"], g["substance"]
    o = oracle.Heat((nx, ny, nz), dx, s["density"], s["conductivity"], s["specific_heat"], g["initial"])
    if g["convection"] != 0.0:
        areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
        for f in range(6):
            o.losing_from(f, g["initial"], g["convection"], areas[f])
    return o


def test_ensemble_limits_match_the_oracle_on_the_host():
    """pm_ensemble_max_stable_dt needs no device: each block's `max_stable_dt` exactly."""
    from pantometry_b200.domains import Ensemble

    grids, _ = small_grids(count=24)
    got = Ensemble.max_stable_dt(grids)
    for g, lim in zip(grids, got):
        assert lim == oracle_block(g).max_stable_dt(), g


def test_ensemble_workload_shapes():
    cfg = W.heat_ensemble()
    assert len(cfg["grids"]) == 512
    sizes = np.array([g["counts"] for g in cfg["grids"]])
    assert sizes.min() >= 16 and sizes.max() <= 128
    alpha = np.array([g["substance"]["conductivity"] / 1e6 for g in cfg["grids"]])
    assert alpha.min() >= 1e-6 and alpha.max() <= 1e-3
    assert cfg == W.heat_ensemble()  # seeded


@pytest.mark.gpu
def test_ensemble_f64_is_bit_exact_per_block_under_every_shape():
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids()
    want, books = [], []
    for g, c in zip(grids, cells):
        o = oracle_block(g)
        o.cells = c
        assert o.step(g["dt"], STEPS) is None
        want.append(o.cells)
        books.append(o.ledger())
    e = Ensemble(grids, precision="f64")
    # one cell per thread (x, planes), then the pair shapes (x, planes, y)
    for shape in ((32, 16), (16, 8), (64, 64), (32, 8), (16, 32, 32), (32, 64, 16), (64, 32, 8)):
        e.set_shape(*shape)
        e.upload(np.concatenate(cells))
        assert e.step(STEPS) is None
        got = e.download()
        for g in range(len(grids)):
            assert np.array_equal(e.block(got, g).view(np.uint64), want[g].view(np.uint64)), (shape, g)
        for led, o in zip(e.ledgers(), books):
            assert abs(led["total"] - o["total"]) <= 1e-12 * max(o["scale"], 1e-300), (led, o)
            assert abs(led["parts"][1] - o["lost"]) <= 1e-12 * max(o["scale"], 1e-300)
            assert led["steps"] == STEPS


@pytest.mark.gpu
def test_ensemble_f32_tracks_the_oracle_and_the_single_block_form():
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids()
    e = Ensemble(grids, precision="f32")
    e.upload(np.concatenate(cells))
    opening = e.ledgers()
    assert e.step(STEPS) is None
    got = e.download()
    bound = 20 * 1e-7 * math.sqrt(STEPS) * 50.0
    for g, (grid, c) in enumerate(zip(grids, cells)):
        o = oracle_block(grid)
        o.cells = c
        assert o.step(grid["dt"], STEPS) is None
        assert np.abs(e.block(got, g) - o.cells).max() < bound, g
        films = []
        if grid["convection"] != 0.0:
            nx, ny, nz = grid["counts"]
            dx = grid["dx"]
            areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
            films = [(f, grid["initial"], grid["convection"], areas[f]) for f in range(6)]
        _, single = heat_pair(grid["counts"], grid["dx"], grid["substance"], grid["initial"], films=films, cells=c,
                              precision="f32")
        assert single.step(grid["dt"], STEPS) is None
        assert np.abs(e.block(got, g) - single.cells).max() <= 1e-5, g
    for l0, l1 in zip(opening, e.ledgers()):
        assert abs(l1["total"] - l0["total"]) < 1e-6 * max(l0["scale"], l1["scale"], 1e-300)


@pytest.mark.gpu
def test_ensemble_autotune_keeps_state_and_books():
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids(count=12)
    e = Ensemble(grids, precision="f32")
    e.upload(np.concatenate(cells))
    assert e.step(10) is None
    before = e.download()
    books = e.ledgers()
    x, y, planes = e.autotune(trial_steps=3)
    assert (x, y, planes) == e.shape()
    assert x * y in (256, 1024) and planes in (8, 16, 32, 64)  # one cell or four cells per thread (f32)
    assert np.array_equal(e.download(), before)
    for a, b in zip(books, e.ledgers()):
        assert a["steps"] == b["steps"]
        assert abs(a["total"] - b["total"]) <= 1e-12 * max(a["scale"], 1e-300)
        assert a["parts"][1] == b["parts"][1]


@pytest.mark.gpu
def test_ensemble_refusals_and_audit_name_the_block():
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids(count=6)
    grids[4] = dict(grids[4], dt=grids[4]["dt"] / 0.9 * 1.01)
    e = Ensemble(grids, precision="f64")
    e.upload(np.concatenate(cells))
    v = e.step(1)
    assert v is not None and v["quantity"] == "Fourier number" and v["site"].startswith("block 4 ")
    assert all(led["steps"] == 0 for led in e.ledgers())  # refused before anything moved

    grids, cells = small_grids(count=6)
    e = Ensemble(grids, precision="f32")
    e.upload(np.concatenate(cells))
    e.set_tolerance(0.0)  # any rounding fails the audit
    v = e.step(5)
    assert v is not None and v["quantity"] == "energy" and v["site"].startswith("block ")
    failed = int(v["site"].split()[1])
    steps = [led["steps"] for led in e.ledgers()]
    assert steps[failed] == v["step"]  # that block stopped where it failed
    e.set_tolerance(-1.0)
    assert e.step(3) is None  # a new call clears the stop; every block steps again
    assert all(s1 == s0 + 3 for s0, s1 in zip(steps, (led["steps"] for led in e.ledgers())))


@pytest.mark.gpu
def test_ensemble_f32_tma_and_brick_kernels_agree():
    """32-wide bricks step with the TMA-staged kernel, 16- and 64-wide with the plain brick kernel,
    the quad shapes with four cells of a row per thread; all do heat_f32_step's arithmetic on the
    same padded rows, so the fields agree bit for bit."""
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids(count=10, seed=0xA11)
    runs = []
    # one cell per thread (x, planes), then the quad shapes (x, planes, y)
    for shape in ((32, 16), (16, 8), (64, 32), (32, 64), (16, 32, 64), (32, 64, 32), (128, 32, 8)):
        e = Ensemble(grids, precision="f32")
        e.set_shape(*shape)
        e.upload(np.concatenate(cells))
        assert e.step(STEPS) is None
        runs.append(e.download())
    for r in runs[1:]:
        assert np.array_equal(r, runs[0])


@pytest.mark.gpu
def test_ensemble_f32_tma_interior_and_face_bricks_agree():
    """Blocks of 65..99 cells per axis: the TMA kernel's 32-wide bricks include ones clear of every
    x face (the whole-stage interior form) beside ones holding a face (the general form, one x face
    selected per lane), with and without films; the plain brick kernel and the quad shapes agree
    bit for bit."""
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids(count=3, seed=0xB16, lo=65, hi=99)
    runs = []
    for shape in ((32, 16), (16, 8), (32, 64), (64, 64, 16), (128, 32, 8)):
        e = Ensemble(grids, precision="f32")
        e.set_shape(*shape)
        e.upload(np.concatenate(cells))
        assert e.step(12) is None
        runs.append(e.download())
    for r in runs[1:]:
        assert np.array_equal(r, runs[0])


@pytest.mark.gpu
def test_ensemble_quads_are_f32_only_and_pairs_f64_only():
    from pantometry_b200.domains import Ensemble

    grids, cells = small_grids(count=2)
    e = Ensemble(grids, precision="f64")
    with pytest.raises(Exception):
        e.set_shape(32, 32, 32)
    e.set_shape(32, 32, 8)  # the one-cell 32 × 8 shape by its extents
    assert e.shape() == (32, 8, 32)
    e.set_shape(32, 64, 16)
    assert e.shape() == (32, 16, 64)
    f = Ensemble(grids, precision="f32")
    with pytest.raises(Exception):
        f.set_shape(32, 64, 16)
