"""The FP32 cavity form staged by TMA (one uniform medium, or per-cell ε with no conductivity and
one μ; with or without obstacles).

Those cavities keep all six components on a padded node lattice and step with `yee_tma_step`;
release, the starting half step and the naive energies run the reference-layout kernels on a
relaid copy, and media with conductivity or per-cell μ (`fill_cells`) move the cavity back to the
reference layout and the cp.async kernel. Checked against the f64 oracle with the f32 bounds of the
other f32 tests through each of those paths.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import cavity_pair, rel

pytestmark = pytest.mark.gpu


def field_err(fo, fg):
    """Worst |GPU − oracle| of E and of H, each relative to its largest component."""
    scale = {q: max(max(np.abs(fo[q + a]).max() for a in "xyz"), 1e-30) for q in "eh"}
    worst = 0.0
    for k in fo:
        assert fg[k].shape == fo[k].shape, k
        worst = max(worst, np.abs(fg[k] - fo[k]).max() / scale[k[0]])
    return worst


@pytest.mark.parametrize("counts", [(24, 20, 22), (13, 9, 7), (33, 5, 40), (4, 4, 4)])
def test_yee_tma_mode_error_and_invariant(counts):
    o, g = cavity_pair(counts, 1e-3, precision="f32")
    dt = 0.99 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    l0 = g.ledger()["total"]
    assert rel(l0, o.ledger()["total"]) < 1e-6
    assert o.step(dt, 300) is None
    assert g.step(dt, 300) is None  # a graph of 64 steps and single launches
    assert field_err(o.fields(), g.fields()) < 1e-4
    assert rel(g.ledger()["total"], o.ledger()["total"]) < 1e-5
    assert rel(g.ledger()["total"], l0) < 1e-5
    eo, go = o.energies(), g.energies()
    assert rel(go[0], eo[0]) < 1e-4 and rel(go[1], eo[1]) < 1e-4


def test_yee_tma_obstacle_and_source_audited():
    counts, dx = (20, 17, 15), 1e-3
    solid = np.zeros(counts[::-1], dtype=np.uint8)
    solid[3:6, 4:7, 12:15] = 1
    nx, ny, nz = counts
    edge = 8 + (nx + 1) * (8 + (ny + 1) * 7)
    o0 = oracle.Yee(counts, dx)
    dt = 0.9 * o0.courant_limit()
    t = (np.arange(400) + 0.5) * dt
    cur = 1e6 * np.exp(-((t - 60 * dt) / (15 * dt)) ** 2) * np.sin(2 * math.pi * t / (20 * dt))
    o, g = cavity_pair(counts, dx, solid=solid.reshape(-1), source=(edge, cur), precision="f32")
    assert o.advance(dt, 400, tol=1e-9) is None
    g.set_tolerance(1e-5)
    assert g.step(dt, 400) is None
    assert field_err(o.fields(), g.fields()) < 1e-4
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-5 * lo["scale"]


def test_yee_tma_checkpoint_restore():
    _, g = cavity_pair((18, 12, 10), 1e-3, precision="f32")
    dt = 0.9 * g.courant_limit()
    g.release_mode((1, 1), 1.0, dt)
    g.step(dt, 5)
    g.checkpoint()
    f0 = g.fields()
    g.step(dt, 70)
    g.restore()
    f1 = g.fields()
    for k in f0:
        assert np.array_equal(f1[k], f0[k]), k


@pytest.mark.parametrize("kind", ["eps", "sigma"])
def test_yee_fill_cells_after_padded_steps(kind):
    """Per-cell media after a few padded steps. Per-cell ε alone stays on the padded layout (the
    TMA kernel reads each edge's gain and weighs its energy by it; audited every step); with
    conductivity the state carries over to the reference layout and the cp.async kernel."""
    counts, dx = (16, 12, 10), 1e-3
    cells = np.arange(np.prod(counts))
    o, g = cavity_pair(counts, dx, precision="f32")
    dt = 0.5 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    assert o.step(dt, 20) is None and g.step(dt, 20) is None
    if kind == "eps":
        eps = np.where(cells % 7 == 0, 2.5, 1.0)
        o.set_cells(eps_r=eps)
        g.fill_cells(eps_r=eps)
    else:
        sig = np.where(cells % 5 == 0, 0.02, 0.0)
        o.set_cells(sigma=sig)
        g.fill_cells(sigma=sig)
    # the new media change the field's energy off the books (the ledger holds the last step's
    # invariant until the next step, cavity.rs:1518-1524), so the audit starts one step later
    assert o.step(dt, 1) is None and g.step(dt, 1) is None
    if kind == "eps":
        g.set_tolerance(1e-5)
    assert o.step(dt, 99) is None and g.step(dt, 99) is None
    assert field_err(o.fields(), g.fields()) < 1e-4
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-5 * lo["scale"]


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_yee_upload_starts_fresh_books(precision):
    """Two runs from uploaded zero fields with the source on, audited: the second upload restarts
    the source's clock and the books, so it repeats the first run exactly (f64 bit for bit)."""
    from pantometry_b200 import workloads as W
    from pantometry_b200.domains import Cavity

    n = 20
    cfg = W.yee_cavity(n, steps=200)
    g = Cavity((n, n, n), cfg["dx"], precision=precision)
    g.set_source(cfg["edge"], cfg["current"])
    g.set_tolerance(1e-9 if precision == "f64" else 1e-5)
    zero = {k: np.zeros(v) for k, v in g.shapes().items()}
    runs = []
    for _ in range(2):
        g.set_fields(zero, started=False)
        assert g.step(cfg["dt"], 120) is None
        runs.append((g.fields(), g.ledger()))
    for k in runs[0][0]:
        assert np.array_equal(runs[0][0][k], runs[1][0][k]), k
    assert runs[0][1]["total"] == runs[1][1]["total"]
    o = oracle.Yee((n, n, n), cfg["dx"])
    o.set_source(cfg["edge"], cfg["current"])
    for _ in range(2):
        o.set_fields(zero, started=False)
        assert o.advance(cfg["dt"], 120, tol=1e-9) is None
    fo = o.fields()
    # each of E and H judged against its largest component (Hz of a z-dipole is zero to rounding)
    scale = {q: max(np.abs(fo[q + a]).max() for a in "xyz") for q in "eh"}
    for k in fo:
        if precision == "f64":
            assert np.array_equal(fo[k].view(np.uint64), runs[1][0][k].view(np.uint64)), k
        else:
            assert np.abs(fo[k] - runs[1][0][k]).max() <= 1e-4 * scale[k[0]], k


def _ledger_gap(runs, dt, calls, every):
    """Step the FP32 and f64 cavities side by side `every` steps at a time and return the worst
    |L32 − L64| / scale64 over the comparisons (scale: the f64 ledger's largest entry then)."""
    worst = 0.0
    for _ in range(calls):
        for c in runs.values():
            assert c.step(dt, every) is None
        a, b = runs["f32"].ledger(), runs["f64"].ledger()
        worst = max(worst, abs(a["total"] - b["total"]) / b["scale"])
    return worst


def test_yee_f32_ledger_within_1e6_of_f64_over_10000_steps():
    """The FP32 cavity driven by the soft dipole current. The source's near field (a 5³ box of
    lattice nodes around the source edge) is kept in f64 by the box kernel, so the ledger stays
    within 1e-6 of the f64 run's, compared every 10 steps over 10 000 steps and audited at 1e-6
    every step. With the whole field in f32 the same run ends a few 1e-6 away."""
    from pantometry_b200 import workloads as W

    n = 64
    cfg = W.yee_cavity(n, steps=10000)
    runs = {p: W.build_cavity(cfg, precision=p) for p in ("f32", "f64")}
    runs["f32"].set_tolerance(1e-6)
    assert _ledger_gap(runs, cfg["dt"], 1000, 10) <= 1e-6


def test_yee_f32_dielectric_source_ledger_within_1e6_of_f64():
    """The same with per-cell ε (ε_r in [1, 4] in 10% of the cells): the box's edges use their own
    f32 gains, as the update does, and weigh their energy by them."""
    from pantometry_b200 import workloads as W

    cfg = W.dielectric_cavities(count=1, n=40, steps=3000)
    runs = {p: W.build_dielectric_cavity(cfg, 0, precision=p) for p in ("f32", "f64")}
    runs["f32"].set_tolerance(1e-6)
    assert _ledger_gap(runs, cfg["dt"], 300, 10) <= 1e-6


def test_yee_f32_near_field_checkpoint_restore_is_exact():
    """The box's f64 values and the source's clock are part of the state: a checkpoint taken during
    the pulse and restored gives the same fields and books bit for bit on the second run."""
    from pantometry_b200 import workloads as W

    cfg = W.yee_cavity(32, steps=400)
    g = W.build_cavity(cfg, precision="f32")
    assert g.step(cfg["dt"], 70) is None
    g.checkpoint()
    runs = []
    for _ in range(2):
        assert g.step(cfg["dt"], 90) is None  # a graph of 64 steps and single launches
        runs.append((g.fields(), g.ledger()))
        g.restore()
        g.checkpoint()
    (fa, la), (fb, lb) = runs
    for k in fa:
        assert np.array_equal(fa[k].view(np.uint64), fb[k].view(np.uint64)), k
    assert la["total"] == lb["total"] and la["parts"] == lb["parts"]


def test_yee_f32_source_near_a_wall_keeps_the_plain_form():
    """A source too close to a wall for the box (it must lie a node inside the walls with the ring
    of edges on its high sides) steps in plain FP32 and still matches the oracle."""
    counts, dx = (12, 10, 9), 1e-3
    nx, ny, nz = counts
    edge = 2 + (nx + 1) * (5 + (ny + 1) * 4)  # Ez at node (2, 5, 4): the box would reach node 0
    o0 = oracle.Yee(counts, dx)
    dt = 0.9 * o0.courant_limit()
    t = (np.arange(200) + 0.5) * dt
    cur = 1e6 * np.exp(-((t - 40 * dt) / (10 * dt)) ** 2) * np.sin(2 * math.pi * t / (20 * dt))
    o, g = cavity_pair(counts, dx, source=(edge, cur), precision="f32")
    assert o.advance(dt, 200, tol=1e-9) is None
    g.set_tolerance(1e-4)
    assert g.step(dt, 200) is None
    assert field_err(o.fields(), g.fields()) < 1e-4


def test_yee_f32_invariant_against_f64_over_2000_steps():
    """A source-free mode at 48³: the FP32 run's invariant stays within 1e-6 of the f64 run's."""
    from pantometry_b200.domains import Cavity

    n = 48
    runs = {}
    for prec in ("f32", "f64"):
        g = Cavity((n, n, n), 1e-3, precision=prec)
        dt = 0.99 * g.courant_limit()
        g.release_mode((1, 1), 1.0, dt)
        g.set_tolerance(1e-5 if prec == "f32" else 1e-9)
        assert g.step(dt, 2000) is None
        runs[prec] = g.ledger()
    assert abs(runs["f32"]["total"] - runs["f64"]["total"]) < 1e-6 * runs["f64"]["scale"]


@pytest.mark.parametrize("media", [False, True], ids=["one-medium", "dielectric"])
def test_yee_tma_every_tile_shape_agrees_bit_for_bit(media):
    """Every tile shape of a form computes each edge and face with the same expressions: the same
    FP32 fields under every shape, with the source's near field in f64, over 70 steps (a 64-step
    graph and single launches) of a cavity whose planes do not fill whole stages."""
    from pantometry_b200 import workloads as W

    n = 30
    shapes = [(4, 2), (3, 2)] if media else [(3, 2), (4, 2), (3, 3)]
    if media:
        cfg = W.dielectric_cavities(count=1, n=n, steps=100)
    else:
        cfg = W.yee_cavity(n, steps=100)
    runs = []
    for shape in shapes:
        c = W.build_dielectric_cavity(cfg, 0, precision="f32") if media else W.build_cavity(cfg, precision="f32")
        c.set_tile(*shape)
        assert c.tile() == shape
        c.set_tolerance(1e-6)
        assert c.step(cfg["dt"], 70) is None
        runs.append((c.fields(), c.ledger()))
    f0, l0 = runs[0]
    for f, l in runs[1:]:
        for k in f0:
            assert np.array_equal(f[k].view(np.uint64), f0[k].view(np.uint64)), k
        # the fields agree bit for bit; the books are FP64 sums taken in each shape's block order,
        # and the total is a small difference of the energy and what the walls and media took, so
        # it agrees to the sums' rounding (about 1e-11 of the scale measured), not bit for bit
        assert abs(l["total"] - l0["total"]) <= 1e-9 * l0["scale"]


def test_yee_autotune_keeps_state_books_and_source_clock():
    from pantometry_b200 import workloads as W

    cfg = W.yee_cavity(32, steps=200)
    a = W.build_cavity(cfg, precision="f32")
    b = W.build_cavity(cfg, precision="f32")
    for c in (a, b):
        assert c.step(cfg["dt"], 30) is None
    shape = a.autotune(trial_steps=4)
    assert shape in [(3, 2), (4, 2), (3, 3)] and a.tile() == shape
    b.set_tile(*shape)
    la, lb = a.ledger(), b.ledger()
    assert la["steps"] == lb["steps"] == 30 and la["total"] == lb["total"]
    for c in (a, b):
        assert c.step(cfg["dt"], 40) is None
    fa, fb = a.fields(), b.fields()
    for k in fa:
        assert np.array_equal(fa[k].view(np.uint64), fb[k].view(np.uint64)), k


def _split_runs(make, steps, dt, books=1e-9):
    runs = []
    for split in (True, False):
        c = make()
        c.set_wall_split(split)
        assert c.step(dt, steps) is None  # a 64-step graph and single launches
        assert c.wall_split() == split
        runs.append((c.fields(), c.ledger()))
    (fa, la), (fb, lb) = runs
    for k in fa:
        assert np.array_equal(fa[k].view(np.uint64), fb[k].view(np.uint64)), k
    # the books: f32 stage sums of the same terms grouped another way, then FP64
    assert abs(la["total"] - lb["total"]) <= books * lb["scale"]


@pytest.mark.parametrize("media", [False, True], ids=["one-medium", "dielectric"])
def test_yee_wall_pass_agrees_with_whole_tiles(media):
    """nx a multiple of 32 and ny of 8: the TMA kernel's wall pass steps the lattice's last column
    and row, and the fields equal those of tiles over the whole lattice bit for bit, with the
    dipole's near field in f64."""
    from pantometry_b200 import workloads as W

    n = 32
    if media:
        cfg = W.dielectric_cavities(count=1, n=n, steps=100)
        make = lambda: W.build_dielectric_cavity(cfg, 0, precision="f32")  # noqa: E731
    else:
        cfg = W.yee_cavity(n, steps=100)
        make = lambda: W.build_cavity(cfg, precision="f32")  # noqa: E731
    _split_runs(make, 70, cfg["dt"])


def test_yee_wall_pass_with_open_and_magnetic_walls_loss_and_obstacles():
    """A lossy 64×40×20 cavity released in a mode, with an open x wall and a magnetic y wall (which
    leave the wall edges of the last column and row non-zero) and obstacles: the wall pass and
    whole tiles agree bit for bit."""
    from pantometry_b200.domains import Cavity

    counts, dx = (64, 40, 20), 1e-3
    nx, ny, nz = counts
    dt = 0.9 * Cavity(counts, dx, precision="f32").courant_limit()
    solid = np.zeros((nz, ny, nx), dtype=np.uint8)
    solid[4:9, 30:39, 50:63] = 1

    def make():
        c = Cavity(counts, dx, sigma=2e-3, precision="f32")
        c.release_mode((1, 2), 1.0, dt)
        c.obstruct(solid)
        c.set_boundary("XHigh", "open")
        c.set_boundary("YHigh", "magnetic")
        return c

    # this cavity's FP32 books hold about 1e-7 of the f64 run's; the two groupings of the f32
    # stage sums differ by a few 1e-9
    _split_runs(make, 70, dt, books=2e-8)


def test_yee_wall_pass_only_where_the_tiles_fit():
    from pantometry_b200.domains import Cavity

    assert Cavity((32, 16, 9), 1e-3, precision="f32").wall_split()
    assert not Cavity((30, 16, 9), 1e-3, precision="f32").wall_split()
    assert not Cavity((32, 12, 9), 1e-3, precision="f32").wall_split()
    assert not Cavity((32, 16, 9), 1e-3, precision="f64").wall_split()
