"""Parity of the GPU path with the oracle, through the C ABI.

Plain f64 forms: every field value bit-exact, ledgers within 1e-12 relative (the tolerance the
reference's own FP64 audit tests use). f32 forms: error bounds against the f64 oracle, stated in
each test.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import AL, T20, assert_bitexact, cavity_pair, dirichlet_films, hall_pair, heat_pair, rel

pytestmark = pytest.mark.gpu

LEDGER_TOL = 1e-12


# ------------------------------------------------------------------------------------------
# Solid3D
# ------------------------------------------------------------------------------------------
@pytest.mark.parametrize("mode", [(1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 1, 1)])
def test_heat_plain_mode_bitexact(mode):
    """solid_closed_forms.rs:46-77 setup: 7×5×3 aluminium, 25 steps at 0.8 × limit."""
    o, g = heat_pair((7, 5, 3), 2e-3, AL, T20)
    o.release_mode(mode, T20, 4.0)
    g.cells = o.cells
    dt = o.max_stable_dt() * 0.8
    assert g.max_stable_dt() == o.max_stable_dt()
    assert o.step(dt, 25) is None
    assert g.step(dt, 25) is None
    assert_bitexact("cells", g.cells, o.cells)
    # a zero-mean mode stores ~nothing net, so the ledger is judged against the heat that moved
    capacity = (AL["density"] * (2e-3 * 2e-3 * 2e-3)) * AL["specific_heat"]
    moved = capacity * np.abs(o.cells - T20).sum()
    assert abs(g.ledger()["total"] - o.ledger()["total"]) < LEDGER_TOL * moved


def test_heat_plain_dirichlet_block_audited_bitexact():
    """The 64³ heat block (Dirichlet faces, hot spot), 300 audited steps: bit-exact cells."""
    from pantometry_b200 import workloads as W

    cfg = W.heat_block(64)
    o, g = heat_pair(cfg["counts"], cfg["dx"], cfg["substance"], cfg["initial"], cfg["films"], cfg["cells"])
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-9)
    assert o.advance(dt, 300, tol=1e-9) is None
    assert g.step(dt, 300) is None
    assert_bitexact("cells", g.cells, o.cells)
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= LEDGER_TOL * lo["scale"]
    assert rel(lg["parts"][1], lo["lost"]) < LEDGER_TOL
    assert lg["steps"] == 300


def test_heat_plain_filled_block_bitexact():
    """A layered block (`fill`, harmonic face means) with Dirichlet films: bit-exact."""
    counts, dx = (12, 7, 5), 1e-3
    mask = np.zeros(counts[::-1], dtype=np.uint8)
    mask[:, :, 6:] = 1
    copper = dict(density=8960.0, conductivity=401.0, specific_heat=385.0, emissivity=0.0)
    steel = dict(density=7850.0, conductivity=45.0, specific_heat=490.0, emissivity=0.0)
    cells = 300.0 + 30.0 * np.random.default_rng(1).random(np.prod(counts))
    o, g = heat_pair(counts, dx, steel, 300.0, dirichlet_films(counts, dx), cells, fill=(mask.reshape(-1), copper))
    dt = 0.7 * o.max_stable_dt()
    assert g.max_stable_dt() == o.max_stable_dt()
    assert o.step(dt, 40) is None
    assert g.step(dt, 40) is None
    assert_bitexact("cells", g.cells, o.cells)


def test_heat_plain_refuses_past_the_limit_like_the_reference():
    o, g = heat_pair((5, 5, 5), 2e-3, AL, T20)
    dt = o.max_stable_dt() * 1.01
    vo, vg = o.step(dt), g.step(dt)
    assert vo is not None and vg is not None
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert vg[key] == vo[key], key


def test_heat_plain_audit_violation_matches_oracle():
    """A zero tolerance makes the first step that moves the books fail, with the same numbers."""
    from pantometry_b200 import workloads as W

    cfg = W.heat_block(16)
    o, g = heat_pair(cfg["counts"], cfg["dx"], cfg["substance"], cfg["initial"], cfg["films"], cfg["cells"])
    dt = 0.9 * o.max_stable_dt()
    vo = o.advance(dt, 50, tol=0.0)
    g.set_tolerance(0.0)
    vg = g.step(dt, 50)
    assert vo is not None and vg is not None
    assert vg["quantity"] == vo["quantity"] and vg["site"] == vo["site"]
    assert rel(vg["before"], vo["before"]) < LEDGER_TOL and rel(vg["after"], vo["after"]) < 1e-9
    assert vg["step"] >= 1


def test_heat_checkpoint_restore_roundtrip():
    from pantometry_b200 import workloads as W

    cfg = W.heat_block(16)
    _, g = heat_pair(cfg["counts"], cfg["dx"], cfg["substance"], cfg["initial"], cfg["films"], cfg["cells"])
    dt = 0.9 * g.max_stable_dt()
    g.step(dt, 7)
    g.checkpoint()
    saved, led = g.cells, g.ledger()
    g.step(dt, 5)
    g.restore()
    assert_bitexact("restored", g.cells, saved)
    assert g.ledger()["total"] == led["total"]


def test_heat_f32_tracks_f64_within_rounding():
    """runtime/gpu/tests/against_the_cpu.rs:99-139 and :180-208 bounds: worst deviation error
    after 60 steps on 16³ below 20·1e-7·√60 of the amplitude; the f32 books drift below 1e-6."""
    o, g = heat_pair((16, 16, 16), 1e-3, AL, T20, precision="f32")
    o.release_mode((1, 1, 1), T20 + 10.0, 5.0)
    g.cells = o.cells
    dt = 0.9 * o.max_stable_dt()
    l0 = g.ledger()
    assert rel(l0["total"], o.ledger()["total"]) < 1e-6
    assert o.step(dt, 60) is None
    assert g.step(dt, 60) is None
    err = np.abs((g.cells - T20) - (o.cells - T20)).max()
    assert err < 20e-7 * math.sqrt(60) * 5.0, err
    l1 = g.ledger()
    assert abs(l1["total"] - l0["total"]) < 1e-6 * max(l0["scale"], l1["scale"])


def test_heat_f32_dirichlet_block_error():
    from pantometry_b200 import workloads as W

    cfg = W.heat_block(32)
    o, g = heat_pair(cfg["counts"], cfg["dx"], cfg["substance"], cfg["initial"], cfg["films"], cfg["cells"],
                     precision="f32")
    dt = 0.9 * o.max_stable_dt()
    assert o.step(dt, 200) is None
    assert g.step(dt, 200) is None
    err = np.abs(g.cells - o.cells).max()
    assert err < 1e-4, err  # kelvin, on a 50 K spot
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-6 * lo["scale"]


# ------------------------------------------------------------------------------------------
# Hall
# ------------------------------------------------------------------------------------------
def test_hall_plain_mode_bitexact():
    """hall_closed_forms.rs:132-181 setup: 13 nodes across, (1,1,1) mode, 400 steps."""
    o, g = hall_pair(4.4, 3.1, 2.4, 13, mode=(1, 1, 1))
    dt = o.max_stable_dt() * 0.9
    assert g.max_stable_dt() == o.max_stable_dt()
    assert o.step(dt, 400) is None
    assert g.step(dt, 400) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy", "vz"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert rel(lg["total"], lo["total"]) < LEDGER_TOL
    assert rel(lg["parts"][1], lo["offset"]) < 1e-9


def test_hall_plain_noise_and_source_bitexact():
    """The acoustic_hall workload at 24³ (noise + Ricker point source), 300 audited steps."""
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(24, steps=300)
    w, h, d = cfg["size"]
    o, g = hall_pair(w, h, d, cfg["across"], cfg["speed"], cfg["density"], pressure=cfg["pressure"],
                     source=(cfg["source_node"], cfg["wave"]))
    dt = cfg["dt"]
    assert o.advance(dt, 300, tol=1e-9) is None
    g.set_tolerance(1e-9)
    assert g.step(dt, 300) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy", "vz"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    # judged against the largest contribution to the books, as `Ledger` judges a change
    scale = max(abs(lo["invariant"]), abs(lo["offset"]), abs(lo["injected"]))
    assert abs(lg["total"] - lo["total"]) <= LEDGER_TOL * scale


def test_hall_courant_refusal_matches():
    o, g = hall_pair(4.4, 3.1, 2.4, 13, mode=(1, 1, 1))
    dt = o.max_stable_dt() * 1.001
    vo, vg = o.step(dt), g.step(dt)
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert vg[key] == vo[key], key


def test_hall_checkpoint_restore():
    _, g = hall_pair(4.4, 3.1, 2.4, 13, mode=(1, 1, 1))
    dt = g.max_stable_dt() * 0.9
    g.step(dt, 3)
    g.checkpoint()
    f0 = g.fields()
    g.step(dt, 9)
    g.restore()
    f1 = g.fields()
    for k in ("p", "vx", "vy", "vz"):
        assert_bitexact(k, f1[k], f0[k])
    assert_bitexact("p_prev", f1["p_prev"], f0["p"])


def test_hall_f32_error_and_drift():
    o, g = hall_pair(4.4, 3.1, 2.4, 25, mode=(1, 1, 1), precision="f32")
    dt = o.max_stable_dt() * 0.9
    assert o.step(dt, 500) is None
    assert g.step(dt, 500) is None
    err = np.abs(g.fields()["p"] - o.fields()["p"]).max()
    assert err < 1e-4 * 2.0, err
    lo, lg = o.ledger(), g.ledger()
    assert rel(lg["total"], lo["total"]) < 1e-5


# ------------------------------------------------------------------------------------------
# Cavity
# ------------------------------------------------------------------------------------------
def test_cavity_plain_mode_bitexact():
    """against_closed_forms.rs:37-100 setup: 12×8×10, (1,1) mode, 300 steps at half the limit."""
    o, g = cavity_pair((12, 8, 10), 2e-3)
    dt = o.courant_limit() * 0.5
    assert g.courant_limit() == o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    assert_bitexact("hy after release", g.fields()["hy"], o.fields()["hy"])
    assert rel(g.ledger()["total"], o.ledger()["total"]) < LEDGER_TOL
    assert o.step(dt, 300) is None
    assert g.step(dt, 300) is None
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])
    assert rel(g.ledger()["total"], o.ledger()["total"]) < LEDGER_TOL


def test_cavity_plain_dielectric_obstacle_source_bitexact():
    """Per-cell ε_r, a solid obstacle and the dipole current together, audited."""
    counts, dx = (14, 11, 9), 1e-3
    rng = np.random.default_rng(7)
    eps = np.where(rng.random(np.prod(counts)) < 0.1, rng.uniform(1.0, 4.0, np.prod(counts)), 1.0)
    solid = np.zeros(counts[::-1], dtype=np.uint8)
    solid[2:4, 3:5, 9:11] = 1
    nx, ny, nz = counts
    edge = 5 + (nx + 1) * (5 + (ny + 1) * 4)
    o0 = oracle.Yee(counts, dx)
    dt = 0.9 * o0.courant_limit()
    t = (np.arange(400) + 0.5) * dt
    cur = 1e6 * np.exp(-((t - 60 * dt) / (15 * dt)) ** 2) * np.sin(2 * math.pi * t / (20 * dt))
    o, g = cavity_pair(counts, dx, eps_cells=eps, solid=solid.reshape(-1), source=(edge, cur))
    assert o.advance(dt, 400, tol=1e-9) is None
    g.set_tolerance(1e-9)
    assert g.step(dt, 400) is None
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= LEDGER_TOL * lo["scale"]


def test_cavity_courant_refusal_matches():
    o, g = cavity_pair((4, 4, 4), 1e-3)
    dt = o.courant_limit() * 1.0000001
    vo, vg = o.step(dt), g.step(dt)
    for key in ("quantity", "site", "before", "after", "scale", "tolerance"):
        assert vg[key] == vo[key], key


def test_cavity_f32_error_and_invariant():
    o, g = cavity_pair((24, 20, 22), 1e-3, precision="f32")
    dt = 0.99 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    l0 = g.ledger()["total"]
    assert o.step(dt, 500) is None
    assert g.step(dt, 500) is None
    err = np.abs(g.fields()["ey"] - o.fields()["ey"]).max()
    assert err < 1e-4, err
    assert rel(g.ledger()["total"], o.ledger()["total"]) < 1e-5
    assert rel(g.ledger()["total"], l0) < 1e-5


def test_ledger_is_reproducible_run_to_run():
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(32, steps=100)
    totals = []
    for _ in range(2):
        w, h, d = cfg["size"]
        _, g = hall_pair(w, h, d, cfg["across"], cfg["speed"], cfg["density"], pressure=cfg["pressure"],
                         source=(cfg["source_node"], cfg["wave"]), precision="f32")
        g.step(cfg["dt"], 100)
        totals.append(g.ledger()["total"])
    assert totals[0] == totals[1]


def test_cavity_plain_bitexact_at_128_repeated():
    """The source-driven vacuum cavity at 128³: large enough that the staged copies of the plane
    above take longer than a plane's work, which is where a missing wait would read stale data.
    Three fresh runs, each bit for bit against the oracle."""
    from pantometry_b200 import workloads as W

    n = 128
    cfg = W.yee_cavity(n, steps=40)
    o = oracle.Yee((n, n, n), cfg["dx"])
    o.set_source(cfg["edge"], cfg["current"])
    assert o.advance(cfg["dt"], 6, tol=1e-9) is None
    fo = o.fields()
    for _ in range(3):
        g = W.build_cavity(cfg, precision="f64")
        g.set_tolerance(1e-9)
        assert g.step(cfg["dt"], 6) is None
        fg = g.fields()
        for k in fo:
            assert_bitexact(k, fg[k], fo[k])


def test_cavity_f32_media_at_96_repeated():
    """The FP32 cp.async form (per-cell media) at 96³, three fresh runs against the oracle."""
    from pantometry_b200 import workloads as W

    n = 96
    cfg = W.yee_cavity(n, steps=40)
    eps = np.where(np.arange(n ** 3) % 11 == 0, 3.0, 1.0)
    o = oracle.Yee((n, n, n), cfg["dx"])
    o.set_cells(eps_r=eps)
    o.set_source(cfg["edge"], cfg["current"])
    assert o.step(cfg["dt"], 8) is None
    fo = o.fields()
    for _ in range(3):
        from pantometry_b200.domains import Cavity

        g = Cavity((n, n, n), cfg["dx"], precision="f32")
        g.fill_cells(eps_r=eps)
        g.set_source(cfg["edge"], cfg["current"])
        assert g.step(cfg["dt"], 8) is None
        fg = g.fields()
        for k in fo:
            scale = max(np.abs(fo[k]).max(), 1e-300)
            assert np.abs(fg[k] - fo[k]).max() < 1e-5 * scale, k
