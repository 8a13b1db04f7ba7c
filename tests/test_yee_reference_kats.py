"""The reference's own known-answer tests for open walls and lossy media, restated.

crates/pantometry-em/tests/against_closed_forms.rs:387-446 (a lossy box moves energy onto the
books: the field loses more than a tenth of its energy in 3000 steps and the ledger drifts less than
the leapfrog's own swing 2·sin(ωΔt/2) of the (1,0,1) mode, 12.8% there; a lossless box dissipates
exactly 0) and :448-512 (a line pulse of Hz leaves an open box: under 1% of its energy left after
2.5 light crossings, against more than 97% in a conducting box, with ∇·B kept to 1e3 of its start;
the reference reports 0.149% and 101% for that run). The oracle must pass them as the reference
does and reproduce the reported figures. The GPU forms must reproduce the oracle through the same
runs (plain f64 bit for bit) and pass the same bounds (FP32 too).
"""
import math

import numpy as np
import pytest

import oracle
from helpers import assert_bitexact

DX = 2e-3  # against_closed_forms.rs:11
C0 = 1.0 / math.sqrt(8.8541878128e-12 * 1.25663706212e-6)


def pulse_fields(shapes, counts, at, amplitude, width_cells):
    """`Cavity::pulse` (cavity.rs:610-626) on a fresh box: Hz += A·exp(−r²/w²), uniform along z,
    Gaussian in x and y about the cell-centre offsets; every other component zero."""
    nx, ny, nz = counts
    w = max(width_cells, 0.5)
    di = np.arange(nx) + 0.5 - at[0]
    dj = np.arange(ny) + 0.5 - at[1]
    r2 = (di[None, :] * di[None, :] + dj[:, None] * dj[:, None]) / (w * w)  # [j, i]
    plane = amplitude * np.exp(-r2)
    f = {k: np.zeros(v) for k, v in shapes.items()}
    f["hz"] = np.broadcast_to(plane, (nz + 1, ny, nx)).reshape(-1).copy()
    return f


def divergence(f, counts):
    """`peak_magnetic_divergence` (cavity.rs:963-993) from downloaded fields."""
    nx, ny, nz = counts
    hx = f["hx"].reshape(nz, ny, nx + 1)
    hy = f["hy"].reshape(nz, ny + 1, nx)
    hz = f["hz"].reshape(nz + 1, ny, nx)
    d = (hx[:, :, 1:] - hx[:, :, :-1]) + (hy[:, 1:, :] - hy[:, :-1, :]) + (hz[1:, :, :] - hz[:-1, :, :])
    return float(np.abs(d).max())


def crossing_steps(dt, cells=24):
    """The reference's loop: step while t < 2.5 crossings, t advancing by dt."""
    crossing = cells * DX / 299_792_458.0
    t, n = 0.0, 0
    while t < 2.5 * crossing:
        n += 1
        t += dt
    return n


def open_box(dom, counts, open_):
    if open_:
        for w in range(6):
            dom.set_boundary(w, "open")
    dt = dom.courant_limit() * 0.5
    dom.set_fields(pulse_fields(dom.shapes(), counts, (12, 12), 1.0, 2.0), started=True)
    return dt


def test_open_box_lets_a_pulse_out_in_the_oracle():
    counts = (24, 24, 24)
    kept = []
    for open_ in (False, True):
        o = oracle.Yee(counts, DX)
        dt = open_box(o, counts, open_)
        start = sum(o.energies())
        div0 = o.peak_divergence()
        assert o.step(dt, crossing_steps(dt)) is None
        assert o.peak_divergence() <= max(div0, 1e-12) * 1e3
        kept.append(sum(o.energies()) / start)
    assert kept[0] > 0.97, kept
    assert kept[1] < 0.01, kept
    # and the figures the reference reports for this run (against_closed_forms.rs:453-454):
    # "0.149% of the energy is left after two and a half crossings, against a conducting box's 101%"
    assert round(kept[1] * 100, 3) == 0.149, kept
    assert round(kept[0] * 100) == 101, kept


def lossy_run(make, steps=3000):
    c = make((10, 6, 10), sigma=5e-3)
    dt = c.courant_limit() * 0.5
    c.release_mode((1, 1), 1.0, dt)
    before = c.ledger()["total"]
    start = sum(c.energies())
    assert c.step(dt, steps) is None
    drift = abs(c.ledger()["total"] - before) / max(abs(before), 1e-300)
    f101 = 0.5 * C0 * math.sqrt((1.0 / (10 * DX)) ** 2 + (1.0 / (10 * DX)) ** 2)  # cavity_frequency
    swing = 2.0 * math.sin(2.0 * math.pi * f101 * dt / 2.0)
    return c, start, drift, swing


def test_lossy_box_books_what_it_takes_in_the_oracle():
    c, start, drift, swing = lossy_run(lambda counts, sigma: oracle.Yee(counts, DX, sigma=sigma))
    assert sum(c.energies()) < 0.9 * start
    assert drift < swing, (drift, swing)
    assert round(swing * 100, 1) == 12.8  # "12.8% here" (against_closed_forms.rs:421)
    clean = oracle.Yee((10, 6, 10), DX)
    dt = clean.courant_limit() * 0.5
    clean.release_mode((1, 1), 1.0, dt)
    assert clean.step(dt, 100) is None
    assert clean.ledger()["dissipated"] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_open_box_lets_a_pulse_out_on_the_gpu(precision):
    from pantometry_b200.domains import Cavity

    counts = (24, 24, 24)
    kept = []
    for open_ in (False, True):
        g = Cavity(counts, DX, precision=precision)
        dt = open_box(g, counts, open_)
        start = sum(g.energies())
        div0 = divergence(g.fields(), counts)
        n = crossing_steps(dt)
        assert g.step(dt, n) is None
        fg = g.fields()
        # the reference's bound is at f64 rounding; FP32 fields round ∇·B at about 1e-7 of the
        # pulse's unit amplitude (2.3e-7 measured), while a boundary writing to H would move it at
        # the size of the field itself
        bound = max(div0, 1e-12) * 1e3 if precision == "f64" else 1e-5 * 1.0
        assert divergence(fg, counts) <= bound
        kept.append(sum(g.energies()) / start)
        if precision == "f64":
            o = oracle.Yee(counts, DX)
            open_box(o, counts, open_)
            assert o.step(dt, n) is None
            fo = o.fields()
            for k in fo:
                assert_bitexact(k, fg[k], fo[k])
    assert kept[0] > 0.97, kept
    assert kept[1] < 0.01, kept


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_lossy_box_books_what_it_takes_on_the_gpu(precision):
    from pantometry_b200.domains import Cavity

    g, start, drift, swing = lossy_run(lambda counts, sigma: Cavity(counts, DX, sigma=sigma, precision=precision))
    assert sum(g.energies()) < 0.9 * start
    assert drift < swing, (drift, swing)
    if precision == "f64":
        o, _, _, _ = lossy_run(lambda counts, sigma: oracle.Yee(counts, DX, sigma=sigma))
        fo, fg = o.fields(), g.fields()
        for k in fo:
            assert_bitexact(k, fg[k], fo[k])
        assert g.ledger()["parts"][1] == pytest.approx(o.ledger()["dissipated"], rel=1e-12)
