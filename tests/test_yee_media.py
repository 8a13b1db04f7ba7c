"""Cavities of mixed media on the GPU: per-cell ε_r, μ_r and σ in any combination.

`Cavity::fill` gives every edge the mean ε and σ of its four cells and every face the mean μ of
its two (crates/pantometry-em/src/cavity.rs:348-458); the update forms g/μ per face
(cavity.rs:1355) and the semi-implicit gain and decay per edge (cavity.rs:1391-1397). The GPU path
forms those coefficients once per step size and the step reads them; σ = 0 everywhere skips the
decay and the Joule term, one μ on every face skips the g/μ array. The plain f64 form must stay
bit-exact with the oracle in every combination, also when the step size changes between calls;
the FP32 form stays within f32 bounds and passes the FP64 audit. A lossy cavity's ledger holds only
to the leapfrog's own swing in the reference (its Joule term takes E at the midpoint against the
naive energy; crates/pantometry-em/tests/against_closed_forms.rs:387-430), so the cases with σ are
compared bit for bit and on their ledger totals, not audited per step.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact

COUNTS = (13, 10, 9)
DX = 1e-3
CASES = ["eps", "sigma", "mu", "all", "one_mu"]
LOSSY = ("sigma", "all")


def media(case, seed=5):
    n = int(np.prod(COUNTS))
    rng = np.random.default_rng(seed)
    kw = {}
    if case in ("eps", "all", "one_mu"):
        kw["eps_r"] = np.where(rng.random(n) < 0.2, rng.uniform(1.0, 4.0, n), 1.0)
    if case in ("sigma", "all"):
        kw["sigma"] = np.where(rng.random(n) < 0.2, rng.uniform(0.0, 0.05, n), 0.0)  # S/m
    if case in ("mu", "all"):
        kw["mu_r"] = np.where(rng.random(n) < 0.2, rng.uniform(1.0, 3.0, n), 1.0)
    if case == "one_mu":
        kw["mu_r"] = np.full(n, 2.0)  # one μ on every face, not the constructor's
    return kw


def pair(case, precision):
    from pantometry_b200.domains import Cavity

    o = oracle.Yee(COUNTS, DX)
    g = Cavity(COUNTS, DX, precision=precision)
    kw = media(case)
    o.set_cells(**kw)
    g.fill_cells(**kw)
    dt = 0.9 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    nx, ny, nz = COUNTS
    edge = 4 + (nx + 1) * (6 + (ny + 1) * 3)
    t = (np.arange(600) + 0.5) * dt
    cur = 1e5 * np.exp(-((t - 40 * dt) / (12 * dt)) ** 2) * np.sin(2 * np.pi * t / (20 * dt))
    o.set_source(edge, cur)
    g.set_source(edge, cur)
    return o, g, dt


def test_media_cases_in_the_oracle():
    for case in CASES:
        o = oracle.Yee(COUNTS, DX)
        o.set_cells(**media(case))
        dt = 0.9 * o.courant_limit()
        o.release_mode((1, 1), 1.0, dt)
        if case in LOSSY:
            assert o.step(dt, 100) is None
            assert o.ledger()["dissipated"] > 0.0, case
        else:
            assert o.advance(dt, 100, tol=1e-9) is None, case


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_media_plain_bitexact(case):
    o, g, dt = pair(case, "f64")
    tol = -1.0 if case in LOSSY else 1e-9
    g.set_tolerance(tol)
    assert (o.step(dt, 150) if case in LOSSY else o.advance(dt, 150, tol=tol)) is None
    assert g.step(dt, 150) is None
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]
    # a new step size: the coefficients are formed again (and a graph run of 70 steps uses them)
    g.set_tolerance(-1.0)
    assert o.step(0.8 * dt, 70) is None
    assert g.step(0.8 * dt, 70) is None
    assert o.step(dt, 3) is None
    assert g.step(dt, 3) is None
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_media_f32_within_bounds_and_audited(case):
    o, g, dt = pair(case, "f32")
    g.set_tolerance(-1.0 if case in LOSSY else 1e-5)
    assert o.step(dt, 200) is None
    assert g.step(dt, 200) is None  # audited every step in FP64
    fo, fg = o.fields(), g.fields()
    for fam in (("ex", "ey", "ez"), ("hx", "hy", "hz")):
        scale = max(float(np.abs(fo[k]).max()) for k in fam)
        for k in fam:
            assert np.abs(fg[k] - fo[k]).max() < 1e-4 * scale, (case, k)
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-5 * lo["scale"]
