"""Hall with a sound speed per cubic block of nodes (the heterogeneous medium of the 1024³
configuration; `Hall` itself has one speed, crates/pantometry-acoustic/src/hall.rs:82-83).

The extension weights each node's pressure update by its own ρc² and its term of the invariant by
V/(2ρc²), so the discrete invariant is conserved exactly as in the uniform hall. The oracle
restates it (oracle.cpp `Hall::speed_at`); the GPU forms are checked against it: plain f64 bit for
bit, FP32 (both the TMA-staged form, x extent a multiple of 4, and the cp.async form) within the
f32 bounds.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, hall_pair


def speeds(nb, seed=7):
    from pantometry_b200 import workloads as W

    return W.Streams(seed, np.arange(nb, dtype=np.uint64)).range(300.0, 1500.0)


def blocks_for(nodes, block):
    return int(np.prod([(n + block - 1) // block for n in nodes]))


def test_speed_blocks_conserve_in_the_oracle():
    h = oracle.Hall(0.115, 0.115, 0.115, 24, 343.0, 1.2)
    h.release_mode((1, 1, 1), 1.0)
    h.set_speed_blocks(8, speeds(blocks_for(h.nodes, 8)))
    dt = 0.9 * h.max_stable_dt()
    assert dt < 0.9 * 0.005 / (343.0 * 3 ** 0.5)  # the limit follows the fastest block
    assert h.advance(dt, 400, tol=1e-9) is None


@pytest.mark.gpu
def test_speed_blocks_plain_bitexact():
    o, g = hall_pair(0.11, 0.09, 0.07, 23, density=1.2, mode=(1, 1, 1))
    sp = speeds(blocks_for(o.nodes, 8))
    o.set_speed_blocks(8, sp)
    g.set_speed_blocks(8, sp)
    dt = 0.9 * o.max_stable_dt()
    assert g.max_stable_dt() == o.max_stable_dt()
    assert o.step(dt, 200) is None
    assert g.step(dt, 200) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy", "vz"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * abs(lo["total"])


@pytest.mark.gpu
@pytest.mark.parametrize("across", [24, 23])  # TMA-staged and cp.async FP32 forms
def test_speed_blocks_f32(across):
    o, g = hall_pair(0.11, 0.09, 0.07, across, density=1.2, mode=(1, 1, 1), precision="f32")
    sp = speeds(blocks_for(o.nodes, 8))
    o.set_speed_blocks(8, sp)
    g.set_speed_blocks(8, sp)
    dt = 0.9 * o.max_stable_dt()
    assert o.step(dt, 300) is None
    assert g.step(dt, 300) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "vx", "vy", "vz"):
        scale = max(np.abs(fo[k]).max(), 1e-30)
        assert np.abs(fg[k] - fo[k]).max() < 1e-4 * scale, k
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-5 * lo["scale"]



def _sourced(order, precision, across):
    """A hall with a Ricker source at an off-centre node, the blocks set before or after the
    source (the source's share of the invariant follows its own block either way); `precision`
    None builds the oracle alone."""
    from pantometry_b200 import workloads as W

    o = oracle.Hall(0.115, 0.115, 0.115, across, 343.0, 1.2)
    doms = [o]
    if precision is not None:
        from pantometry_b200.domains import Hall

        doms.append(Hall(0.115, 0.115, 0.115, across, 343.0, 1.2, precision=precision))
    noise = W.Streams(11, np.arange(o.n, dtype=np.uint64)).range(-1e-3, 1e-3)
    sp = speeds(blocks_for(o.nodes, 8), seed=3)
    node = 5 + across * (6 + across * 9)
    dt = 0.5 * (0.115 / (across - 1)) / (float(sp.max()) * 3 ** 0.5)
    wave = W.ricker((np.arange(400) + 1.0) * dt, 2.0 / (40 * dt))
    for d in doms:
        d.release(noise)
        if order == "blocks_first":
            d.set_speed_blocks(8, sp)
            d.set_source(node, wave)
        else:
            d.set_source(node, wave)
            d.set_speed_blocks(8, sp)
    return doms, dt


@pytest.mark.parametrize("order", ["blocks_first", "source_first"])
def test_speed_blocks_with_source_conserve_in_the_oracle(order):
    (o,), dt = _sourced(order, None, 24)
    assert o.advance(dt, 300, tol=1e-9) is None
    led = o.ledger()
    # the injected work is booked as an entry of its own, so the scale covers it (here the net
    # total is the noise's energy, some 600 times smaller than what the source moved)
    assert led["scale"] >= abs(led["injected"]) > 100 * abs(led["total"])


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["blocks_first", "source_first"])
def test_speed_blocks_with_source_plain_bitexact(order):
    (o, g), dt = _sourced(order, "f64", 24)
    g.set_tolerance(1e-9)
    assert o.advance(dt, 300, tol=1e-9) is None
    assert g.step(dt, 300) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy", "vz"):
        assert_bitexact(k, fg[k], fo[k])
    lo, lg = o.ledger(), g.ledger()
    # the source's injected work is an entry of the ledger: its scale covers it
    assert abs(lg["scale"] - lo["scale"]) <= 1e-12 * lo["scale"]
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["blocks_first", "source_first"])
@pytest.mark.parametrize("across", [24, 23])
def test_speed_blocks_with_source_f32_audited(order, across):
    (o, g), dt = _sourced(order, "f32", across)
    g.set_tolerance(1e-5)
    assert o.advance(dt, 300, tol=1e-9) is None
    assert g.step(dt, 300) is None  # audited every step in FP64
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-5 * lo["scale"]
