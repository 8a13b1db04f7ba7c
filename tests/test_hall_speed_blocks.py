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
    assert abs(lg["total"] - lo["total"]) < 1e-5 * abs(lo["total"])
