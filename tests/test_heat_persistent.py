"""Many steps of a small plain f64 block in one cooperative launch (`heat_plain_pair_steps`).

A 64³ block is launch-bound: its state (2 MiB) sweeps from L2 in about a microsecond, far below a
kernel launch. Calls of two or more steps on a small uniform block take every step in one launch
with one bounded grid-wide wait per step; one block keeps the books, auditing each step while the
others take the next (a failed audit ends the call with that step's state). These tests
check that path against the one-step kernels (a call of one step never takes it): the same fields
bit for bit, the same books, the same step when an audit fails, and a wait that runs out (its
budget set to zero) ending the call with PM_DEVICE_TIMEOUT while the handle stays usable.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, heat_pair
from pantometry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def block64():
    cfg = W.heat_block(64)
    s = cfg["substance"]
    return cfg, s


def pair(precision="f64"):
    cfg, s = block64()
    return heat_pair(cfg["counts"], cfg["dx"], s, cfg["initial"], cfg["films"], cfg["cells"], precision=precision)


def test_fp32_many_step_launch_matches_single_steps():
    """The FP32 quad form's many-step kernel runs the one-step kernel's arithmetic: the same
    deviations bit for bit, and within the FP32 bounds of the oracle."""
    o, g = pair("f32")
    _, g1 = pair("f32")
    dt = 0.9 * o.max_stable_dt()
    g.set_tolerance(1e-6)
    assert o.step(dt, 1100) is None
    assert g.step(dt, 1100) is None
    for _ in range(1100):
        assert g1.step(dt, 1) is None
    assert_bitexact("cells", g.cells, g1.cells)
    assert np.abs(g.cells - o.cells).max() < 1e-3
    lg, l1 = g.ledger(), g1.ledger()
    assert lg["steps"] == l1["steps"] == 1100
    assert abs(lg["total"] - l1["total"]) <= 1e-9 * lg["scale"]


def test_many_step_launch_matches_single_steps_and_the_oracle():
    o, g = pair()
    _, g1 = pair()
    dt = 0.9 * o.max_stable_dt()
    for h in (g, g1):
        h.set_tolerance(1e-9)
    assert o.step(dt, 1100) is None
    assert g.step(dt, 1100) is None  # two launches of the many-step path (1024 + 76 steps)
    for _ in range(1100):
        assert g1.step(dt, 1) is None
    assert_bitexact("cells", g.cells, o.cells)
    assert_bitexact("cells", g1.cells, g.cells)
    lg, l1, lo = g.ledger(), g1.ledger(), o.ledger()
    assert lg["steps"] == l1["steps"] == 1100
    assert abs(lg["total"] - lo["total"]) <= 1e-12 * lo["scale"]
    assert abs(lg["total"] - l1["total"]) <= 1e-12 * lo["scale"]
    assert lg["parts"][1] == l1["parts"][1] or abs(lg["parts"][1] - l1["parts"][1]) <= 1e-12 * lo["scale"]


def test_an_audit_failure_stops_the_call_after_that_step():
    """With a zero tolerance the first rounding fails the audit; the call stops with that step
    done and none after it: the fields are those of that many single steps, bit for bit."""
    _, g = pair()
    _, g1 = pair()
    dt = 0.9 * g.max_stable_dt()
    g.set_tolerance(0.0)  # any rounding fails
    v = g.step(dt, 50)
    assert v is not None and v["quantity"] == "energy" and 1 <= v["step"] <= 50
    for _ in range(v["step"]):
        assert g1.step(dt, 1) is None
    assert_bitexact("cells", g.cells, g1.cells)
    assert g.ledger()["steps"] == v["step"]


def test_a_wait_that_runs_out_ends_the_call_and_the_handle_goes_on():
    from pantometry_b200._native import PM_DEVICE_TIMEOUT, NativeError

    cfg, _ = block64()
    _, g = pair()
    dt = 0.9 * g.max_stable_dt()
    g.set_wait_budget(0)  # every block but the last to arrive gives up at once
    with pytest.raises(NativeError) as err:
        g.step(dt, 10)
    assert err.value.status == PM_DEVICE_TIMEOUT
    g.set_wait_budget(1 << 24)
    g.cells = cfg["cells"]  # a fresh state: the interrupted step's fields are incomplete
    o, _ = pair()
    assert o.step(dt, 10) is None
    assert g.step(dt, 10) is None
    assert_bitexact("cells", g.cells, o.cells)
