"""The FP32 Hall form staged by TMA (halls whose x extent is a multiple of 4 nodes).

Those halls keep their face velocities padded to the node grid on the device and step with
`hall_tma_step`; every other hall, and the plain f64 form, keep the reference layout. Checked
here against the f64 oracle with the f32 bounds the other f32 tests use, through every host path
that touches the padded layout: release, download (fields back in the reference's shapes),
checkpoint/restore, the source extension and the audit. The same form against the cp.async
kernel on identical inputs is in test_zz_no_alloc.py.
"""
import numpy as np
import pytest

from helpers import hall_pair

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("across", [24, 32, 8])
def test_hall_tma_mode_error_and_drift(across):
    o, g = hall_pair(4.4, 3.1, 2.4, across, mode=(1, 1, 1), precision="f32")
    assert g.nodes[0] % 4 == 0
    dt = o.max_stable_dt() * 0.9
    assert o.step(dt, 500) is None
    assert g.step(dt, 500) is None
    fo, fg = o.fields(), g.fields()
    for k in ("p", "p_prev", "vx", "vy", "vz"):
        assert fg[k].shape == fo[k].shape, k
        scale = max(np.abs(fo[k]).max(), 1e-30)
        assert np.abs(fg[k] - fo[k]).max() < 1e-4 * max(scale, 2.0), k
    lo, lg = o.ledger(), g.ledger()
    assert rel(lg["total"], lo["total"]) < 1e-5


def test_hall_tma_noise_and_source_audited():
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(32, steps=300)
    w, h, d = cfg["size"]
    o, g = hall_pair(w, h, d, cfg["across"], cfg["speed"], cfg["density"], pressure=cfg["pressure"],
                     source=(cfg["source_node"], cfg["wave"]), precision="f32")
    assert o.advance(cfg["dt"], 300, tol=1e-9) is None
    # the f32 books of a ±1 mPa field move by about 1e-6 per step from rounding alone
    g.set_tolerance(1e-5)
    assert g.step(cfg["dt"], 300) is None
    fo, fg = o.fields(), g.fields()
    peak = np.abs(fo["p"]).max()
    assert np.abs(fg["p"] - fo["p"]).max() < 1e-5 * peak
    lo, lg = o.ledger(), g.ledger()
    scale = max(abs(lo["invariant"]), abs(lo["offset"]), abs(lo["injected"]))
    assert abs(lg["total"] - lo["total"]) < 1e-5 * scale


def test_hall_tma_checkpoint_restore():
    _, g = hall_pair(4.4, 3.1, 2.4, 24, mode=(1, 1, 1), precision="f32")
    dt = g.max_stable_dt() * 0.9
    g.step(dt, 3)
    g.checkpoint()
    f0 = g.fields()
    g.step(dt, 70)  # a graph of 64 steps and single launches
    g.restore()
    f1 = g.fields()
    for k in ("p", "vx", "vy", "vz"):
        assert np.array_equal(f1[k], f0[k]), k
    assert np.array_equal(f1["p_prev"], f0["p"])


def test_hall_tma_thin_halls():
    """Halls thinner than a tile in y or z (boxes reaching past every edge)."""
    for dims in ((0.7, 0.1, 0.1), (0.7, 0.3, 0.05), (1.5, 0.02, 0.4)):
        o, g = hall_pair(*dims, 8, mode=(1, 0, 0), precision="f32")
        dt = o.max_stable_dt() * 0.9
        vo, vg = o.step(dt, 100), g.step(dt, 100)
        assert (vo is None) == (vg is None), (dims, vo, vg)
        if vo is not None:  # the reference's own startup check refused it: so must the GPU
            assert vg["quantity"] == vo["quantity"] and vg["site"] == vo["site"]
            continue
        fo, fg = o.fields(), g.fields()
        for k in ("p", "vx", "vy", "vz"):
            assert fg[k].shape == fo[k].shape, (dims, k)
            if fo[k].size == 0:  # one node thick: no faces on that axis
                continue
            scale = max(np.abs(fo[k]).max(), 1e-30)
            assert np.abs(fg[k] - fo[k]).max() <= 1e-4 * max(scale, 2.0), (dims, k)


SHAPES = [(8, 2), (6, 2), (4, 3), (4, 2)]  # planes per stage × stages of the TMA kernel


@pytest.mark.parametrize("speed_blocks", [False, True], ids=["one-medium", "speed-blocks"])
def test_hall_tma_every_tile_shape_agrees_bit_for_bit(speed_blocks):
    """Every tile shape computes each node with the same expressions; only the staging differs. A
    hall with noise and the point source (and with speed blocks: the heterogeneous form) gives the
    same FP32 fields and books under every shape, over 70 steps (a 64-step graph and single ones),
    in chunks that exercise partial stages (28 planes)."""
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(28, steps=80)
    runs = []
    for shape in SHAPES:
        h = W.build_hall(cfg, precision="f32")
        if speed_blocks:
            h.set_speed_blocks(8, np.linspace(300.0, 343.0, 64))
        h.set_tile(*shape)
        assert h.tile() == shape
        h.set_tolerance(1e-6)
        assert h.step(cfg["dt"], 70) is None
        runs.append((h.fields(), h.ledger()))
    (f0, l0) = runs[0]
    for f, l in runs[1:]:
        for k in f0:
            assert np.array_equal(f[k].view(np.uint64), f0[k].view(np.uint64)), k
        assert l["total"] == l0["total"] or abs(l["total"] - l0["total"]) <= 1e-12 * l0["scale"]


def test_hall_autotune_keeps_state_books_and_source_clock():
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(36, steps=200)
    a = W.build_hall(cfg, precision="f32")
    b = W.build_hall(cfg, precision="f32")
    for h in (a, b):
        assert h.step(cfg["dt"], 30) is None
    shape = a.autotune(trial_steps=4)
    assert shape in SHAPES and a.tile() == shape
    b.set_tile(*shape)
    fa, fb = a.fields(), b.fields()
    for k in fa:
        assert np.array_equal(fa[k].view(np.uint64), fb[k].view(np.uint64)), k
    la, lb = a.ledger(), b.ledger()
    assert la["steps"] == lb["steps"] == 30 and la["total"] == lb["total"]
    for h in (a, b):
        assert h.step(cfg["dt"], 40) is None  # the source goes on from its 31st sample in both
    fa, fb = a.fields(), b.fields()
    for k in fa:
        assert np.array_equal(fa[k].view(np.uint64), fb[k].view(np.uint64)), k
