"""Scene-level drop-in: single-domain world scenes run frame by frame as `World::run` runs them
(crates/pantometry-world/src/lib.rs:3204-3215) under the multirate schedule, through
`pantometry_b200.scenes`.

The scenes are the reference's own files, read into tests/golden/scenes.json by
tests/golden/make_scenes.py (each entry names the file it came from). The oracle's domains must
hold each scene's conservation tolerance across every window; the GPU's plain f64 domains must
reproduce the oracle's frames (the same substeps, the same ledgers to 1e-12, the final state bit
for bit); the FP32 forms must hold the scenes whose tolerance is an FP32 one (1e-6).
"""
import json
import os

import numpy as np
import pytest

import oracle
from pantometry_b200 import scenes as S

with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes.json")) as _f:
    SCENES = {k: v["scene"] for k, v in json.load(_f).items()}
ACOUSTIC_FP32 = [k for k, v in SCENES.items() if v["domains"][0]["kind"] in ("hall", "room", "cavity")]


def oracle_domain(scene):
    """The same domain built from the oracle's restatements, released with the same host fields."""
    d = scene["domains"][0]
    if d["kind"] == "block":
        m, fills, t = S.block_layout(d)
        counts = tuple(d["cells"])
        o = oracle.Heat(counts, d["cell_mm"] * 1e-3, m["density"], m["conductivity"], m["specific_heat"],
                        S.celsius(d["initial_c"]), emissivity=m["emissivity"])
        for mask, sub in fills:
            o.fill(mask, sub["density"], sub["conductivity"], sub["specific_heat"], sub["emissivity"])
        o.cells = t
        return o
    if d["kind"] == "hall":
        o = oracle.Hall(d["width_m"], d["height_m"], d["depth_m"], d["nodes_across"], S.AIR["speed"], S.AIR["density"])
        o.release(S.hall_mode_profile(o.nodes, o.dx, d["mode"], d["amplitude_pa"]))
        return o
    if d["kind"] == "room":
        o = oracle.Room(d["width_m"], d["height_m"], d["cells_across"], 1.0, S.AIR["density"], S.AIR["speed"])
        o.release(S.room_release(o.cells, o.dx, d["release"]))
        return o
    o = oracle.Yee(tuple(d["cells"]), d["cell_mm"] * 1e-3)
    steps = max(int(np.ceil(S.window(scene) / o.courant_limit())), 1)
    o.release_mode(tuple(d["mode"]), d["amplitude_v_per_m"], S.window(scene) / steps)
    return o


def test_the_fixture_holds_the_reference_files():
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes.json")) as f:
        entries = json.load(f)
    for k, v in entries.items():
        assert v["source"].startswith("crates/pantometry-world/scenes/") and v["source"].endswith(".json"), k
        assert len(v["scene"]["domains"]) == 1, k


def test_substeps_follow_the_reference_rule():
    assert S.substeps_for(1e-3, 14.58e-6) == 69  # the 1 m tube's window (acoustic lib.rs:938-966)
    assert S.substeps_for(1.0, 0.3) == 4  # sim.rs:1352-1354
    assert S.substeps_for(1.0, float("inf")) == 1 and S.substeps_for(0.0, 1.0) == 1


@pytest.mark.parametrize("name", list(SCENES))
def test_the_scenes_hold_in_the_oracle(name):
    scene = SCENES[name]
    out = S.run(scene, oracle_domain(scene))
    assert out["violation"] is None, out["violation"]
    assert len(out["frames"]) == scene["frames"] + 1
    assert all(n >= 1 for n in out["substeps"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SCENES))
def test_the_scenes_on_the_gpu_match_the_oracle(name):
    scene = SCENES[name]
    g = S.build(scene, precision="f64")
    o = oracle_domain(scene)
    got, want = S.run(scene, g), S.run(scene, o)
    assert got["violation"] is None and want["violation"] is None
    assert got["substeps"] == want["substeps"]
    for fg, fo in zip(got["frames"], want["frames"]):
        assert abs(fg["total"] - fo["total"]) <= 1e-12 * max(fo["scale"], 1e-300)
    if SCENES[name]["domains"][0]["kind"] == "block":
        assert np.array_equal(g.cells.view(np.uint64), o.cells.view(np.uint64))
    else:
        fg, fo = g.fields(), o.fields()
        for k in fo:
            assert np.array_equal(fg[k].view(np.uint64), fo[k].view(np.uint64)), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", ACOUSTIC_FP32)
def test_the_scenes_hold_in_fp32(name):
    scene = SCENES[name]
    out = S.run(scene, S.build(scene, precision="f32"))
    assert out["violation"] is None, out["violation"]
    want = S.run(scene, oracle_domain(scene))
    for fg, fo in zip(out["frames"], want["frames"]):
        assert abs(fg["total"] - fo["total"]) <= 1e-6 * fo["scale"]
