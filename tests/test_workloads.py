"""The synthetic-input generator's Rng restatement agrees with the oracle's, draw for draw."""
import numpy as np

import oracle
from pantometry_b200 import workloads as W


def test_streams_match_the_oracle_rng():
    idx = np.array([0, 1, 2, 17, 12345, 2**40 + 3], dtype=np.uint64)
    s = W.Streams(W.SEED, idx)
    draws = np.stack([s.unit() for _ in range(4)], axis=1)
    for row, i in enumerate(idx):
        assert list(draws[row]) == oracle.rng_for_index_units(W.SEED, int(i), 4)


def test_workload_shapes():
    cfg = W.heat_block(64)
    assert cfg["cells"].shape == (64 ** 3,)
    assert 349.0 < cfg["cells"].max() < 350.0
    h = W.acoustic_hall(16, steps=10)
    assert h["pressure"].shape == (16 ** 3,) and np.abs(h["pressure"]).max() <= 1e-3
    e = W.heat_ensemble(8)
    assert all(16 <= n <= 128 for g in e["grids"] for n in g["counts"])


def test_heat_block_baseline_holds_its_audit():
    """Config 1's CPU baseline leg (bench.py --workload heat): the oracle's audited
    `Simulation::advance` over the heat block at 0.9 of its limit keeps the books at 1e-9, and the
    record carries the keys of a bench line's cpu_baseline."""
    import bench

    cfg = W.heat_block(16, steps=20)
    out = bench.cpu_baseline_heat(cfg, 20)  # asserts the audit held on every step
    assert out["value"] > 0.0 and out["cores"] == 1 and out["kind"] == "port"
    assert out["unit"] == bench.UNIT and "20 audited" in out["sample"]


def test_heat_reference_arm_prints_its_line():
    """`bench.py --workload heat --impl reference` runs the oracle's audited steps of the heat block
    on the host cores and prints one line with the reference arm's keys."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--workload", "heat", "--impl", "reference",
                          "--n", "16", "--timesteps", "10", "--steps", "1"],
                         capture_output=True, text=True, timeout=300, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0.0 and line["dtype"] == "f64"
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_cavity_sample_holds_its_audit():
    """The cavity's CPU baseline and reference arm (bench.py): the oracle's audited steps of the
    vacuum cavity with its soft source, on independent copies, one per thread."""
    import bench

    rate, secs = bench.cavity_sample(16, 5, copies=2)  # asserts every step's audit held
    assert rate > 0.0 and secs > 0.0
    out = bench.cpu_baseline_cavity(16, 5)
    assert out["cores"] == 1 and out["kind"] == "port" and out["value"] > 0.0


def test_mix_sample_holds_its_audit():
    """The mix's CPU baseline and reference arm (bench.py): the oracle's audited speed-block hall and
    dielectric cavity, independent pairs one per thread, weighted by the mix's cells."""
    import bench

    value, t_hall, t_cav = bench.mix_sample(1024 ** 3, 64 * 128 ** 3, n_sample=16, sample_steps=3, copies=2)
    assert value > 0.0 and t_hall > 0.0 and t_cav > 0.0
