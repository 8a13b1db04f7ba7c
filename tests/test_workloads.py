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
