"""Magnetic and open (Mur) walls on the GPU against the oracle (cavity.rs:1074-1236).

After each step the walls are applied one at a time in the reference's order: conducting walls
held at zero, magnetic walls mirrored from one cell in, open walls by Mur's first-order update
from the previous step's E (or held at zero before any step has run). Mur's history is what the
last step left, also after E was rewritten between steps (a second release), as in the reference.
Plain f64 is compared bit for bit; FP32 (both the padded TMA form and the per-cell-media form)
within the f32 bounds of the other tests. With obstacles the walls come before the obstacles'
edges are zeroed, as in the reference.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, cavity_pair

pytestmark = pytest.mark.gpu

MIXED = {0: 1, 1: 1, 4: 2, 5: 2}  # x walls magnetic, z walls open, y walls conducting
OPEN = {w: 2 for w in range(6)}


def with_walls(o, g, walls):
    for w, kind in walls.items():
        o.set_boundary(w, kind)
        g.set_boundary(w, kind)


def e_h_err(fo, fg):
    scale = {q: max(max(np.abs(fo[q + a]).max() for a in "xyz"), 1e-300) for q in "eh"}
    return max(np.abs(fg[k] - fo[k]).max() / scale[k[0]] for k in fo)


@pytest.mark.parametrize("walls", [MIXED, OPEN], ids=["mixed", "open"])
def test_walls_plain_bitexact_through_a_second_release(walls):
    o, g = cavity_pair((14, 11, 12), 1e-3)
    with_walls(o, g, walls)
    dt = 0.9 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    assert o.step(dt, 70) is None and g.step(dt, 70) is None  # a graph of 64 steps and single launches
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])
    # E rewritten between steps: the next step's open walls take the history of before
    o.release_mode((2, 1), 0.5, dt)
    g.release_mode((2, 1), 0.5, dt)
    assert o.step(dt, 40) is None and g.step(dt, 40) is None
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])
    eo, eg = o.energies(), g.energies()
    assert abs(eg[0] - eo[0]) <= 1e-12 * abs(eo[0]) and abs(eg[1] - eo[1]) <= 1e-12 * abs(eo[1])


def test_open_box_lets_energy_out_and_conducting_keeps_it():
    """against_closed_forms.rs:463 in spirit: the same released mode in a conducting box and in an
    open one; after two crossings the open box holds far less (GPU and oracle alike)."""
    kept = {}
    for name, walls in (("conducting", {}), ("open", OPEN)):
        o, g = cavity_pair((16, 16, 16), 1e-3)
        with_walls(o, g, walls)
        dt = 0.5 * o.courant_limit()
        o.release_mode((1, 1), 1.0, dt)
        g.release_mode((1, 1), 1.0, dt)
        start = sum(g.energies())
        steps = int(2 * 16 * 1e-3 / 299_792_458.0 / dt)
        assert o.step(dt, steps) is None and g.step(dt, steps) is None
        kept[name] = sum(g.energies()) / start
        assert abs(sum(g.energies()) - sum(o.energies())) <= 1e-12 * sum(o.energies())
    assert kept["conducting"] > 0.9
    assert kept["open"] < 0.5 * kept["conducting"]


@pytest.mark.parametrize("media", [False, True], ids=["tma", "media"])
def test_walls_f32(media):
    counts = (20, 15, 17)
    o, g = cavity_pair(counts, 1e-3, precision="f32")
    if media:
        eps = np.where(np.arange(np.prod(counts)) % 5 == 0, 2.0, 1.0)
        o.set_cells(eps_r=eps)
        g.fill_cells(eps_r=eps)
    with_walls(o, g, MIXED)
    dt = 0.9 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    assert o.step(dt, 200) is None and g.step(dt, 200) is None
    assert e_h_err(o.fields(), g.fields()) < 1e-4


@pytest.mark.parametrize("walls", [MIXED, OPEN], ids=["mixed", "open"])
def test_obstacles_with_magnetic_and_open_walls_bitexact(walls):
    """Obstacles beside magnetic and open walls: the reference applies the walls, keeps E as Mur's
    history and only then zeroes the obstacles' edges (cavity.rs:1497-1499), so an obstacle edge on
    a wall's inner plane feeds Mur's update before it is zeroed. Solid cells touch the x, y and z
    walls' inner planes; plain f64 bit for bit through a release between runs, FP32 within bounds."""
    counts = (12, 10, 9)
    solid = np.zeros(counts[::-1], dtype=np.uint8)
    solid[0:2, 3:5, 1:3] = 1      # against the z-low wall and the x-low wall's inner planes
    solid[4:6, 8:10, 9:11] = 1    # against the y-high and x-high walls
    solid[7:9, 0:2, 5:7] = 1      # against the z-high and y-low walls
    dt = None
    for precision in ("f64", "f32"):
        o, g = cavity_pair(counts, 1e-3, solid=solid.reshape(-1), precision=precision)
        with_walls(o, g, walls)
        dt = 0.9 * o.courant_limit()
        o.release_mode((1, 1), 1.0, dt)
        g.release_mode((1, 1), 1.0, dt)
        assert o.step(dt, 70) is None and g.step(dt, 70) is None  # a graph of 64 steps and single launches
        if precision == "f64":
            fo, fg = o.fields(), g.fields()
            for k in fo:
                assert_bitexact(k, fg[k], fo[k])
            o.release_mode((2, 1), 0.5, dt)
            g.release_mode((2, 1), 0.5, dt)
            assert o.step(dt, 40) is None and g.step(dt, 40) is None
            fo, fg = o.fields(), g.fields()
            for k in fo:
                assert_bitexact(k, fg[k], fo[k])
        else:
            assert e_h_err(o.fields(), g.fields()) < 1e-4


def test_walls_set_after_obstructed_steps():
    """Open walls set on an obstructed cavity that has already stepped: the history is the field
    the last step left (its obstacles' edges already zeroed), and the runs go on together."""
    counts = (10, 9, 8)
    solid = np.zeros(counts[::-1], dtype=np.uint8)
    solid[3:5, 3:5, 3:5] = 1
    o, g = cavity_pair(counts, 1e-3, solid=solid.reshape(-1))
    dt = 0.9 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    assert o.step(dt, 10) is None and g.step(dt, 10) is None
    with_walls(o, g, OPEN)
    assert o.step(dt, 30) is None and g.step(dt, 30) is None
    fo, fg = o.fields(), g.fields()
    for k in fo:
        assert_bitexact(k, fg[k], fo[k])
