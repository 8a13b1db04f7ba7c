"""scene::capture's field sampling (crates/pantometry-scene/src/lib.rs:347-420): each domain's
`ScalarField::at` over an extent's sample grid. The oracle's samplers are pinned by the properties
the reference states for them (a sample on a cell centre or node is that value exactly, void reads
NaN, points outside are clamped, one sample along an axis is its middle); the device samplers are
bit for bit with the oracle in f64 and within f32 rounding in FP32, on the resident fields.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import heat_pair


def heat_oracle(counts=(6, 5, 4), dx=1e-3, void=None, seed=1):
    o = oracle.Heat(counts, dx, 1000.0, 100.0, 1000.0, 300.0)
    if void is not None:
        o.empty(void)
    cells = 300.0 + 40.0 * np.random.default_rng(seed).random(int(np.prod(counts)))
    o.cells = cells
    return o, cells


def test_heat_samples_on_cell_centres_are_the_cells():
    """solid.rs:2041-2043: a sample at a cell centre is that cell exactly; a grid laid over the centres
    lands on them to the rounding of lo + (hi − lo)·f."""
    o, cells = heat_oracle()
    got = o.sample((0.5e-3, 0.5e-3, 0.5e-3), (5.5e-3, 4.5e-3, 3.5e-3), (6, 5, 4))
    assert np.allclose(got, cells, rtol=1e-12, atol=0)
    one = o.sample((2.5e-3, 1.5e-3, 0.5e-3), (2.5e-3, 1.5e-3, 0.5e-3), (1, 1, 1))[0]
    assert one == cells[2 + 6 * 1]  # exactly on a centre: that cell, bit for bit


def test_heat_samples_clamp_outside_and_blend_between():
    o, cells = heat_oracle()
    nx, ny, nz = 6, 5, 4
    c = cells.reshape(nz, ny, nx)
    # far outside every face: the corner cells, clamped rather than extrapolated
    got = o.sample((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0), (2, 2, 2))
    assert got[0] == c[0, 0, 0] and got[-1] == c[-1, -1, -1]
    # halfway between two cell centres along x: the mean of the two
    mid = o.sample((1.0e-3, 0.5e-3, 0.5e-3), (1.0e-3, 0.5e-3, 0.5e-3), (1, 1, 1))[0]
    assert mid == pytest.approx(0.5 * (c[0, 0, 0] + c[0, 0, 1]), rel=1e-15)


def test_heat_samples_in_void_are_nan_and_neighbours_renormalise():
    """solid.rs:2034-2044, 2069-2079: a sample in a void cell is NaN; one leaning on a void
    neighbour takes the solid corners' values alone."""
    counts = (6, 5, 4)
    void = np.zeros(counts[::-1], dtype=np.uint8)
    void[:, :, 3] = 1  # the x = 3 column of cells
    o, cells = heat_oracle(counts, void=void.reshape(-1))
    c = cells.reshape(4, 5, 6)
    assert math.isnan(o.sample((3.5e-3, 2.5e-3, 1.5e-3), (3.5e-3, 2.5e-3, 1.5e-3), (1, 1, 1))[0])
    # a quarter of the way from cell 2 towards void cell 3: cell 2 alone
    v = o.sample((2.75e-3, 2.5e-3, 1.5e-3), (2.75e-3, 2.5e-3, 1.5e-3), (1, 1, 1))[0]
    assert v == c[1, 2, 2]


def test_one_sample_along_an_axis_is_its_middle():
    """lib.rs:398-406: a single sample along an axis is taken at the middle of the extent."""
    o, cells = heat_oracle()
    a = o.sample((0.5e-3, 0.5e-3, 0.0), (0.5e-3, 0.5e-3, 3.0e-3), (1, 1, 1))[0]
    b = o.sample((0.5e-3, 0.5e-3, 1.5e-3), (0.5e-3, 0.5e-3, 1.5e-3), (1, 1, 1))[0]
    assert a == b


def test_hall_samples_on_nodes_are_the_pressures_and_blend_linearly():
    h = oracle.Hall(0.01, 0.008, 0.006, 6, 343.0, 1.2)
    nx, ny, nz = h.nodes
    dx = 0.01 / (nx - 1)
    pr = np.random.default_rng(2).uniform(-1.0, 1.0, nx * ny * nz)
    h.release(pr)
    got = h.sample((0.0, 0.0, 0.0), ((nx - 1) * dx, (ny - 1) * dx, (nz - 1) * dx), (nx, ny, nz))
    assert np.allclose(got, pr, rtol=0, atol=1e-15)
    g = pr.reshape(nz, ny, nx)
    mid = h.sample((0.5 * dx, 0.0, 0.0), (0.5 * dx, 0.0, 0.0), (1, 1, 1))[0]
    assert mid == pytest.approx(0.5 * (g[0, 0, 0] + g[0, 0, 1]), rel=1e-14)


def test_cavity_samples_are_the_length_of_the_cells_edges():
    """cavity.rs:197-206, 735-742: |E| from the cell's own x, y and z edges, nearest cell."""
    y = oracle.Yee((5, 4, 3), 1e-3)
    dt = 0.9 * y.courant_limit()
    y.release_mode((1, 1), 1.0, dt)
    f = y.fields()
    nx, ny, nz = 5, 4, 3
    got = y.sample((0.5e-3, 0.5e-3, 0.5e-3), (4.5e-3, 3.5e-3, 2.5e-3), (nx, ny, nz))
    ex = f["ex"].reshape(nz + 1, ny + 1, nx)
    ey = f["ey"].reshape(nz + 1, ny, nx + 1)
    ez = f["ez"].reshape(nz, ny + 1, nx + 1)
    want = np.array([math.sqrt((ex[k, j, i] ** 2 + ey[k, j, i] ** 2) + ez[k, j, i] ** 2)
                     for k in range(nz) for j in range(ny) for i in range(nx)])
    assert np.array_equal(got, want)


EXTENTS = [((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (7, 5, 3)), ((-2e-3, 1e-4, 3e-4), (9e-3, 7.3e-3, 2e-3), (13, 1, 9)),
           ((1.7e-3, 2.2e-3, 0.9e-3), (1.7e-3, 2.2e-3, 0.9e-3), (1, 1, 1))]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_heat_device_samples_match_the_oracle(precision):
    counts, dx = (16, 12, 10), 1e-3
    void = np.zeros(counts[::-1], dtype=np.uint8)
    void[3:6, 4:8, 7:11] = 1
    cells = 300.0 + 40.0 * np.random.default_rng(5).random(int(np.prod(counts)))
    o, g = heat_pair(counts, dx, dict(density=1000.0, conductivity=100.0, specific_heat=1000.0), 300.0,
                     cells=cells, precision=precision)
    o.empty(void.reshape(-1))
    g.empty(void.reshape(-1))
    o.cells = cells
    g.cells = cells
    for lo, hi, n in EXTENTS + [((0.5e-3, 0.5e-3, 0.5e-3), (15.5e-3, 11.5e-3, 9.5e-3), counts)]:
        want, got = o.sample(lo, hi, n), g.sample(lo, hi, n)
        assert np.array_equal(np.isnan(got), np.isnan(want))
        if precision == "f64":
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        else:
            ok = ~np.isnan(want)
            assert np.abs(got[ok] - want[ok]).max() < 1e-4  # kelvin: f32 deviations of ~40 K


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_hall_device_samples_match_the_oracle(precision):
    from pantometry_b200.domains import Hall

    n = 12
    w = 0.011
    o = oracle.Hall(w, 0.008, 0.006, n, 343.0, 1.2)
    g = Hall(w, 0.008, 0.006, n, 343.0, 1.2, precision=precision)
    pr = np.random.default_rng(3).uniform(-1.0, 1.0, int(np.prod(o.nodes)))
    o.release(pr)
    g.release(pr)
    for lo, hi, cnt in EXTENTS:
        want, got = o.sample(lo, hi, cnt), g.sample(lo, hi, cnt)
        if precision == "f64":
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        else:
            assert np.abs(got - want).max() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("counts,precision", [((10, 8, 6), "f64"), ((10, 8, 6), "f32"), ((32, 16, 9), "f32")])
def test_cavity_device_samples_match_the_oracle(counts, precision):
    """The f64 form on the reference layout, the FP32 form on the padded lattice (and with the wall
    split where nx is a multiple of 32), after 30 steps of a released mode."""
    from pantometry_b200.domains import Cavity

    dx = 1e-3
    o = oracle.Yee(counts, dx)
    g = Cavity(counts, dx, precision=precision)
    dt = 0.9 * o.courant_limit()
    o.release_mode((1, 1), 1.0, dt)
    g.release_mode((1, 1), 1.0, dt)
    assert o.step(dt, 30) is None and g.step(dt, 30) is None
    nx, ny, nz = counts
    for lo, hi, cnt in EXTENTS + [((0.5e-3, 0.5e-3, 0.5e-3), ((nx - 0.5) * dx, (ny - 0.5) * dx, (nz - 0.5) * dx), counts)]:
        want, got = o.sample(lo, hi, cnt), g.sample(lo, hi, cnt)
        if precision == "f64":
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        else:
            assert np.abs(got - want).max() <= 1e-5 * max(np.abs(want).max(), 1e-30)


@pytest.mark.gpu
def test_sample_refuses_a_mismatched_buffer():
    from pantometry_b200._native import NativeError
    from pantometry_b200.domains import Cavity

    g = Cavity((4, 4, 4), 1e-3)
    with pytest.raises(NativeError):
        g.sample((0, 0, 0), (1, 1, 1), (0, 2, 2))


@pytest.mark.gpu
def test_capture_draws_placed_fields_only():
    """scene::capture: a placed field becomes a panel of its samples; a field with no extent is not
    drawn (lib.rs:343-345)."""
    from pantometry_b200 import scenes
    from pantometry_b200.domains import Cavity, Hall

    hall = Hall(0.01, 0.008, 0.006, 6, 343.0, 1.2)
    cav = Cavity((6, 5, 4), 1e-3)
    extent = {"min": (0.0, 0.0, 0.0), "max": (0.004, 0.003, 0.002), "samples": (5, 4, 3)}
    frame = scenes.capture({"hall": hall, "cavity": cav}, {"hall": {"extent": extent}, "cavity": {}}, 0.25)
    assert frame["time_s"] == 0.25
    assert [p["name"] for p in frame["panels"]] == ["hall"]
    panel = frame["panels"][0]
    assert panel["unit"] == "Pa" and panel["grid"] == (5, 4, 3) and panel["values"].shape == (60,)
    assert np.array_equal(panel["values"], hall.sample(extent["min"], extent["max"], extent["samples"]))


def _py_heat_at(cells, void, counts, dx, p):
    """solid.rs:2045-2104 restated line by line in Python, for the oracle's sampler to be checked."""
    nx, ny, nz = counts
    q = [p[a] / dx - 0.5 for a in range(3)]
    if any(math.isnan(v) for v in q):
        return math.nan

    def axis(v, n):
        last = max(n - 1, 0)
        if v <= 0.0:
            return 0, 0.0
        if v >= last:
            return last, 0.0
        i = math.floor(v)
        return int(i), v - i

    (i, fx), (j, fy), (k, fz) = axis(q[0], nx), axis(q[1], ny), axis(q[2], nz)

    def nearest(v, n):  # f64::round: half away from zero
        r = math.floor(abs(v) + 0.5) * (1 if v >= 0 else -1)
        return min(int(max(r, 0.0)), max(n - 1, 0))

    if void[nearest(q[0], nx) + nx * (nearest(q[1], ny) + ny * nearest(q[2], nz))]:
        return math.nan
    i1, j1, k1 = min(i + 1, nx - 1), min(j + 1, ny - 1), min(k + 1, nz - 1)
    s = w_sum = 0.0
    for a, wa in ((i, 1.0 - fx), (i1, fx)):
        for b, wb in ((j, 1.0 - fy), (j1, fy)):
            for c, wc in ((k, 1.0 - fz), (k1, fz)):
                w = wa * wb * wc
                at = a + nx * (b + ny * c)
                if w > 0.0 and not void[at]:
                    s += w * cells[at]
                    w_sum += w
    return s / w_sum if w_sum > 0.0 else math.nan


def test_oracle_heat_sampler_against_a_python_restatement():
    counts, dx = (7, 6, 5), 1e-3
    void = np.zeros(int(np.prod(counts)), dtype=np.uint8)
    void[np.random.default_rng(9).random(void.size) < 0.2] = 1
    o, cells = heat_oracle(counts, dx, void=void)
    rng = np.random.default_rng(11)
    for _ in range(60):
        p = rng.uniform(-1e-3, 8e-3, 3)
        got = o.sample(p, p, (1, 1, 1))[0]
        want = _py_heat_at(cells, void, counts, dx, p)
        assert (math.isnan(got) and math.isnan(want)) or got == want, (p, got, want)


def test_oracle_hall_sampler_against_a_python_restatement():
    h = oracle.Hall(0.01, 0.008, 0.006, 7, 343.0, 1.2)
    nx, ny, nz = h.nodes
    dx = 0.01 / (nx - 1)
    pr = np.random.default_rng(4).uniform(-1.0, 1.0, nx * ny * nz)
    h.release(pr)

    def clamp(v, n):
        if math.isnan(v) or v <= 0.0:
            return 0, 0.0
        if v >= n - 1:
            return n - 1, 0.0
        i = math.floor(v)
        return int(i), v - i

    def lerp(a, b, t):
        return a * (1.0 - t) + b * t

    rng = np.random.default_rng(12)
    for _ in range(60):
        p = rng.uniform(-2e-3, 0.012, 3)
        (i, fx), (j, fy), (k, fz) = clamp(p[0] / dx, nx), clamp(p[1] / dx, ny), clamp(p[2] / dx, nz)
        i1, j1, k1 = min(i + 1, nx - 1), min(j + 1, ny - 1), min(k + 1, nz - 1)
        g = lambda a, b, c: pr[a + nx * (b + ny * c)]  # noqa: E731
        z0 = lerp(lerp(g(i, j, k), g(i1, j, k), fx), lerp(g(i, j1, k), g(i1, j1, k), fx), fy)
        z1 = lerp(lerp(g(i, j, k1), g(i1, j, k1), fx), lerp(g(i, j1, k1), g(i1, j1, k1), fx), fy)
        assert h.sample(p, p, (1, 1, 1))[0] == lerp(z0, z1, fz)


def room_oracle(seed=6):
    r = oracle.Room(0.011, 0.007, 12)
    pr = np.random.default_rng(seed).uniform(-1.0, 1.0, r.n)
    r.release(pr)
    return r, pr


def test_room_samples_on_nodes_are_the_pressures_and_ignore_depth():
    """room.rs:587-601: a sample on a node is that node's pressure, halfway between two nodes the mean
    of the two; z is not read; each NaN coordinate is clamped to node 0 along its own axis."""
    r, pr = room_oracle()
    nx, ny = r.cells
    dx = r.dx
    got = r.sample((0.0, 0.0, 0.3), ((nx - 1) * dx, (ny - 1) * dx, 0.3), (nx, ny, 1))
    assert np.allclose(got, pr, rtol=0, atol=1e-14)  # lo + (hi − lo)·f lands on a node to its rounding
    g = pr.reshape(ny, nx)
    assert r.sample((dx * 2, dx * 3, -5.0), (dx * 2, dx * 3, -5.0), (1, 1, 1))[0] == g[3, 2]
    mid = r.sample((1.5 * dx, 0.0, 0.0), (1.5 * dx, 0.0, 0.0), (1, 1, 1))[0]
    assert mid == pytest.approx(0.5 * (g[0, 1] + g[0, 2]), rel=1e-14)
    nan_x = r.sample((math.nan, 4 * dx, 0.0), (math.nan, 4 * dx, 0.0), (1, 1, 1))[0]
    assert nan_x == g[4, 0]
    # beyond the walls: the corner nodes, clamped rather than extrapolated
    out = r.sample((-1.0, -1.0, 0.0), (1.0, 1.0, 0.0), (2, 2, 1))
    assert out[0] == g[0, 0] and out[-1] == g[-1, -1]


def bar_oracle(cells=9, seed=7):
    b = oracle.Bar(cells, 1e-3, 1e-4, 2700.0, 167.0, 896.0, 300.0)
    t = 300.0 + 30.0 * np.random.default_rng(seed).random(b.n)
    b.cells = t
    return b, t


def test_bar_samples_on_centres_and_beyond_the_ends():
    """lib.rs:736-751: cell centres at (i + ½)·dx read the cells, between two centres the blend,
    beyond either end centre and at a NaN x the end cell; y and z are not read."""
    b, t = bar_oracle()
    n = b.n
    got = b.sample((0.5e-3, 7.0, -3.0), ((n - 0.5) * 1e-3, 7.0, -3.0), (n, 1, 1))
    assert np.allclose(got, t, rtol=1e-15, atol=0)
    assert b.sample((0.0, 0, 0), (0.0, 0, 0), (1, 1, 1))[0] == t[0]
    assert b.sample((1.0, 0, 0), (1.0, 0, 0), (1, 1, 1))[0] == t[-1]
    assert b.sample((math.nan, 0, 0), (math.nan, 0, 0), (1, 1, 1))[0] == t[0]
    mid = b.sample((2.0e-3, 0, 0), (2.0e-3, 0, 0), (1, 1, 1))[0]
    assert mid == pytest.approx(0.5 * (t[1] + t[2]), rel=1e-15)


def test_oracle_room_and_bar_samplers_against_a_python_restatement():
    r, pr = room_oracle(8)
    nx, ny = r.cells
    dx = r.dx

    def clamp(v, n):  # room.rs:739-749
        if math.isnan(v) or v <= 0.0:
            return 0, 0.0
        if v >= n - 1:
            return n - 1, 0.0
        i = math.floor(v)
        return int(i), v - i

    rng = np.random.default_rng(13)
    for _ in range(60):
        p = rng.uniform(-2e-3, 0.013, 3)
        if rng.random() < 0.1:
            p[rng.integers(0, 2)] = math.nan
        (i, fx), (j, fy) = clamp(p[0] / dx, nx), clamp(p[1] / dx, ny)
        i1, j1 = min(i + 1, nx - 1), min(j + 1, ny - 1)
        bottom = pr[j * nx + i] * (1.0 - fx) + pr[j * nx + i1] * fx
        top = pr[j1 * nx + i] * (1.0 - fx) + pr[j1 * nx + i1] * fx
        assert r.sample(p, p, (1, 1, 1))[0] == bottom * (1.0 - fy) + top * fy

    b, t = bar_oracle(11, 9)
    last = b.n - 1
    for _ in range(60):
        x = rng.uniform(-2e-3, 0.013)
        u = x / 1e-3 - 0.5
        if u <= 0.0:
            want = t[0]
        elif u >= last:
            want = t[last]
        else:
            i = math.floor(u)
            f = u - i
            want = t[int(i)] * (1.0 - f) + t[int(i) + 1] * f
        assert b.sample((x, 0, 0), (x, 0, 0), (1, 1, 1))[0] == want


NAN_EXTENT = ((math.nan, 1e-3, 0.0), (math.nan, 5e-3, 1e-3), (1, 4, 2))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_room_device_samples_match_the_oracle(precision):
    """After 25 steps of a released (1, 1) mode (white noise would trip the startup check,
    room.rs:460-475). The f64 form is stepped beside the oracle; the FP32 form's own pressures are
    handed to the oracle, so both forms' samples are bit for bit."""
    from pantometry_b200.domains import Room

    o = oracle.Room(0.011, 0.007, 12)
    g = Room(0.011, 0.007, 12, precision=precision)
    pr = o.mode_profile(1, 1, 1.0)
    o.release(pr)
    g.release(pr)
    dt = 0.9 * o.max_stable_dt()
    assert g.step(dt, 25) is None
    if precision == "f64":
        assert o.step(dt, 25) is None
    else:
        o.release(g.fields()["p"])
    for lo, hi, cnt in EXTENTS + [NAN_EXTENT]:
        want, got = o.sample(lo, hi, cnt), g.sample(lo, hi, cnt)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_bar_device_samples_match_the_oracle(precision):
    from pantometry_b200.domains import Bar

    sub = (2700.0, 167.0, 896.0)
    o = oracle.Bar(40, 1e-3, 1e-4, *sub, 300.0)
    g = Bar(40, 1e-3, 1e-4, *sub, 300.0, precision=precision)
    t = 300.0 + 30.0 * np.random.default_rng(7).random(40)
    o.cells = t
    g.cells = t
    dt = 0.9 * o.max_stable_dt()
    assert g.step(dt, 25) is None
    if precision == "f64":
        assert o.step(dt, 25) is None
    else:
        o.cells = g.cells  # kelvin as the FP32 form reads it: T_ref + deviation
    for lo, hi, cnt in EXTENTS + [NAN_EXTENT, ((0.5e-3, 0, 0), (39.5e-3, 0, 0), (40, 1, 1))]:
        want, got = o.sample(lo, hi, cnt), g.sample(lo, hi, cnt)
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


@pytest.mark.gpu
def test_capture_labels_every_field_kind():
    """Each field kind is drawn with the unit its ScalarField::unit gives (solid.rs, lib.rs:732-734,
    hall.rs:586-588, room.rs:583-585, cavity.rs)."""
    from pantometry_b200 import scenes
    from pantometry_b200.domains import Bar, Cavity, Hall, Room, Solid3D

    doms = {"block": Solid3D((4, 4, 4), 1e-3, 1000.0, 100.0, 1000.0, 300.0),
            "bar": Bar(8, 1e-3, 1e-4, 2700.0, 167.0, 896.0, 310.0),
            "hall": Hall(0.01, 0.008, 0.006, 6, 343.0, 1.2),
            "room": Room(0.011, 0.007, 12),
            "cavity": Cavity((4, 4, 4), 1e-3)}
    extent = {"min": (0.0, 0.0, 0.0), "max": (0.004, 0.003, 0.002), "samples": (3, 2, 2)}
    frame = scenes.capture(doms, {k: {"extent": extent} for k in doms})
    units = {p["name"]: p["unit"] for p in frame["panels"]}
    assert units == {"block": "K", "bar": "K", "hall": "Pa", "room": "Pa", "cavity": "V/m"}
    for p in frame["panels"]:
        want = doms[p["name"]].sample(extent["min"], extent["max"], extent["samples"])
        assert np.array_equal(p["values"], want)


# nothing_is_not_a_temperature.rs: Substance::copper (substance.rs:462-471), 10 mm cells at 20 °C
COPPER = dict(density=8.96e3, conductivity=401.0, specific_heat=385.0, emissivity=0.04)
C20, C300 = 20.0 + 273.15, 300.0 + 273.15


def copper_block(counts, make=None, precision="f64"):
    s = COPPER
    if make is None:
        return oracle.Heat(counts, 10e-3, s["density"], s["conductivity"], s["specific_heat"], C20,
                           emissivity=s["emissivity"])
    return make(counts, 10e-3, s["density"], s["conductivity"], s["specific_heat"], C20,
                emissivity=s["emissivity"], precision=precision)


def gapped_bar(make=None, precision="f64"):
    """nothing_is_not_a_temperature.rs:20-32: four cells along x, the first at 300 °C, the middle two
    emptied."""
    b = copper_block((4, 1, 1), make, precision)
    b.cells = np.array([C300, C20, C20, C20])
    b.empty(np.array([0, 1, 1, 0], dtype=np.uint8))
    return b


def at_mm(block, mm):
    p = (mm * 1e-3, 5e-3, 5e-3)
    return block.sample(p, p, (1, 1, 1))[0]


def check_void_readings(block, tol):
    # nothing_is_not_a_temperature.rs:34-60: exact on the metal, no value in the gap
    assert abs(at_mm(block, 5.0) - C300) < tol
    assert abs(at_mm(block, 35.0) - C20) < tol
    for mm in (15.0, 20.0, 25.0):
        assert math.isnan(at_mm(block, mm)), mm
    # :62-83: a sample straddling the boundary belongs to the cell it is in
    assert math.isfinite(at_mm(block, 9.0))
    assert math.isnan(at_mm(block, 11.0))
    face = at_mm(block, 10.0)
    assert math.isnan(face) or abs(face - C300) < tol


def check_unmasked_block_interpolates(block, tol):
    """nothing_is_not_a_temperature.rs:85-125: a 2×2×2 block with nothing masked is plain trilinear."""
    cell = lambda i, j, k: 100.0 * (i + 2 * j + 4 * k) + 273.15  # noqa: E731
    block.cells = np.array([cell(i, j, k) for k in range(2) for j in range(2) for i in range(2)])
    fx, fy, fz = 0.3, 0.6, 0.8
    mm = lambda f: (5.0 + 10.0 * f) * 1e-3  # noqa: E731
    p = (mm(fx), mm(fy), mm(fz))
    got = block.sample(p, p, (1, 1, 1))[0]
    lerp = lambda lo, hi, t: lo * (1.0 - t) + hi * t  # noqa: E731
    z0 = lerp(lerp(cell(0, 0, 0), cell(1, 0, 0), fx), lerp(cell(0, 1, 0), cell(1, 1, 0), fx), fy)
    z1 = lerp(lerp(cell(0, 0, 1), cell(1, 0, 1), fx), lerp(cell(0, 1, 1), cell(1, 1, 1), fx), fy)
    assert abs(got - lerp(z0, z1, fz)) < tol


def test_oracle_void_readings_restate_the_reference():
    check_void_readings(gapped_bar(), 1e-12)
    check_unmasked_block_interpolates(copper_block((2, 2, 2)), 1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_void_readings_restate_the_reference(precision):
    from pantometry_b200.domains import Solid3D

    tol = 1e-12 if precision == "f64" else 1e-4  # FP32: kelvin from f32 deviations
    check_void_readings(gapped_bar(Solid3D, precision), tol)
    check_unmasked_block_interpolates(copper_block((2, 2, 2), Solid3D, precision), max(tol, 1e-9))
