"""FP32 form of a filled (multi-material) `Solid3D`.

`Solid3D::fill` gives each face the harmonic mean of its two cells' conductivities and each cell
its own capacity and mobility (crates/pantometry-thermal/src/solid.rs:588-784); the step is
`cells[c] += dt·mobility·(Σ k_f·(T_nb − T) − shed)` (solid.rs:1773-1826). The FP32 form keeps the
deviation T − T0 in f32 and reads the face conductivities, dt·mobility and each boundary cell's
film conductance in f32; stored and shed heat are FP64 with per-cell capacities. Checked against the
f64 oracle with the bounds of the uniform FP32 tests: within 1e-4 K of the oracle on a 30 K spread
and the books within 1e-6 of the ledger's scale, audited every step.
"""
import numpy as np
import pytest

from helpers import dirichlet_films, heat_pair

pytestmark = pytest.mark.gpu

COPPER = dict(density=8960.0, conductivity=401.0, specific_heat=385.0, emissivity=0.0)
STEEL = dict(density=7850.0, conductivity=45.0, specific_heat=490.0, emissivity=0.0)
GLASS = dict(density=2500.0, conductivity=1.0, specific_heat=840.0, emissivity=0.0)


def layered(counts, seed=1):
    """Steel with a copper layer in the upper half of x and a glass slab in the middle of z."""
    nx, ny, nz = counts
    cu = np.zeros(counts[::-1], dtype=np.uint8)
    cu[:, :, nx // 2:] = 1
    gl = np.zeros(counts[::-1], dtype=np.uint8)
    gl[nz // 3: 2 * nz // 3, :, :] = 1
    cells = 300.0 + 30.0 * np.random.default_rng(seed).random(np.prod(counts))
    return cu.reshape(-1), gl.reshape(-1), cells


def pair(counts, dx, films):
    cu, gl, cells = layered(counts)
    o, g = heat_pair(counts, dx, STEEL, 300.0, films, None, precision="f32", fill=(cu, COPPER))
    for d in (o, g):
        d.fill(gl, GLASS["density"], GLASS["conductivity"], GLASS["specific_heat"], 0.0)
        d.cells = cells
    return o, g


def finite_films(counts, dx):
    """Convective films of finite h at two ambients on four faces (two faces insulated)."""
    nx, ny, nz = counts
    areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
    return [(0, 280.0, 50.0, areas[0]), (1, 320.0, 2000.0, areas[1]), (2, 290.0, 10.0, areas[2]),
            (5, 310.0, 500.0, areas[5])]


@pytest.mark.parametrize("films", ["dirichlet", "finite"])
@pytest.mark.parametrize("counts", [(12, 7, 5), (40, 24, 18)])
def test_heat_filled_f32_tracks_the_oracle(films, counts):
    dx = 1e-3
    fl = dirichlet_films(counts, dx) if films == "dirichlet" else finite_films(counts, dx)
    o, g = pair(counts, dx, fl)
    assert g.max_stable_dt() == o.max_stable_dt()
    dt = 0.7 * o.max_stable_dt()
    l0o, l0g = o.ledger(), g.ledger()
    assert abs(l0g["total"] - l0o["total"]) < 1e-6 * l0o["scale"]
    g.set_tolerance(1e-6)
    assert o.step(dt, 120) is None
    assert g.step(dt, 120) is None  # audited every step in FP64
    assert np.abs(g.cells - o.cells).max() < 1e-4
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-6 * lo["scale"]
    assert abs(lg["parts"][1] - lo["lost"]) < 1e-6 * lo["scale"]
    # a new step size: dt·mobility is formed again (and a graph run of 70 steps uses it)
    assert o.step(0.5 * dt, 70) is None
    assert g.step(0.5 * dt, 70) is None
    assert np.abs(g.cells - o.cells).max() < 1e-4
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-6 * lo["scale"]


def test_heat_filled_f32_films_set_after_the_fill():
    """Films added after the fill: each boundary cell's film conductance follows its material."""
    counts, dx = (16, 9, 7), 1e-3
    cu, gl, cells = layered(counts)
    o, g = heat_pair(counts, dx, STEEL, 300.0, (), None, precision="f32", fill=(cu, COPPER))
    for d in (o, g):
        d.cells = cells
        for f, amb, h, area in finite_films(counts, dx):
            d.losing_from(f, amb, h, area)
    dt = 0.7 * o.max_stable_dt()
    assert o.step(dt, 100) is None
    assert g.step(dt, 100) is None
    assert np.abs(g.cells - o.cells).max() < 1e-4
    lo, lg = o.ledger(), g.ledger()
    assert abs(lg["total"] - lo["total"]) < 1e-6 * lo["scale"]
