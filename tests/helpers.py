"""Shared builders for the parity tests: the same inputs for the oracle and the GPU path."""
import math

import numpy as np

import oracle

AL = dict(density=2.70 * 1e3, conductivity=167.0, specific_heat=896.0, emissivity=0.09)
T20 = 20.0 + 273.15


def heat_pair(counts, dx, substance, initial, films=(), cells=None, precision="f64", fill=None):
    """An oracle `Solid3D` and a GPU one with identical construction and state."""
    from pantometry_b200.domains import Solid3D

    s = substance
    o = oracle.Heat(counts, dx, s["density"], s["conductivity"], s["specific_heat"], initial,
                    emissivity=s.get("emissivity", 0.0))
    g = Solid3D(counts, dx, s["density"], s["conductivity"], s["specific_heat"], initial,
                emissivity=s.get("emissivity", 0.0), precision=precision)
    if fill is not None:
        mask, sub = fill
        o.fill(mask, sub["density"], sub["conductivity"], sub["specific_heat"], sub.get("emissivity", 0.0))
        g.fill(mask, sub["density"], sub["conductivity"], sub["specific_heat"], sub.get("emissivity", 0.0))
    for f, amb, h, area in films:
        o.losing_from(f, amb, h, area)
        g.losing_from(f, amb, h, area)
    if cells is not None:
        o.cells = cells
        g.cells = cells
    return o, g


def dirichlet_films(counts, dx, ambient=300.0):
    nx, ny, nz = counts
    areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
    return [(f, ambient, math.inf, areas[f]) for f in range(6)]


def hall_pair(width, height, depth, across, speed=343.0, density=1.204, pressure=None, mode=None, amplitude=2.0,
              precision="f64", source=None):
    from pantometry_b200.domains import Hall

    o = oracle.Hall(width, height, depth, across, speed, density)
    g = Hall(width, height, depth, across, speed, density, precision=precision)
    if mode is not None:
        o.release_mode(mode, amplitude)
        pressure = o.fields()["p"]
        g.release(pressure)
    elif pressure is not None:
        o.release(pressure)
        g.release(pressure)
    if source is not None:
        node, wave = source
        o.set_source(node, wave)
        g.set_source(node, wave)
    return o, g


def cavity_pair(counts, dx, precision="f64", mode=None, dt=None, eps_cells=None, solid=None, source=None):
    from pantometry_b200.domains import Cavity

    o = oracle.Yee(counts, dx)
    g = Cavity(counts, dx, precision=precision)
    if eps_cells is not None:
        o.set_cells(eps_r=eps_cells)
        g.fill_cells(eps_r=eps_cells)
    if mode is not None:
        o.release_mode(mode, 1.0, dt)
        g.release_mode(mode, 1.0, dt)
    if solid is not None:
        o.obstruct(solid)
        g.obstruct(solid)
    if source is not None:
        edge, cur = source
        o.set_source(edge, cur)
        g.set_source(edge, cur)
    return o, g


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def assert_bitexact(name, got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    bad = np.flatnonzero(got.view(np.uint64) != want.view(np.uint64))
    assert bad.size == 0, (
        f"{name}: {bad.size} of {got.size} values differ; first at {bad[0]}: "
        f"{got[bad[0]]!r} vs {want[bad[0]]!r} (max abs diff {np.abs(got - want).max():.3e})"
    )
