"""Seeded synthetic inputs for the benchmark configurations.

Every random draw uses the reference's own generator, `Rng::for_index(seed, index)`
(crates/pantometry-core/src/rng.rs:36-100: SplitMix64's finaliser to seed, xorshift64* to draw,
`unit() = (x >> 11) / 2^53`), restated here over numpy uint64 arrays so that millions of
independent per-cell streams are drawn at once. Fields are generated once in f64 on the host;
the f32 forms receive the same bytes rounded on the device.

Configurations (sizes, media and sources as the benchmark names them):
  heat_block      64³ conduction block, Dirichlet 300 K faces, Gaussian hot spot, 1000 steps
  acoustic_hall   256³ acoustic hall, ±1e-3 Pa noise, 2 kHz Ricker point source, 5000 steps
  yee_cavity      384³ vacuum Yee cavity, PEC walls, Gaussian-modulated dipole current
  heat_ensemble   512 uneven heat grids, 16..128 cells per axis
"""
from __future__ import annotations

import math
import os

import numpy as np

SEED = 0x70616E746F  # "panto"

_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xBF58476D1CE4E5B9)
_M3 = np.uint64(0x94D049BB133111EB)
_XS = np.uint64(0x2545F4914F6CDD1D)


def _mix64(z):
    with np.errstate(over="ignore"):
        z = z + _M1
        z = (z ^ (z >> np.uint64(30))) * _M2
        z = (z ^ (z >> np.uint64(27))) * _M3
        return z ^ (z >> np.uint64(31))


class Streams:
    """Independent `Rng::for_index(seed, i)` streams for a vector of indices, drawn in lockstep."""

    def __init__(self, seed, index):
        idx = np.asarray(index, dtype=np.uint64)
        s = _mix64(np.uint64(seed) ^ _mix64(idx))
        self.state = np.where(s == 0, _M1, s)  # Rng::new replaces a zero seed

    def next_u64(self):
        with np.errstate(over="ignore"):
            x = self.state
            x = x ^ (x >> np.uint64(12))
            x = x ^ (x << np.uint64(25))
            x = x ^ (x >> np.uint64(27))
            self.state = x
            return x * _XS

    def unit(self):
        return (self.next_u64() >> np.uint64(11)).astype(np.float64) / float(1 << 53)

    def range(self, lo, hi):
        return lo + (hi - lo) * self.unit()


def uniform_noise(seed, count, lo, hi, out=None, chunk=1 << 22):
    """`Rng::for_index(seed, i).range(lo, hi)` for i in 0..count, drawn in chunks so that a
    10⁹-node field needs no more host memory than its own array (`out`, if given, e.g. pinned)."""
    from concurrent.futures import ThreadPoolExecutor

    out = np.empty(count, dtype=np.float64) if out is None else out

    def fill(a):
        b = min(count, a + chunk)
        out[a:b] = Streams(seed, np.arange(a, b, dtype=np.uint64)).range(lo, hi)

    if count <= chunk:
        fill(0)
        return out
    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as pool:  # numpy drops the GIL
        list(pool.map(fill, range(0, count, chunk)))
    return out


# ------------------------------------------------------------------------------------------
# heat_block: 64³, α = 1e-4 m²/s, dx = 1 mm, dt = 0.9 × limit, Dirichlet 300 K via h = ∞ films
# ------------------------------------------------------------------------------------------
HEAT_SUBSTANCE = dict(density=1000.0, conductivity=100.0, specific_heat=1000.0, emissivity=0.0)


def hot_spot(counts, centre, amplitude=50.0, sigma=8.0, base=300.0):
    nx, ny, nz = counts
    i = np.arange(nx) + 0.5 - centre[0]
    j = np.arange(ny) + 0.5 - centre[1]
    k = np.arange(nz) + 0.5 - centre[2]
    r2 = k[:, None, None] ** 2 + j[None, :, None] ** 2 + i[None, None, :] ** 2
    return (base + amplitude * np.exp(-r2 / (2.0 * sigma * sigma))).reshape(-1)


def heat_block(n=64, seed=SEED, steps=1000):
    jitter = np.array([Streams(seed, [a]).range(-4.0, 4.0)[0] for a in range(3)])
    centre = n / 2 + jitter
    dx = 1e-3
    return {
        "counts": (n, n, n),
        "dx": dx,
        "initial": 300.0,
        "substance": dict(HEAT_SUBSTANCE),
        "films": [(f, 300.0, math.inf, (n * dx) * (n * dx)) for f in range(6)],
        "cells": hot_spot((n, n, n), centre),
        "steps": steps,
        "dt_fraction": 0.9,
    }


def build_heat(cfg, precision="f64", device=0):
    from .domains import Solid3D

    s = cfg["substance"]
    b = Solid3D(cfg["counts"], cfg["dx"], s["density"], s["conductivity"], s["specific_heat"], cfg["initial"],
                emissivity=s["emissivity"], precision=precision, device=device)
    for f, amb, h, area in cfg["films"]:
        b.losing_from(f, amb, h, area)
    b.cells = cfg["cells"]
    return b


# ------------------------------------------------------------------------------------------
# acoustic_hall: 256³ nodes of air, CFL 0.5, ±1e-3 Pa noise, 1 Pa 2 kHz Ricker at the centre
# ------------------------------------------------------------------------------------------
def ricker(t, f):
    a = (math.pi * f * (t - 1.2 / f)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def acoustic_hall(n=256, seed=SEED, steps=5000, dx=5e-3, speed=343.0, density=1.2, source=True):
    width = (n - 1) * dx
    nodes = n * n * n
    p = uniform_noise(seed, nodes, -1e-3, 1e-3)
    dx_eff = max(width / (n - 1), np.finfo(np.float64).tiny)  # Hall::new (hall.rs:109)
    dt = 0.5 * dx_eff / (speed * math.sqrt(3.0))
    c = n // 2
    cfg = {
        "size": (width, width, width),
        "across": n,
        "speed": speed,
        "density": density,
        "pressure": p,
        "dt": dt,
        "steps": steps,
    }
    if source:
        t = (np.arange(steps, dtype=np.float64) + 1.0) * dt
        cfg["source_node"] = c + n * (c + n * c)
        cfg["wave"] = ricker(t, 2000.0)
    return cfg


def build_hall(cfg, precision="f64", device=0):
    from .domains import Hall

    w, h, d = cfg["size"]
    hall = Hall(w, h, d, cfg["across"], cfg["speed"], cfg["density"], precision=precision, device=device)
    hall.release(cfg["pressure"])
    if "wave" in cfg:
        hall.set_source(cfg["source_node"], cfg["wave"])
    return hall


# ------------------------------------------------------------------------------------------
# yee_cavity: 384³ vacuum cells, PEC walls, Courant 0.99/√3, soft z-current at the centre edge
# ------------------------------------------------------------------------------------------
C0 = 1.0 / math.sqrt(8.8541878128e-12 * 1.25663706212e-6)


def yee_cavity(n=384, steps=10000, dx=1e-3, amplitude=1.0):
    limit = 0.5773502691896258 * dx / C0
    dt = 0.99 * limit
    f0 = C0 / (20.0 * dx)
    tau = 1.0 / (math.pi * 0.5 * f0)
    t0 = 4.0 * tau
    t = (np.arange(steps, dtype=np.float64) + 0.5) * dt
    current = amplitude / (dx * dx) * np.exp(-(((t - t0) / tau) ** 2)) * np.sin(2.0 * math.pi * f0 * t)
    c = n // 2
    edge = c + (n + 1) * (c + (n + 1) * c)  # iez(c, c, c), cavity.rs:1052-1055
    return {"counts": (n, n, n), "dx": dx, "dt": dt, "steps": steps, "edge": edge, "current": current}


def build_cavity(cfg, precision="f64", device=0):
    from .domains import Cavity

    cav = Cavity(cfg["counts"], cfg["dx"], precision=precision, device=device)
    if "current" in cfg:
        cav.set_source(cfg["edge"], cfg["current"])
    return cav


# ------------------------------------------------------------------------------------------
# config 5: a 1024³ hall in a medium of 32³-node blocks (c uniform in [300, 1500] m/s per block)
# and 64 Yee cavities of 128³ cells with dielectric inclusions (ε_r uniform in [1, 4] in 10% of
# cells)
# ------------------------------------------------------------------------------------------
def hetero_hall(n=1024, block=32, seed=SEED, steps=2000, dx=5e-3, density=1.2, lo=300.0, hi=1500.0):
    cfg = acoustic_hall(n, seed=seed, steps=steps, dx=dx, density=density, source=True)
    nb = -(-n // block)
    speeds = Streams(seed ^ 0x5EED, np.arange(nb ** 3, dtype=np.uint64)).range(lo, hi)
    cfg["block"] = block
    cfg["speeds"] = speeds
    cfg["speed"] = float(speeds.max())  # the descriptor's speed: the limit follows the fastest block
    cfg["dt"] = 0.5 * dx / (cfg["speed"] * math.sqrt(3.0))  # CFL 0.5 of the fastest block
    return cfg


def build_hetero_hall(cfg, precision="f32", device=0):
    hall = build_hall(cfg, precision=precision, device=device)
    hall.set_speed_blocks(cfg["block"], cfg["speeds"])
    return hall


def dielectric_cavities(count=64, n=128, seed=SEED, steps=2000, dx=1e-3, fraction=0.1, lo=1.0, hi=4.0):
    """Per cavity g: a Bernoulli(fraction) draw per cell from Rng::for_index(seed + g, cell) picks the
    inclusions, a second draw their ε_r; the dipole current of yee_cavity at the centre edge."""
    base = yee_cavity(n, steps=steps, dx=dx)
    cavities = []
    for g in range(count):
        r = Streams(seed + 1 + g, np.arange(n ** 3, dtype=np.uint64))
        pick = r.unit() < fraction
        eps = np.where(pick, r.range(lo, hi), 1.0)
        cavities.append({"eps": eps})
    return {"counts": (n, n, n), "dx": dx, "dt": base["dt"], "edge": base["edge"], "current": base["current"],
            "cavities": cavities, "steps": steps}


def build_dielectric_cavity(cfg, g, precision="f32", device=0):
    from .domains import Cavity

    cav = Cavity(cfg["counts"], cfg["dx"], precision=precision, device=device)
    cav.fill_cells(eps_r=cfg["cavities"][g]["eps"])
    cav.set_source(cfg["edge"], cfg["current"])
    return cav


# ------------------------------------------------------------------------------------------
# heat_ensemble: 512 grids, sizes U{16..128} per axis, α log-uniform in [1e-6, 1e-3]
# ------------------------------------------------------------------------------------------
def heat_ensemble(count=512, seed=SEED, lo=16, hi=128, steps=2000):
    grids = []
    for g in range(count):
        r = Streams(seed, [g])
        nx, ny, nz = (lo + int(r.unit()[0] * (hi - lo + 1)) for _ in range(3))
        alpha = 10.0 ** r.range(-6.0, -3.0)[0]
        centre = (r.range(0.0, nx)[0], r.range(0.0, ny)[0], r.range(0.0, nz)[0])
        sigma = min(8.0, min(nx, ny, nz) / 8.0)
        grids.append({
            "counts": (nx, ny, nz),
            "dx": 1e-3,
            "substance": dict(density=1000.0, conductivity=alpha * 1e6, specific_heat=1000.0, emissivity=0.0),
            "initial": 300.0,
            "centre": centre,
            "sigma": sigma,
        })
    return {"grids": grids, "steps": steps}


def ensemble_cells(grid):
    return hot_spot(grid["counts"], grid["centre"], sigma=grid["sigma"])


def ensemble_grids(cfg, dt_fraction=0.9):
    """The ensemble's block descriptors: Dirichlet (h = +inf) films at 300 K on every face and
    each block's dt at `dt_fraction` of its own stability limit."""
    from .domains import Ensemble

    grids = [{"counts": g["counts"], "dx": g["dx"], "substance": g["substance"], "initial": g["initial"],
              "convection": math.inf} for g in cfg["grids"]]
    for g, limit in zip(grids, Ensemble.max_stable_dt(grids)):
        g["dt"] = dt_fraction * limit
    return grids


def build_ensemble(cfg, precision="f32", device=0, cells=None):
    from .domains import Ensemble

    e = Ensemble(ensemble_grids(cfg), precision=precision, device=device)
    e.upload(np.concatenate([ensemble_cells(g) for g in cfg["grids"]]) if cells is None else cells)
    return e
