"""Single-domain scenes, run the way `World::run` runs them (crates/pantometry-world/src/lib.rs:3204-3215).

The clock advances `duration_s / frames` per frame, and every window is one `Simulation::advance`
under the multirate schedule (crates/pantometry-core/src/sim.rs:947-1111): the window split into
ceil(window / limit) equal substeps of the domain (`substeps_for`,
crates/pantometry-core/src/integrator.rs:186-199), with the ledger before and after the window
audited at the scene's conservation tolerance (`audit_with`,
crates/pantometry-core/src/conserved.rs:323-363).

A scene is a dict with the keys of the reference's scene files (`schedule`, `duration_s`, `frames`,
`conservation_tolerance`, `domains`) holding one domain of kind "block" (of the catalogue's
aluminium and borosilicate, with regions and a hot spot), "hall", "room" (released in a mode or
from a pulse) or "cavity", with the keys the world reads for it (lib.rs:1405-1433, 1786-1812,
1876-1960, 2192-2350). `build` makes the GPU domain, with the initial fields generated here on the host;
`run` runs any domain object with `step`, `ledger` and `max_stable_dt` (or `courant_limit`).
"""
from __future__ import annotations

import math

import numpy as np

from .domains import Bar, Cavity, Hall, Room, Solid3D

# substance.rs:362-373 (`Substance::aluminium_6061`; g/cm³ × 1e3, units lib.rs:751-753) and
# substance.rs:336-347 (`Substance::borosilicate_crown`), the catalogue names a scene gives them
# (substance.rs:318-319)
ALUMINIUM_6061 = dict(density=2.70 * 1e3, conductivity=167.0, specific_heat=896.0, emissivity=0.09)
BOROSILICATE_CROWN = dict(density=2.51 * 1e3, conductivity=1.114, specific_heat=858.0, emissivity=0.90)
MATERIALS = {"aluminium": ALUMINIUM_6061, "borosilicate": BOROSILICATE_CROWN}
AIR = dict(speed=343.0, density=1.204)  # hall.rs:139-152, room.rs:122-138


def celsius(c):
    return c + 273.15  # units lib.rs:729-731


def substeps_for(dt, limit):
    """integrator.rs:186-199: how many equal substeps a window needs under a domain's limit."""
    if not math.isfinite(limit) or limit <= 0.0 or dt <= 0.0:
        return 1
    n = math.ceil(dt / limit)
    return 1 if n < 1 else min(n, 2**32 - 1)


def limit_of(domain):
    return domain.max_stable_dt() if hasattr(domain, "max_stable_dt") else domain.courant_limit()


def _phase(n, x, length):
    return np.cos(n * math.pi * x / length) if length > 0.0 else np.ones_like(x)


def hall_mode_profile(nodes, dx, mode, amplitude):
    """`Hall::released_in_mode` (hall.rs:190-210), sampled at the nodes (x fastest)."""
    nx, ny, nz = nodes
    lx, ly, lz = (nx - 1) * dx, (ny - 1) * dx, (nz - 1) * dx
    px = _phase(mode[0], np.arange(nx) * dx, lx)
    py = _phase(mode[1], np.arange(ny) * dx, ly)
    pz = _phase(mode[2], np.arange(nz) * dx, lz)
    return (amplitude * px[None, None, :] * py[None, :, None] * pz[:, None, None]).reshape(-1)


def room_mode_profile(cells, dx, mode, amplitude):
    """`Room::released_in_mode` (room.rs:166-183), sampled at the nodes (x fastest)."""
    nx, ny = cells
    px = _phase(mode[0], np.arange(nx) * dx, (nx - 1) * dx)
    py = _phase(mode[1], np.arange(ny) * dx, (ny - 1) * dx)
    return (amplitude * px[None, :] * py[:, None]).reshape(-1)


def room_pulse_profile(cells, dx, x_m, y_m, radius_m, amplitude):
    """A room released from a Gaussian pulse (lib.rs:1424-1433): a·exp(−|r − c|²/R²) at the nodes
    (`Room::released_from` samples x = i·dx, y = j·dx, room.rs:140-147)."""
    nx, ny = cells
    r = max(radius_m, 1e-9)
    x = np.arange(nx) * dx - x_m
    y = np.arange(ny) * dx - y_m
    d2 = x[None, :] * x[None, :] + y[:, None] * y[:, None]
    return (amplitude * np.exp(-d2 / (r * r))).reshape(-1)


def room_release(cells, dx, rel):
    """The pressure a room is released with: a mode or a pulse (lib.rs:1418-1433)."""
    if rel.get("as") == "mode":
        return room_mode_profile(cells, dx, (rel["nx"], rel["ny"]), rel["amplitude_pa"])
    if rel.get("as") == "pulse":
        return room_pulse_profile(cells, dx, rel["x_m"], rel["y_m"], rel["radius_m"], rel["amplitude_pa"])
    raise ValueError(f"room release {rel.get('as')!r}")


def block_layout(d):
    """A block's bulk material, its regions' fills in order (later wins where they overlap) and its
    initial kelvin per cell (x fastest): the world's block construction (lib.rs:2192-2350) for
    regions of catalogue materials, region temperatures and a hot spot."""
    counts = tuple(d["cells"])
    bulk = MATERIALS[d.get("material", "aluminium")]
    k, j, i = np.indices(counts[::-1]).reshape(3, -1)
    t = np.full(int(np.prod(counts)), celsius(d["initial_c"]))
    fills = []
    for r in d.get("regions", []):
        if r["material"] not in MATERIALS:
            raise ValueError(f"region material {r['material']!r}: the catalogue's aluminium and borosilicate only")
        lo, hi = r["from"], r["to"]
        inside = (i >= lo[0]) & (i < hi[0]) & (j >= lo[1]) & (j < hi[1]) & (k >= lo[2]) & (k < hi[2])
        fills.append((inside.astype(np.uint8), MATERIALS[r["material"]]))
        if r.get("initial_c") is not None:
            t[inside] = celsius(r["initial_c"])
    spot = d.get("hot_spot")
    if spot:
        si, sj, sk = spot["at"]
        t[si + counts[0] * (sj + counts[1] * sk)] = celsius(d["initial_c"] + spot["above_k"])
    return bulk, fills, t


def window(scene):
    return scene["duration_s"] / scene["frames"]


def build(scene, precision="f64", device=0):
    """The scene's one domain on the GPU, released as the world releases it."""
    if scene.get("schedule", "multirate") != "multirate":
        raise ValueError("only the multirate schedule is run here")
    if len(scene["domains"]) != 1:
        raise ValueError("a scene of one domain")
    d = scene["domains"][0]
    kind = d["kind"]
    if kind == "block":  # lib.rs:2192-2350
        if d.get("cooling") or d.get("parts"):
            raise ValueError("blocks without cooling films or voxelised parts only")
        m, fills, t = block_layout(d)
        counts = tuple(d["cells"])
        dom = Solid3D(counts, d["cell_mm"] * 1e-3, m["density"], m["conductivity"], m["specific_heat"],
                      celsius(d["initial_c"]), emissivity=m["emissivity"], precision=precision, name=d["name"],
                      device=device)
        for mask, sub in fills:
            dom.fill(mask, sub["density"], sub["conductivity"], sub["specific_heat"], sub["emissivity"])
        dom.cells = t
        return dom
    if kind == "hall":  # lib.rs:1786-1812
        dom = Hall(d["width_m"], d["height_m"], d["depth_m"], d["nodes_across"], AIR["speed"], AIR["density"],
                   precision=precision, name=d["name"], device=device)
        dom.release(hall_mode_profile(dom.nodes, dom.dx, d["mode"], d["amplitude_pa"]))
        return dom
    if kind == "room":  # lib.rs:1405-1430
        rel = d["release"]
        dom = Room(d["width_m"], d["height_m"], d["cells_across"], 1.0, AIR["density"], AIR["speed"],
                   precision=precision, name=d["name"], device=device)
        dom.release(room_release(dom.cells, dom.dx, rel))
        return dom
    if kind == "cavity":  # lib.rs:1876-1960, 3144-3149
        if d.get("medium", "vacuum") != "vacuum":
            raise ValueError("vacuum cavities only")
        dom = Cavity(tuple(d["cells"]), d["cell_mm"] * 1e-3, precision=precision, name=d["name"], device=device)
        if d.get("mode"):
            steps = max(math.ceil(window(scene) / dom.courant_limit()), 1)
            dom.release_mode(tuple(d["mode"]), d.get("amplitude_v_per_m", 1.0), window(scene) / steps)
        return dom
    raise ValueError(f"{kind!r} is not a domain kind this path steps")


def run(scene, domain):
    """`World::run` over one domain: the frames (time, ledger total and scale, the first frame the
    state as released), the substeps each window took, and the first violation (None if the run
    held). A violation stops the run, as in the reference."""
    h_window = window(scene)
    tol = scene.get("conservation_tolerance", 1e-9)
    frames, substeps = [], []
    led = domain.ledger()
    t = 0.0
    frames.append({"t": t, "total": led["total"], "scale": led["scale"]})
    for _ in range(scene["frames"]):
        n = substeps_for(h_window, limit_of(domain))
        v = domain.step(h_window / n, n)
        if v is not None:
            return {"frames": frames, "substeps": substeps, "violation": v}
        after = domain.ledger()
        # audit_with (conserved.rs:323-363) across the window
        scale = max(abs(led["total"]), abs(after["total"]), led["scale"], after["scale"])
        if scale >= 1e-300 and abs(after["total"] - led["total"]) / scale > tol:
            return {"frames": frames, "substeps": substeps,
                    "violation": {"quantity": "energy", "site": "simulation", "before": led["total"],
                                  "after": after["total"], "scale": scale, "tolerance": tol}}
        t += h_window
        led = after
        substeps.append(n)
        frames.append({"t": t, "total": led["total"], "scale": led["scale"]})
    return {"frames": frames, "substeps": substeps, "violation": None}


# ScalarField::unit of each field domain (solid.rs:2030-2032, hall.rs:586-588, cavity.rs:191-193)
UNITS = {Solid3D: "K", Bar: "K", Hall: "Pa", Room: "Pa", Cavity: "V/m"}


def capture(domains, placed, time_s=0.0):
    """`scene::capture` (crates/pantometry-scene/src/lib.rs:347-372) over domains on the device.

    `domains` maps names to domains; `placed` maps names to placements, each with an optional
    "extent": {"min": (x, y, z), "max": (x, y, z), "samples": (nx, ny, nz)} in metres. Every domain
    that is a field and was placed with an extent becomes a panel: its `ScalarField::at` at each
    point of the extent's sample grid, sampled on the device from the resident state (only the
    samples cross to the host). A field placed with no extent is not drawn (lib.rs:343-345), as
    the reference leaves it. Scalar readings and body sets are outside this path.
    """
    panels = []
    for name, domain in domains.items():
        extent = (placed.get(name) or {}).get("extent")
        unit = next((u for cls, u in UNITS.items() if isinstance(domain, cls)), None)
        if extent is None or unit is None:
            continue
        samples = tuple(int(v) for v in extent["samples"])
        values = domain.sample(extent["min"], extent["max"], samples)
        panels.append({"name": name, "unit": unit, "grid": samples, "values": values})
    return {"time_s": float(time_s), "panels": panels}
