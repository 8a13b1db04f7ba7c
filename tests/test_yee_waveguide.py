"""A rectangular waveguide: a cavity with conducting side walls and Mur (`Open`) ends, restating the
reference's own known answers (crates/pantometry-em/tests/a_waveguide.rs). One launched TE10 pulse,
recorded at a row of stations and transformed there, gives the propagation constant from the phase
slope above cutoff, within 4% of √(k² − k_c²) from 1.4 to 3.1 f_c (:206-257); a driven source
below cutoff gives a field decaying at √(k_c² − k²) within 8% (:259-367); v_p·v_g = c² within 5%
(:369-412); and the cutoff depends on the cross-section alone (:419-455). Below cutoff the oracle
also reproduces the three biases the reference prints for its own run (0.4%, 5.5%, 4.2%), which
pins the oracle's conducting walls, Mur end and soft source to the reference itself; the device
runs the same launched guide bit for bit with the oracle in f64.
"""
import math

import numpy as np
import pytest

import oracle

ACROSS, ALONG = 20, 420  # a_waveguide.rs:39-42
C0 = 299_792_458.0
ZLOW, ZHIGH = 4, 5


def transform(series, frequency, dt):
    """a_waveguide.rs:44-53: (amplitude, phase) of the series at one frequency."""
    phase = -2.0 * math.pi * frequency * np.arange(series.size) * dt
    re = float(np.sum(series * np.cos(phase)))
    im = float(np.sum(series * np.sin(phase)))
    return math.sqrt(re * re + im * im), math.atan2(im, re)


def slope(x, y):
    """a_waveguide.rs:55-62: the least-squares slope."""
    x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
    n = float(x.size)
    sx, sy = x.sum(), y.sum()
    return (n * (x * y).sum() - sx * sy) / (n * (x * x).sum() - sx * sx)


def unwrapped(phases):
    """a_waveguide.rs:64-80: a monotone phase out of one that wraps at ±π."""
    out, offset = [], 0.0
    for n, p in enumerate(phases):
        if n > 0:
            jump = p + offset - out[n - 1]
            if jump > math.pi:
                offset -= 2.0 * math.pi
            elif jump < -math.pi:
                offset += 2.0 * math.pi
        out.append(p + offset)
    return out


class Run:
    def __init__(self, dt, cutoff, stations, series):
        self.dt, self.cutoff, self.stations, self.series = dt, cutoff, stations, series

    def beta(self, frequency):
        """a_waveguide.rs:90-100: the propagation constant from the phase slope along the guide."""
        phases = [transform(s, frequency, self.dt)[1] for s in self.series]
        return -slope(self.stations, unwrapped(phases))


def guide(length):
    dx = 1.0 / ACROSS
    return oracle.Yee((ACROSS, 4, length), dx), dx


def launch(c, dx, carrier_over_cutoff, width_wavelengths):
    """a_waveguide.rs:124-158: both ends open, a TE10 Gaussian pulse six guide widths in."""
    a = ACROSS * dx
    c.set_boundary(ZLOW, "open")
    c.set_boundary(ZHIGH, "open")
    cutoff = c.cutoff_frequency((1, 0))
    wavelength = C0 / (cutoff * carrier_over_cutoff)
    dt = c.courant_limit() * 0.5
    k = 2.0 * math.pi / wavelength
    centre, width = 6.0 * a, width_wavelengths * wavelength

    def envelope(x, y, z):
        u = (z - centre) / width
        return np.sin(math.pi * x / a) * np.exp(-u * u) * np.cos(k * (z - centre))

    c.launch_along_z(dt, envelope)
    return cutoff, dt, envelope


def march(carrier_over_cutoff, width_wavelengths, first_cell, spacing, count):
    """a_waveguide.rs:117-204: the launched pulse recorded (Ey at x = a/2, y index 2) at `count`
    stations, stopped before either end's reflection returns."""
    c, dx = guide(ALONG)
    cutoff, dt, _ = launch(c, dx, carrier_over_cutoff, width_wavelengths)
    probes = np.array([first_cell + n * spacing for n in range(count)])
    nx, ny = ACROSS, 4
    at = ACROSS // 2 + (nx + 1) * (2 + ny * probes)  # electric_at(ACROSS/2, 2, p).y (cavity.rs:735-742)
    steps = int(0.8 * ALONG / 0.2887)
    series = np.empty((count, steps))
    for n in range(steps):
        assert c.step(dt) is None
        series[:, n] = c.fields()["ey"][at]
    return Run(dt, cutoff, probes * dx, series)


def test_above_cutoff_the_phase_turns_more_slowly_than_in_free_space():  # a_waveguide.rs:206-257
    worst, widest = 0.0, 1.0
    for carrier, ratios in [(1.5, [1.4, 1.5, 1.7]), (2.6, [2.1, 2.6, 3.1])]:
        run = march(carrier, 1.4, ALONG // 3, 4, 20)
        for ratio in ratios:
            f = run.cutoff * ratio
            beta = abs(run.beta(f))
            k = 2.0 * math.pi * f / C0
            kc = 2.0 * math.pi * run.cutoff / C0
            closed = math.sqrt(k * k - kc * kc)
            worst = max(worst, abs(beta / closed - 1.0))
            widest = max(widest, k / beta)
    assert worst < 0.04, f"the dispersion relation holds across the band: worst {worst:.4f}"
    assert widest > 1.4, f"near cutoff the guide wavelength is much longer than free space: {widest:.3f}"


def test_below_cutoff_the_mode_decays_without_being_absorbed():  # a_waveguide.rs:259-367
    dx = 1.0 / ACROSS
    a = ACROSS * dx
    probe = oracle.Yee((ACROSS, 4, 120), dx)
    cutoff = probe.cutoff_frequency((1, 0))
    dt = probe.courant_limit() * 0.5
    source = 40
    probes = np.array([source + 4 + n for n in range(14)])
    at = ACROSS // 2 + (ACROSS + 1) * (2 + 4 * probes)
    biases = []
    for ratio in (0.45, 0.6, 0.75):
        g = oracle.Yee((ACROSS, 4, 120), dx)
        g.set_boundary(ZHIGH, "open")  # ZLow stays a conductor (a_waveguide.rs:268-273)
        f = cutoff * ratio
        omega = 2.0 * math.pi * f
        period = 1.0 / f
        settle = int(16.0 * period / dt)
        window = int(round(4.0 * period / dt))
        series = np.empty((probes.size, window))
        for n in range(settle + window):
            t = n * dt
            assert g.step(dt) is None
            # impressed after the step (a_waveguide.rs:291-300)
            g.impress(source, lambda x, y, t=t: 0.02 * np.sin(math.pi * x / a) * math.sin(omega * t))
            if n >= settle:
                series[:, n - settle] = g.fields()["ey"][at]
        logs = [math.log(transform(s, f, dt)[0]) for s in series]
        alpha = -slope(probes * dx, logs)
        k = omega / C0
        kc = 2.0 * math.pi * cutoff / C0
        closed = math.sqrt(kc * kc - k * k)
        assert abs(alpha / closed - 1.0) < 0.08, (ratio, alpha, closed)
        biases.append(abs(alpha / closed - 1.0))
    # The reference reports its own run's biases, to the tenth of a percent, as 0.4%, 5.5% and 4.2%
    # (a_waveguide.rs:346-349): the same boundary, source and transform give the same three figures.
    assert [round(100.0 * b, 1) for b in biases] == [0.4, 5.5, 4.2], biases


def test_the_phase_velocity_and_the_group_velocity_multiply_to_c_squared():  # a_waveguide.rs:369-412
    run = march(2.0, 1.4, ALONG // 3, 4, 20)
    f = run.cutoff * 2.0
    step = f * 0.05
    b_lo, b_hi = abs(run.beta(f - step)), abs(run.beta(f + step))
    v_group = 2.0 * math.pi * 2.0 * step / (b_hi - b_lo)
    v_phase = 2.0 * math.pi * f / abs(run.beta(f))
    assert v_phase > C0
    assert v_group < C0
    assert abs(v_phase * v_group / (C0 * C0) - 1.0) < 0.05


def test_the_cutoff_is_a_property_of_the_cross_section():  # a_waveguide.rs:419-455
    dx = 1.0 / ACROSS
    short = oracle.Yee((ACROSS, 4, 40), dx)
    long = oracle.Yee((ACROSS, 4, 400), dx)
    assert abs(short.cutoff_frequency((1, 0)) - long.cutoff_frequency((1, 0))) < 1e-6
    closed = C0 / (2.0 * ACROSS * dx)
    assert abs(short.cutoff_frequency((1, 0)) / closed - 1.0) < 1e-12
    narrow = oracle.Yee((ACROSS // 2, 4, 40), dx)
    assert abs(narrow.cutoff_frequency((1, 0)) / short.cutoff_frequency((1, 0)) - 2.0) < 1e-12


def test_launch_along_z_sets_the_pulse_and_clears_the_conducting_walls():
    """cavity.rs:488-521: Ey is the envelope at its edges, Hx is −envelope/η half a step on, and the
    tangential E of the conducting x walls is zero; with open z ends those planes keep the pulse."""
    c, dx = guide(60)
    _, dt, envelope = launch(c, dx, 2.0, 1.4)
    nx, ny, nz = ACROSS, 4, 60
    f = c.fields()
    ey = f["ey"].reshape(nz + 1, ny, nx + 1)
    x = np.arange(nx + 1) * dx
    y = (np.arange(ny) + 0.5) * dx
    z = np.arange(nz + 1) * dx
    want = envelope(x[None, None, :], y[None, :, None], z[:, None, None]) * np.ones_like(ey)
    want[:, :, 0] = 0.0
    want[:, :, nx] = 0.0
    assert np.array_equal(ey, want)
    eta = math.sqrt(oracle.MU_0 / oracle.EPSILON_0)
    zh = (np.arange(nz) + 0.5) * dx + c.wave_speed * dt / 2.0
    hx = f["hx"].reshape(nz, ny, nx + 1)
    assert np.array_equal(hx, -(envelope(x[None, None, :], y[None, :, None], zh[:, None, None]) * np.ones_like(hx)) / eta)
    for k in ("ex", "ez", "hy", "hz"):
        assert not f[k].any()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_guide_matches_the_oracle(precision):
    """The launched guide of a_waveguide.rs (both ends open, 20 × 4 × 120 cells) for 200 steps: the
    device's own launch and walls, f64 bit for bit with the oracle, FP32 within f32 rounding."""
    from pantometry_b200.domains import Cavity

    o, dx = guide(120)
    g = Cavity((ACROSS, 4, 120), dx, precision=precision)
    _, dt, envelope = launch(o, dx, 2.0, 1.4)
    g.set_boundary(ZLOW, "open")
    g.set_boundary(ZHIGH, "open")
    assert g.cutoff_frequency((1, 0)) == o.cutoff_frequency((1, 0))
    g.launch_along_z(dt, envelope)
    want, got = o.fields(), g.fields()
    if precision == "f64":
        for k in want:
            assert np.array_equal(got[k].view(np.uint64), want[k].view(np.uint64)), k
    assert o.step(dt, 200) is None and g.step(dt, 200) is None
    want, got = o.fields(), g.fields()
    if precision == "f64":
        for k in want:
            assert np.array_equal(got[k].view(np.uint64), want[k].view(np.uint64)), k
    else:  # each error against the largest E (or H) value, as the other FP32 wall tests measure it
        scale = {q: max(max(np.abs(want[q + a]).max() for a in "xyz"), 1e-300) for q in "eh"}
        assert max(np.abs(got[k] - want[k]).max() / scale[k[0]] for k in want) < 1e-4
