"""`Cavity`'s closed forms, restating the rest of crates/pantometry-em/tests/against_closed_forms.rs
(the ∇·B, energy-swing, lossy and open-box tests are restated with the other pins):
  * a released (1, 1) mode rings at the cavity frequency, the error falling at second order from
    8 to 32 cells (each refinement 2.6–6×) to under 1% (:110-215);
  * a standing mode shares its energy equally between E and H, averaged over 4000 steps, to 2%
    (:289-312);
  * the limit is COURANT_3D·dx/c, 0.1% past it is refused as the "Courant number", and the limit
    itself is taken (:314-337);
  * the sharpest mode holds at 0.98 of the limit and is refused at 1.15 (:339-385);
  * Mur's coefficient depends on c·dt/dx alone (:524-547).
The device passes the same bounds in f64 and FP32 and refuses where the oracle does; its f64
figures agree with the oracle's to 1e-6 (its energies are summed in a different order, so the
figures derived from them are not compared bit for bit; the fields themselves are, elsewhere).
"""
import math

import pytest

import oracle

DX = 2e-3  # against_closed_forms.rs:11
COURANT_3D = 0.577_350_269_189_625_8  # cavity.rs:15


def box_of(counts, dx=DX, make=None, precision="f64", eps_r=1.0):
    if make is None:
        return oracle.Yee(counts, dx, eps_r=eps_r)
    return make(counts, dx, eps_r=eps_r, precision=precision)


def released(counts, mode, make=None, precision="f64", dx=DX):
    """against_closed_forms.rs:17-22: released at half the limit."""
    c = box_of(counts, dx, make, precision)
    dt = c.courant_limit() * 0.5
    c.release_mode(mode, 1.0, dt)
    return c, dt


def ring_error(cells, make=None, precision="f64"):
    """against_closed_forms.rs:110-190: time 200 peaks of the electric energy (a parabola through
    each local maximum) and compare the frequency with (c/2)·√((1/Lx)² + (1/Lz)²)."""
    dx = 0.048 / cells
    c, dt = released((cells, 4, cells), (1, 1), make, precision, dx)
    size = [cells * dx, 4 * dx, cells * dx]
    closed = 0.5 * C_VACUUM * math.sqrt((1.0 / size[0]) ** 2 + (0.0 / size[1]) ** 2 + (1.0 / size[2]) ** 2)
    cycles = 200
    t = 0.0
    window = [(0.0, c.energies()[0])] * 3
    peaks = []
    for _ in range(200_000):
        assert c.step(dt) is None
        t += dt
        window = [window[1], window[2], (t, c.energies()[0])]
        if window[1][1] > window[0][1] and window[1][1] >= window[2][1]:
            a, b, cc = window[0][1], window[1][1], window[2][1]
            denom = a - 2.0 * b + cc
            shift = 0.5 * (a - cc) / denom if abs(denom) > 0.0 else 0.0
            peaks.append(window[1][0] + shift * dt)
            if len(peaks) > cycles:
                break
    assert len(peaks) > cycles
    half_period = (peaks[cycles] - peaks[0]) / cycles
    return abs((0.5 / half_period) / closed - 1.0)


C_VACUUM = 1.0 / math.sqrt(oracle.EPSILON_0 * oracle.MU_0)


def check_ring(make=None, precision="f64"):
    errors = [ring_error(n, make, precision) for n in (8, 16, 32)]
    for lo, hi in zip(errors, errors[1:]):
        assert 2.6 < lo / hi < 6.0, errors
    assert errors[2] < 0.01, errors
    return errors


def check_equipartition(make=None, precision="f64"):
    c, dt = released((10, 6, 10), (1, 1), make, precision)
    e_sum = h_sum = 0.0
    for _ in range(4000):
        assert c.step(dt) is None
        e, h = c.energies()
        e_sum += e
        h_sum += h
    assert abs(e_sum / h_sum - 1.0) < 0.02
    return e_sum, h_sum


def check_courant(make=None, precision="f64"):
    c = box_of((8, 8, 8), make=make, precision=precision)
    limit = c.courant_limit()
    assert abs(limit / (COURANT_3D * DX / 299_792_458.0) - 1.0) < 1e-9
    v = c.step(limit * 1.001)
    assert v is not None and v["quantity"] == "Courant number"
    assert c.step(limit) is None


def check_growth(make=None, precision="f64"):
    for factor, should_grow in ((0.98, False), (1.15, True)):
        c = box_of((10, 10, 10), make=make, precision=precision)
        dt = c.courant_limit() * factor
        c.release_mode((5, 5), 1.0, c.courant_limit() * 0.5)
        start = sum(c.energies())
        grew = False
        for _ in range(600):
            if c.step(dt) is not None or not math.isfinite(sum(c.energies())):
                grew = True
                break
        grew = grew or sum(c.energies()) > 100.0 * start
        assert grew == should_grow, factor


def test_the_cavity_rings_at_the_closed_form_frequency():  # :110-215
    check_ring()


def test_a_standing_mode_shares_its_energy_equally():  # :289-312
    check_equipartition()


def test_past_the_courant_limit_is_refused():  # :314-337
    check_courant()


def test_the_limit_is_where_the_field_starts_to_grow():  # :339-385
    check_growth()


def test_the_mur_coefficient_is_a_function_of_the_courant_number_alone():  # :524-547
    a = box_of((8, 8, 8))
    b = box_of((8, 8, 8), DX * 3.0, eps_r=4.0)  # Medium::dielectric(4.0)
    s = 0.4
    ka = a.mur_coefficient(a.courant_limit() * s)
    kb = b.mur_coefficient(b.courant_limit() * s)
    assert abs(ka - kb) < 1e-12
    assert abs(ka - (COURANT_3D * s - 1.0) / (COURANT_3D * s + 1.0)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_device_cavity_closed_forms(precision):
    from pantometry_b200.domains import Cavity

    got = check_equipartition(Cavity, precision)
    if precision == "f64":
        want = check_equipartition()
        assert abs(got[0] / got[1] - want[0] / want[1]) < 1e-9
    check_courant(Cavity, precision)
    check_growth(Cavity, precision)
    got = check_ring(Cavity, precision)
    if precision == "f64":
        want = check_ring()
        assert all(abs(g / w - 1.0) < 1e-6 for g, w in zip(got, want)), (got, want)
