"""Handles on a second GPU after the first.

A kernel's shared-memory opt-in belongs to the function on one device, so a library that set it
once per process would launch the >48 KB kernels (the TMA-staged hall, cavity and ensemble, the
plain f64 hall) on a second device without it and fail there. These tests step the same FP32 hall,
cavity and ensemble on cuda:0 and then on cuda:1 and compare the fields bit for bit. They skip on
a machine with one device.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _two_devices():
    from pantometry_b200.domains import device_count

    if device_count() < 2:
        pytest.skip("one CUDA device: the second-device cases need two")


def test_hall_on_the_second_device_after_the_first():
    _two_devices()
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(32, steps=20)
    out = []
    for dev in (0, 1):
        h = W.build_hall(cfg, precision="f32", device=dev)
        assert h.step(cfg["dt"], 20) is None
        out.append(h.fields()["p"])
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


def test_cavity_on_the_second_device_after_the_first():
    _two_devices()
    from pantometry_b200.domains import Cavity

    out = []
    for dev in (0, 1):
        c = Cavity((32, 24, 16), 1e-3, precision="f32", device=dev)
        dt = 0.9 * c.courant_limit()
        c.release_mode((1, 1), 1.0, dt)
        assert c.step(dt, 20) is None
        out.append(c.fields()["ey"])
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


def test_ensemble_on_the_second_device_after_the_first():
    _two_devices()
    from pantometry_b200 import workloads as W

    cfg = W.heat_ensemble(count=4, lo=16, hi=40)
    out = []
    for dev in (0, 1):
        e = W.build_ensemble(cfg, precision="f32", device=dev)
        assert e.step(20) is None
        out.append(e.download())
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))
