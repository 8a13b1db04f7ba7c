"""The entry point that allocates nothing, against the handle-based one.

Some callers of this library cannot allocate device memory — a host that owns all device memory
through its own pool, a plugin inside such a host, code that must not cause the synchronisation
cudaMalloc/cudaFree can. `pm_hall_step_f32_noalloc` serves them: the caller passes device buffers
for the old and new state, and the kernel's scratch lives in a fixed array inside the library.

This test (in its own file, collected last) drives it through the C ABI on buffers the test owns,
two calls in a row, and checks each result against `pm_hall_step` on a handle holding the same
state: fields and invariant within the f32 tests' tolerance.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_hall_step_matches_the_handle_two_calls_in_a_row():
    import torch

    from pantometry_b200 import _native as N
    from pantometry_b200 import workloads as W
    from pantometry_b200.domains import Hall

    cfg = W.acoustic_hall(40, steps=4, source=False)
    w, h, d = cfg["size"]
    ref = Hall(w, h, d, cfg["across"], cfg["speed"], cfg["density"], precision="f32")
    ref.release(cfg["pressure"])
    nx, ny, nz = ref.nodes
    dt = cfg["dt"]

    dev = torch.device("cuda", 0)
    p = torch.tensor(cfg["pressure"], dtype=torch.float64, device=dev).float()
    state = [p, torch.zeros((nx - 1) * ny * nz, device=dev), torch.zeros(nx * (ny - 1) * nz, device=dev),
             torch.zeros(nx * ny * (nz - 1), device=dev)]
    lib = N.load()
    for call in range(2):
        out = [torch.empty_like(t) for t in state]
        inv = C.c_double(0.0)
        torch.cuda.synchronize()
        st = lib.pm_hall_step_f32_noalloc(nx, ny, nz, ref.dx, cfg["speed"], cfg["density"], dt, 1 if call == 0 else 0,
                                          *[C.c_void_p(t.data_ptr()) for t in state],
                                          *[C.c_void_p(t.data_ptr()) for t in out],
                                          C.c_void_p(torch.cuda.current_stream().cuda_stream), C.byref(inv))
        assert st == N.PM_OK, lib.pm_last_error().decode()
        assert ref.step(dt, 1) is None
        want = ref.fields()
        for name, got in zip(("p", "vx", "vy", "vz"), out):
            g = got.double().cpu().numpy()
            scale = max(np.abs(want[name]).max(), 1e-30)
            assert np.abs(g - want[name]).max() <= 1e-6 * scale, (call, name)
        want_inv = ref.ledger()["parts"][0]
        assert abs(inv.value - want_inv) <= 1e-12 * abs(want_inv), (call, inv.value, want_inv)
        state = out


def test_noalloc_refuses_sizes_beyond_its_limits():
    """Refusals happen on the host, before anything reaches the GPU: a grid of 2^32 nodes or more
    (the kernel's 32-bit node index), a step past the Courant limit, a non-positive step, and an
    output buffer that is also an input or another output (the kernel reads neighbours' old
    values while it writes new ones)."""
    import torch

    from pantometry_b200 import _native as N

    lib = N.load()
    bufs = [torch.zeros(8, device="cuda") for _ in range(8)]
    ptrs = [C.c_void_p(t.data_ptr()) for t in bufs]
    inv = C.c_double(0.0)
    st = lib.pm_hall_step_f32_noalloc(2048, 2048, 1024, 1.0, 1.0, 1.0, 0.1, 1, *ptrs, None, C.byref(inv))
    assert st == N.PM_BAD_ARG and b"2^32" in lib.pm_last_error()
    st = lib.pm_hall_step_f32_noalloc(4, 2, 1, 1.0, 1.0, 1.0, 10.0, 1, *ptrs, None, C.byref(inv))
    assert st == N.PM_VIOLATION and b"Courant" in lib.pm_last_error()
    st = lib.pm_hall_step_f32_noalloc(4, 2, 1, 1.0, 1.0, 1.0, 0.0, 1, *ptrs, None, C.byref(inv))
    assert st == N.PM_BAD_ARG and b"dt" in lib.pm_last_error()
    for out, same in ((4, 0), (5, 1), (7, 3), (6, 5)):
        aliased = list(ptrs)
        aliased[out] = ptrs[same]
        st = lib.pm_hall_step_f32_noalloc(4, 2, 1, 1.0, 1.0, 1.0, 0.1, 1, *aliased, None, C.byref(inv))
        assert st == N.PM_BAD_ARG and b"output buffer" in lib.pm_last_error(), (out, same)


def test_noalloc_on_a_second_device_after_the_first():
    """The array exists once per GPU that loads the library; a call on the second device after one
    on the first looks up that device's own copy and gives the same fields."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device: the second-device case needs two")
    from pantometry_b200 import _native as N
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(24, steps=2, source=False)
    lib = N.load()
    results = []
    for d in (0, 1):
        with torch.cuda.device(d):
            dev = torch.device("cuda", d)
            nx = ny = nz = 24
            p = torch.tensor(cfg["pressure"], dtype=torch.float64, device=dev).float()
            state = [p, torch.zeros((nx - 1) * ny * nz, device=dev), torch.zeros(nx * (ny - 1) * nz, device=dev),
                     torch.zeros(nx * ny * (nz - 1), device=dev)]
            out = [torch.empty_like(t) for t in state]
            inv = C.c_double(0.0)
            torch.cuda.synchronize(dev)
            st = lib.pm_hall_step_f32_noalloc(nx, ny, nz, cfg["size"][0] / (nx - 1), cfg["speed"], cfg["density"], cfg["dt"], 1,
                                              *[C.c_void_p(t.data_ptr()) for t in state],
                                              *[C.c_void_p(t.data_ptr()) for t in out],
                                              C.c_void_p(torch.cuda.current_stream(dev).cuda_stream), C.byref(inv))
            assert st == N.PM_OK, lib.pm_last_error().decode()
            results.append(([t.cpu() for t in out], inv.value))
    for a, b in zip(results[0][0], results[1][0]):
        assert torch.equal(a, b)
    assert results[0][1] == results[1][1]
