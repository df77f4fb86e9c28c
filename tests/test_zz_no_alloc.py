"""oi_band_spectrum_noalloc: the band spectrum for callers that cannot allocate device memory.

Such a caller only holds the pointers a host application hands it (its inputs and its output) and may not
create a scratch buffer of its own.  The entry point keeps its scratch in an array built into the library.
This file is collected last so that a run stopping at its first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest
import torch

from tests.fixtures import rel_err

pytestmark = pytest.mark.gpu

TOL = 2e-6   # the band-spectrum tolerance of the other GPU tests


def _call_noalloc(lib, field, kind, nch, plan, out, stream):
    from opticalimaging_b200 import _native as N
    b = plan.band
    return lib.oi_band_spectrum_noalloc(N.ptr(field), kind, field.shape[0], plan.ny, plan.nx, nch, b.br, b.bc,
                                        N.ptr(plan.wx), N.ptr(plan.wy), ctypes.c_float(1.0 / (plan.ny * plan.nx)),
                                        N.ptr(out), stream)


def test_noalloc_band_spectrum_matches_scratch_form_twice():
    from opticalimaging_b200 import _native as N, engine as E
    lib = N.load()
    dev = torch.device('cuda')
    rng = np.random.default_rng(2024)
    stream = N.stream_handle(dev)
    cases = [  # (grid, band, kind, channels): two calls in a row with different data and shapes
        ((256, 192), E.Band(-20, 41, -15, 31), N.FIELD_REAL_F32, 1),
        ((96, 128), E.Band(-11, 23, -30, 61), N.FIELD_COMPLEX_C64, 3),
    ]
    for (ny, nx), band, kind, nch in cases:
        plan = E.Plan.get(ny, nx, band, dev)
        if kind == N.FIELD_REAL_F32:
            field = torch.from_numpy(rng.random((3, ny, nx), dtype=np.float32)).to(dev)
        else:
            f = rng.standard_normal((2, ny, nx, nch)) + 1j * rng.standard_normal((2, ny, nx, nch))
            field = torch.from_numpy(f.astype(np.complex64)).to(dev)
        # the existing entry point, with a caller-provided scratch buffer
        ref = E.band_spectrum(field, kind, plan, nch=nch, form='dft')
        out = torch.full_like(ref, float('nan'))
        assert _call_noalloc(lib, field, kind, nch, plan, out, stream) == 0, lib.oi_last_error()
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < TOL


def test_noalloc_rejects_oversize_before_launching():
    from opticalimaging_b200 import _native as N, engine as E
    lib = N.load()
    dev = torch.device('cuda')
    plan = E.Plan.get(256, 256, E.Band(-29, 59, -29, 59), dev)
    field = torch.zeros((1, 256, 256), device=dev)
    out = torch.zeros((1, 1, 59, 59), dtype=torch.complex64, device=dev)
    b = plan.band
    too_many = N.NOALLOC_SCRATCH_COMPLEX // (256 * 59) + 1   # one image more than the built-in scratch holds
    rc = lib.oi_band_spectrum_noalloc(N.ptr(field), N.FIELD_REAL_F32, too_many, 256, 256, 1, b.br, b.bc,
                                      N.ptr(plan.wx), N.ptr(plan.wy), ctypes.c_float(1.0), N.ptr(out),
                                      N.stream_handle(dev))
    assert rc == -3
    assert b'built-in scratch' in lib.oi_last_error()


def test_noalloc_calls_allocate_no_device_memory():
    """The property the entry point exists for: after a first call, further calls leave the device's free
    memory and torch's reserved pool exactly as they were."""
    from opticalimaging_b200 import _native as N, engine as E
    lib = N.load()
    dev = torch.device('cuda')
    stream = N.stream_handle(dev)
    plan = E.Plan.get(256, 256, E.Band(-20, 41, -20, 41), dev)
    field = torch.from_numpy(np.random.default_rng(7).random((4, 256, 256), dtype=np.float32)).to(dev)
    out = torch.empty((4, 1, 41, 41), dtype=torch.complex64, device=dev)
    assert _call_noalloc(lib, field, N.FIELD_REAL_F32, 1, plan, out, stream) == 0, lib.oi_last_error()
    torch.cuda.synchronize()
    free0, reserved0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
    for _ in range(50):
        assert _call_noalloc(lib, field, N.FIELD_REAL_F32, 1, plan, out, stream) == 0, lib.oi_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == reserved0
