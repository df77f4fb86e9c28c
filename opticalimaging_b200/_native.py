"""ctypes binding of liboi_b200.so (declared in include/oi_b200.h).

The library is built in-tree by ``opticalimaging_b200.build``.  There is no fallback: if the library or a CUDA
device is missing, every imaging call raises.
"""
import ctypes
import os

import torch

from . import build as _build

_lib = None

_vp, _i, _ll, _d, _f = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_float
_SIGS = {
    'oi_version': [],
    'oi_twiddle': [_vp, _i, _i, _ll, _ll, _ll, _i, _d, _vp],
    'oi_band_spectrum': [_vp, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _f, _vp, _vp, _vp],
    'oi_abbe_pupils': [_vp, _vp, _i, _i, _vp, _vp, _vp, _i, _d, _vp, _i, _vp, _i, _vp, _d, _d, _d, _d, _vp, _vp,
                       _vp],
    'oi_coherent_coarse': [_vp, _i, _i, _i, _i, _vp, _ll, _vp, _i, _i, _i, _i, _vp, _vp, _i, _vp, _vp],
    'oi_coarse_to_image': [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp],
    'oi_tcc_pupils64': [_vp, _i, _vp, _i, _vp, _vp, _vp, _i, _d, _d, _vp, _i, _vp, _d, _d, _d, _d, _vp, _vp],
    'oi_tcc_pupils64_pol': [_vp, _i, _vp, _i, _vp, _vp, _vp, _i, _d, _d, _vp, _i, _vp, _d, _d, _d, _d, _vp, _vp],
    'oi_abbe_pupils_pol': [_vp, _vp, _i, _i, _vp, _vp, _vp, _i, _d, _vp, _i, _vp, _i, _vp, _d, _d, _d, _d, _vp,
                           _vp, _vp],
    'oi_tcc_assemble64': [_vp, _i, _i, _i, _vp, _vp],
    'oi_fft_supported': [_i, _i],
    'oi_band_spectrum_fft': [_vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _f, _vp, _vp, _vp],
    'oi_coarse_to_image_fft': [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp,
                               _vp],
    'oi_spectrum_to_image': [_vp, _i, _i, _i, _vp, _vp, _i, _i, _vp, _vp],
    'oi_spectrum_to_image_fft': [_vp, _i, _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp],
    'oi_coherent_adjoint': [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _i, _i, _vp, _i, _i, _vp, _vp, _i, _vp, _vp,
                            _vp],
    'oi_band_spectrum_noalloc': [_vp, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _f, _vp, _vp],
    'oi_coherent_coarse_fft': [_vp, _i, _i, _i, _i, _i, _i, _vp, _ll, _vp, _i, _i, _i, _i, _vp, _vp, _i, _vp, _vp],
    'oi_coherent_tc_layout': [_ll, _i, _vp, _vp],
    'oi_coherent_coarse_tc': [_vp, _i, _i, _i, _i, _i, _i, _vp, _ll, _vp, _i, _i, _vp, _i, _i, _vp, _vp],
    'oi_tc_constants': [_i, _i, _vp, _vp, _vp, _ll, _vp],
    'oi_device_status': [_vp, _i],
    'oi_launch_count': [_vp],
    'oi_wait_probe': [_ll, _i, _vp],
    'oi_eig_topk64_workspace': [_i, _i, _i, _i, _vp],
    'oi_eig_topk64': [_vp, _vp, _i, _i, _i, _i, _i, _i, _d, _vp, _vp, _vp, _ll, _vp, _vp],
    'oi_rows_tc_constants': [_i, _i, _i, _i, _vp, _ll, _vp],
    'oi_rows_fwd_tc': [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp],
    'oi_rows_fwd_tc_half': [_vp, _i, _i, _i, _i, _i, _vp, _vp, _vp],
    'oi_rows_inv_tc': [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp],
    'oi_rows_inv_tc_tiles': [_vp, _i, _i, _i, _vp, _vp, _vp],
    'oi_band_spectrum_tc': [_vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _f, _vp, _vp, _vp],
    'oi_coarse_half_spectrum_fft': [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp],
    'oi_band_spectrum_tc_sym': [_vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _f, _vp, _vp, _vp],
    'oi_coarse_to_image_tc': [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp],
    'oi_synth_tc_constants': [_i, _i, _i, _vp, _ll, _vp],
    'oi_synth_tiles_tc': [_vp, _i, _i, _i, _i, _vp, _i, _vp, _vp],
    'oi_coarse_to_image_tcs': [_vp, _i, _i, _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp],
}

FIELD_REAL_F32, FIELD_COMPLEX_C64, FIELD_U8 = 0, 1, 2
NOALLOC_SCRATCH_COMPLEX = 1 << 21   # OI_NOALLOC_SCRATCH_COMPLEX of include/oi_b200.h


class NativeError(RuntimeError):
    """A liboi_b200 entry point returned a non-zero status."""


def lib_path():
    return _build.LIB


def load(build_if_missing=True):
    """Load liboi_b200.so (building it first when it is missing or stale and nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_missing and (not os.path.exists(path) or _build.stale()):
        try:
            _build.build()
        except (OSError, RuntimeError) as e:
            if not os.path.exists(path):
                raise NativeError(f'liboi_b200.so is not built and the build failed: {e}') from e
    if not os.path.exists(path):
        raise NativeError(f'{path} missing: run `python -m opticalimaging_b200.build`')
    lib = ctypes.CDLL(path)
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.oi_last_error.argtypes = []
    lib.oi_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def exported_symbols():
    return ['oi_last_error'] + list(_SIGS)


def call(name, *args):
    """Call entry point `name`; raise NativeError with the library's message on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc < 0:
        msg = lib.oi_last_error().decode(errors='replace')
        raise NativeError(f'{name} failed ({rc}): {msg}')


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_handle(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def host_doubles(values):
    arr = (ctypes.c_double * len(values))(*[float(v) for v in values])
    return arr


def tc_layout(images: int, fields: int):
    """(ctas, nparts) of oi_coherent_coarse_tc for `images` coarse images of `fields` fields each."""
    ctas, nparts = ctypes.c_int(0), ctypes.c_int(0)
    call('oi_coherent_tc_layout', int(images), int(fields), ctypes.byref(ctas), ctypes.byref(nparts))
    return ctas.value, nparts.value


def device_status(reset: bool = False) -> int:
    """The device status word set by kernels whose bounded waits expired (0 = none); synchronous."""
    st = ctypes.c_int(0)
    call('oi_device_status', ctypes.byref(st), int(reset))
    return st.value


class DeviceWaitError(NativeError):
    """A kernel's bounded wait expired (the device status word was set): the results it wrote are invalid."""


def check_device_status(what: str, reader=None) -> None:
    """Raise DeviceWaitError if a kernel's bounded wait has expired since the last check (the status word is
    then cleared, so the next work starts clean).  Call it after synchronising with the work it covers.
    `reader(reset)` replaces device_status (tests)."""
    read = device_status if reader is None else reader
    st = read(False)
    if st:
        read(True)
        raise DeviceWaitError(f'{what}: a kernel ended early on an expired wait (device status {st}); its results '
                              'are invalid')


def launch_count() -> int:
    """Kernel launches the library has enqueued so far (graph replays are not counted)."""
    n = ctypes.c_longlong(0)
    call('oi_launch_count', ctypes.byref(n))
    return n.value
