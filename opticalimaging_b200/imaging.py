"""Drop-in imaging entry points with the reference's names, arguments and return values.

* ``CalculateAbbeImage``, ``CalculateHopkinsImage``, ``CalculateOptimized``  (CalculateAerialImage.py:18-152)
* ``CalculateTCCMatrix``, ``GetTCCMatrix``                                   (CalculateTCCMatrix.py:9-75)
* ``DecomposeTCC_SOCS``                                                       (DecomposeTCC_SOCS.py:3-37)
* ``CalculateAerialImage_SOCS``, ``CalculateSOCS``                            (CalculateAerialImage_SOCS.py:3-32)
* ``CalculateCharacteristicMatrix``                                           (CalculateCharacteristicMatrix.py:3-17)
* ``calculate_spectrum`` behind ``Scatter.CalculateSpectrum``                 (Scatter.py:10-35)

All numerical work runs in liboi_b200 on the current CUDA device.  Results come back on the device of the
caller's ``ScatterField`` (CPU in, CPU out), with the reference's shapes.  Precision: FP32 transforms with FP64
pupil synthesis; the TCC and its eigendecomposition are FP64 (so ``CalculateTCCMatrix`` returns complex128).

Divergences from the reference, all deliberate and documented:
* ``Hopkins_SettingType='threshold'`` works (the reference raises on a multi-element comparison): K is the
  smallest count whose leading eigenvalues reach the threshold fraction of the trace.
* An ``ImageCalculationMode`` other than 'scalar'/'vector' raises ValueError (the reference fails later with
  UnboundLocalError or IndexError).
* Out-of-domain optics (NA/Magnification > IndexImage, or NA >= 1, where the reference's obliquity and defocus
  roots go negative) produce the reference's NaN image and a RuntimeWarning.
"""
from __future__ import annotations

import ctypes
import threading
import warnings

import torch
from torch.utils.weak import WeakIdKeyDictionary

from . import _native as N
from .engine import (Band, CoherentModel, Plan, SocsKernels, abbe_band, band_spectrum, coherent_image,
                     require_cuda)
from .params import ImageData, cartesian_to_polar  # noqa: F401

__all__ = ['CalculateAbbeImage', 'CalculateHopkinsImage', 'CalculateOptimized', 'CalculateTCCMatrix',
           'GetTCCMatrix', 'DecomposeTCC_SOCS', 'CalculateAerialImage_SOCS', 'CalculateSOCS',
           'CalculateCharacteristicMatrix', 'calculate_spectrum', 'socs_kernels_from_tcc', 'socs_model',
           'abbe_model']


# ------------------------------------------------------------------------------------------- helpers
def _mode(numerics):
    m = numerics.ImageCalculationMode
    if m not in ('scalar', 'vector'):
        raise ValueError(f"ImageCalculationMode must be 'scalar' or 'vector', got {m!r}")
    return m == 'vector'


def _check_domain(projector):
    na, mag, n = float(projector.NA), float(projector.Magnification), float(projector.IndexImage)
    if na / mag > n or na >= 1.0:
        warnings.warn(f'optics outside the model domain (NA={na}, Magnification={mag}, IndexImage={n}): the '
                      'obliquity or defocus root is negative inside the pupil and the image is NaN, as in the '
                      'reference', RuntimeWarning, stacklevel=3)


def _jones(source):
    px, py = (complex(v) for v in source.PolarizationVector)
    return N.host_doubles([px.real, px.imag, py.real, py.imag])


def _zernike(projector):
    z = torch.as_tensor(projector.Aberration_Zernike, dtype=torch.float64).flatten().tolist()
    z = (z + [0.0] * 37)[:37]
    return N.host_doubles(z)


def _focus_list(projector):
    return [float(v) for v in torch.as_tensor(projector.FocusRange).flatten().tolist()]


def _axes(scatter, projector, source):
    """The reference's float32 spectrum axes f (X, columns) and g (Y, rows) (Scatter.py:15-18)."""
    ny, nx = scatter.ScatterField.shape[0], scatter.ScatterField.shape[1]
    npx = scatter.Period_X / (source.Wavelength / projector.NA)
    npy = scatter.Period_Y / (source.Wavelength / projector.NA)
    f = (1 / npx) * torch.arange(-(nx // 2), (nx + 1) // 2)
    g = (1 / npy) * torch.arange(-(ny // 2), (ny + 1) // 2)
    return f, g, npx, npy


class _HostStage:
    """Pinned staging for host-to-device copies of pageable host tensors (what a reference caller passes): the
    tensor moves in 4 MiB chunks through four pinned buffers, the host-side copy of one chunk (torch's threaded
    memcpy) overlapping the DMA of the ones before it; pageable copies go through the driver's own bounce buffer at
    a fraction of the link rate.  (24 MiB: 0.73 ms, against 0.82 ms with two 8 MiB buffers and 2.5 ms through a
    pageable copy; the host link moves it in 0.49 ms from pinned memory.)"""
    CHUNK, NBUF = 4 << 20, 4

    def __init__(self):
        self.bufs, self.events, self.lock = None, None, threading.Lock()

    def to_device(self, host: torch.Tensor, dev) -> torch.Tensor:
        flat = host.contiguous().view(torch.uint8).reshape(-1)
        out = torch.empty(flat.numel(), dtype=torch.uint8, device=dev)
        # the host-side copies move 8-byte words (a byte-typed copy runs element by element, at a few GB/s)
        word = torch.int64 if flat.numel() % 8 == 0 else torch.uint8
        with self.lock:
            if self.bufs is None:
                self.bufs = [torch.empty(self.CHUNK, dtype=torch.uint8, pin_memory=True) for _ in range(self.NBUF)]
                self.events = [None] * self.NBUF
            stream = torch.cuda.current_stream(dev)
            for k, a in enumerate(range(0, flat.numel(), self.CHUNK)):
                b = min(flat.numel(), a + self.CHUNK)
                i = k % self.NBUF
                if self.events[i] is not None:
                    self.events[i].synchronize()          # the buffer's previous chunk has left for the device
                self.bufs[i][:b - a].view(word).copy_(flat[a:b].view(word))
                out[a:b].copy_(self.bufs[i][:b - a], non_blocking=True)
                self.events[i] = torch.cuda.Event()
                self.events[i].record(stream)
        return out.view(host.dtype).reshape(host.shape)


_STAGE = _HostStage()


class _DropInField:
    """A drop-in call's ScatterField [Ny, Nx, C] on the device, reduced to what carries it.

    real: float32 [Ny, Nx] when the field is one real channel (channel 0; every other channel and every imaginary
    part zero: the thin masks a reference caller usually passes), else None.  live: the indices of the channels
    that are not all zero ([0] when none is: the reference transforms every channel, CalculateAerialImage.py:76-86,
    and a zero channel adds nothing).  One reduction on the device and one host read decide both."""

    def __init__(self, scatter, dev):
        h = torch.as_tensor(scatter.ScatterField)
        if h.dim() != 3:
            raise ValueError('ScatterField must be [Ny, Nx, C]')
        self.ny, self.nx, self.nch = h.shape
        if h.device.type == 'cpu' and not h.is_pinned() and h.numel() * h.element_size() >= (4 << 20):
            h = _STAGE.to_device(h.contiguous(), dev)
        self._cplx = h.to(dev).to(torch.complex64).contiguous()
        nz = (torch.view_as_real(self._cplx) != 0).any(dim=(0, 1)).tolist()   # [C][re, im]
        self.real = None
        if not nz[0][1] and not any(re or im for re, im in nz[1:]):
            self.real = self._cplx[:, :, 0].real.contiguous()
        self.live = [c for c in range(self.nch) if nz[c][0] or nz[c][1]] or [0]

    def carrier(self) -> torch.Tensor:
        """What the imaging takes: the real channel (float32 [Ny, Nx]) when there is one, else live_complex()."""
        return self.real if self.real is not None else self.live_complex()

    def live_complex(self) -> torch.Tensor:
        """The live channels as complex64 [Ny, Nx, L] on the device."""
        h = self._cplx if len(self.live) == self.nch else self._cplx[:, :, self.live]
        return h.contiguous()

    def pupil_image(self, scatter, projector, source, dev):
        """PupilImage of Scatter.CalculateSpectrum (Scatter.py:22-33): the cropped centred spectrum [br, bc, C], NaN
        outside the unit disc; the live channels are transformed (from the real channel when there is one), the
        others are zero."""
        f, g, npx, npy = _axes(scatter, projector, source)
        band, ph, outside, sl = _pupil_geometry(self.ny, self.nx, f, g, npx, npy, dev)
        if self.real is not None and sl is None:
            plan = Plan.get(self.ny, self.nx, band, dev)
            part = band_spectrum(self.real.unsqueeze(0), N.FIELD_REAL_F32, plan, scale=npx * npy)[0]
            part = part.permute(1, 2, 0) * ph[:, :, None]
        else:
            part = _spectrum_band(self.live_complex(), band, npx * npy, dev, ph)
        if len(self.live) == self.nch:
            hk = part
        else:
            hk = torch.zeros((band.br, band.bc, self.nch), dtype=torch.complex64, device=dev)
            hk[:, :, self.live] = part
        if sl is not None:
            hk = hk[sl]
        return hk.masked_fill(outside[:, :, None], float('nan'))


def _device_field(scatter, dev):
    """ScatterField [Ny, Nx, C] as a contiguous complex64 device tensor (one host-to-device copy; large pageable
    host fields go through the pinned staging)."""
    h = torch.as_tensor(scatter.ScatterField)
    if h.device.type == 'cpu' and not h.is_pinned() and h.numel() * h.element_size() >= (4 << 20):
        h = _STAGE.to_device(h.contiguous(), dev)
    return h.to(dev).to(torch.complex64).contiguous()


def _to_host(t: torch.Tensor, rd) -> torch.Tensor:
    """`t` on the result device `rd`; a host result is copied asynchronously into pinned memory (the caller's
    synchronisation, _check, completes it)."""
    if rd.type != 'cpu':
        return t.to(rd)
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    out.copy_(t, non_blocking=True)
    return out


def _live_channels(hfull):
    """The channels of a device field [Ny, Nx, C] that are not all zero, as one contiguous tensor (the
    reference transforms every channel, CalculateAerialImage.py:76-86; a zero channel adds nothing).  One
    reduction and one host read decide all channels."""
    live = torch.nonzero((hfull != 0).flatten(0, 1).any(dim=0)).flatten().tolist() or [0]
    h = hfull if len(live) == hfull.shape[2] else hfull[:, :, live]
    return h.contiguous()


def _field_on_device(scatter, dev):
    """ScatterField [Ny, Nx, C] as complex64 on the device, with all-zero channels dropped."""
    return _live_channels(_device_field(scatter, dev))


_SOCS_CACHE = WeakIdKeyDictionary()   # reference-layout kernel tensor -> (its version, SocsKernels)


def _socs_kernels_of(kernels, dev) -> SocsKernels:
    """The band form of a reference-layout kernel array [Ny, Nx, K] (what DecomposeTCC_SOCS returns), found once
    per tensor: later calls with the same, unmodified tensor object reuse it (the scan and any host-to-device
    copy of the full-grid array happen once).  Kernels from this module's DecomposeTCC_SOCS are registered at
    creation."""
    if isinstance(kernels, SocsKernels):
        return kernels
    t = torch.as_tensor(kernels)
    hit = _SOCS_CACHE.get(t) if isinstance(kernels, torch.Tensor) else None
    if hit is not None and hit[0] == t._version and hit[1].device == dev:
        return hit[1]
    sk = SocsKernels.from_full_grid(t.to(dev))
    if isinstance(kernels, torch.Tensor):
        _SOCS_CACHE[kernels] = (kernels._version, sk)
    return sk


def _check(what):
    """Raise if a kernel of this call ended early on an expired bounded wait: the caller's stream is synchronised
    first (the results are about to be returned anyway), so the status word covers the kernels the call launched."""
    torch.cuda.current_stream().synchronize()
    N.check_device_status(what)


def _result_device(scatter):
    h = scatter.ScatterField
    return h.device if isinstance(h, torch.Tensor) else torch.device('cpu')


_PUPIL_GEOMETRY: dict = {}   # (grid, pupil radius in frequencies, device) -> what _pupil_image needs of it


def _pupil_geometry(ny, nx, f, g, npx, npy, dev):
    """The grid-dependent part of PupilImage, built once per grid and pupil: the crop band (or the full band and
    the reference's slices when the crop leaves the grid), the centring phase on it and the mask of the samples
    outside the unit disc, on the device."""
    key = (ny, nx, float(npx), float(npy), str(dev))
    geo = _PUPIL_GEOMETRY.get(key)
    if geo is None:
        ox, oy = int(npx) + 3, int(npy) + 3
        r0, c0 = ny // 2 - oy, nx // 2 - ox
        sl = None
        if r0 >= 0 and c0 >= 0 and ny // 2 + oy <= ny and nx // 2 + ox <= nx:
            band = Band(r0 - ny // 2, 2 * oy, c0 - nx // 2, 2 * ox)
            fm, gm = torch.meshgrid(g[r0:r0 + 2 * oy], f[c0:c0 + 2 * ox], indexing='ij')
        else:   # crop window leaves the grid: Python slicing of the full spectrum, as the reference does
            band = Band(-(ny // 2), ny, -(nx // 2), nx)
            fm, gm = torch.meshgrid(g, f, indexing='ij')
            sl = (slice(ny // 2 - oy, ny // 2 + oy), slice(nx // 2 - ox, nx // 2 + ox))
            fm, gm = fm[sl], gm[sl]
        outside = (fm ** 2 + gm ** 2 > 1).to(dev)
        if len(_PUPIL_GEOMETRY) >= 64:
            _PUPIL_GEOMETRY.clear()
        geo = _PUPIL_GEOMETRY[key] = (band, _centring_phase(ny, nx, band).to(dev), outside, sl)
    return geo


def _pupil_image(scatter, projector, source, h, dev):
    """PupilImage of Scatter.CalculateSpectrum (Scatter.py:22-33): the cropped centred spectrum, NaN outside
    the unit disc."""
    ny, nx = h.shape[0], h.shape[1]
    f, g, npx, npy = _axes(scatter, projector, source)
    band, ph, outside, sl = _pupil_geometry(ny, nx, f, g, npx, npy, dev)
    hk = _spectrum_band(h, band, npx * npy, dev, ph)
    if sl is not None:
        hk = hk[sl]
    return hk.masked_fill(outside[:, :, None], float('nan'))


def _centring_phase(ny, nx, band: Band) -> torch.Tensor:
    """exp(-2 pi i m (N//2)/N) per axis on `band`: [br, bc] complex64 (host)."""
    mr = torch.arange(band.m0r, band.m0r + band.br, dtype=torch.float64)
    mc = torch.arange(band.m0c, band.m0c + band.bc, dtype=torch.float64)
    ph = torch.exp(-2j * torch.pi * ((mr * (ny // 2) % ny / ny)[:, None] + (mc * (nx // 2) % nx / nx)[None, :]))
    return ph.to(torch.complex64)


def _spectrum_band(h, band: Band, scale, dev, ph: torch.Tensor | None = None):
    """Centred spectrum Hk on `band` of a [Ny, Nx, C] complex64 device field -> [br, bc, C].

    The engine's band spectrum has its origin at pixel 0; the reference's centred spectrum has it at pixel
    N//2 (ifftshift before the transform, Scatter.py:20), i.e. an extra phase exp(-2 pi i m (N//2)/N) per axis
    (`ph`, [br, bc] on the device, when the caller holds it).  The phase cancels in every intensity, so only the
    spectrum outputs apply it.
    """
    ny, nx, nch = h.shape
    plan = Plan.get(ny, nx, band, dev)
    c = band_spectrum(h.unsqueeze(0), N.FIELD_COMPLEX_C64, plan, nch=nch, scale=scale)
    if ph is None:
        ph = _centring_phase(ny, nx, band).to(dev)
    return c[0].permute(1, 2, 0) * ph[:, :, None]


def calculate_spectrum(scatter, projector, source):
    """Hk [Ny, Nx, 3], f, g and PupilImage (Scatter.py:10-35), computed on the device."""
    dev = require_cuda()
    h = torch.as_tensor(scatter.ScatterField).to(dev).to(torch.complex64).contiguous()
    ny, nx = h.shape[0], h.shape[1]
    f, g, npx, npy = _axes(scatter, projector, source)
    hk = _spectrum_band(h, Band(-(ny // 2), ny, -(nx // 2), nx), npx * npy, dev)
    pim = _pupil_image(scatter, projector, source, h, dev)
    rd = _result_device(scatter)
    return hk.to(rd), f, g, pim.to(rd)


def _image_data(intensity, scatter, projector):
    out = ImageData()
    out.Intensity = intensity
    out.ImageX = torch.linspace(-scatter.Period_X / 2, scatter.Period_X / 2, scatter.ScatterField.shape[1])
    out.ImageY = torch.linspace(-scatter.Period_Y / 2, scatter.Period_Y / 2, scatter.ScatterField.shape[0])
    out.ImageZ = projector.FocusRange
    return out


# ----------------------------------------------------------------------------------------------- Abbe
def abbe_model(source, projector, numerics, period_y, period_x, ny, nx, focus=None, pack=True) -> CoherentModel:
    """Abbe pupils of every (focus plane, source point, field component) resident on the device
    (CalculateAerialImage.py:30-75): a CoherentModel whose image() is the Abbe image of a batch of masks."""
    vector = _mode(numerics)
    _check_domain(projector)
    dev = require_cuda()
    sd = source.Calc_SourceSimple()
    X, Y, V = (t.reshape(-1).to(torch.float32) for t in (sd.X, sd.Y, sd.Value))
    zs = _focus_list(projector) if focus is None else [float(z) for z in focus]
    npx = period_x / (source.Wavelength / projector.NA)
    npy = period_y / (source.Wavelength / projector.NA)
    f = (1 / npx) * torch.arange(-(nx // 2), (nx + 1) // 2)
    g = (1 / npy) * torch.arange(-(ny // 2), (ny + 1) // 2)
    nsrc = X.numel()
    if nsrc == 0:
        raise ValueError('the source has no points above the weight threshold')
    band = abbe_band(ny, nx, npy, npx, X, Y)
    if band is None:
        return None
    ne = 3 if vector else 1
    fr = g[band.m0r + ny // 2: band.m0r + ny // 2 + band.br].to(dev)
    fc = f[band.m0c + nx // 2: band.m0c + nx // 2 + band.bc].to(dev)
    Xd, Yd, Vd = X.to(dev), Y.to(dev), V.to(dev)
    fz = torch.tensor(zs, dtype=torch.float64, device=dev)
    states = _pol_states(source, X, Y, vector, dev)
    sets = []
    for st in states:   # one field set per incoherent polarisation state, [Z, S*E] each
        pupils = torch.empty((len(zs), nsrc * ne, band.br, band.bc), dtype=torch.complex64, device=dev)
        weights = torch.empty((len(zs), nsrc * ne), dtype=torch.float32, device=dev)
        args = (N.ptr(fr), N.ptr(fc), band.br, band.bc, N.ptr(Xd), N.ptr(Yd), N.ptr(Vd), nsrc, float(torch.sum(V)),
                N.ptr(fz), len(zs), _zernike(projector), int(vector))
        tail = (float(projector.NA), float(projector.Magnification), float(projector.IndexImage),
                float(source.Wavelength), N.ptr(pupils), N.ptr(weights), N.stream_handle(dev))
        if st is None:
            N.call('oi_abbe_pupils', *args, _jones(source), *tail)
        else:
            N.call('oi_abbe_pupils_pol', *args, N.ptr(st), *tail)
        sets.append((pupils, weights))
    if len(sets) == 1:
        pupils, weights = sets[0]
    else:
        pupils = torch.cat([p for p, _ in sets], dim=1)
        weights = torch.cat([w for _, w in sets], dim=1)
    model = CoherentModel(pupils, weights, band, ny, nx, kind='abbe', pack=pack)
    model.pol_states = len(sets)
    return model


def _pol_states(source, X, Y, vector, dev):
    """The polarisation states of a vector image as device Jones arrays [S, 4] float64 (Px.re, Px.im, Py.re,
    Py.im per point), or [None] for the source's constant PolarizationVector.  Scalar images carry no
    polarisation (as in the reference): one state."""
    states = source.polarization_states(X, Y) if vector and hasattr(source, 'polarization_states') else None
    if states is None:
        return [None]
    return [torch.view_as_real(st.to(torch.complex128)).reshape(-1, 4).contiguous().to(dev) for st in states]


def _field_image(model, h):
    """model.image of one field: h float32 [Ny, Nx] (one real channel, the real-mask band pass) or complex64
    [Ny, Nx, C]."""
    if h.dim() == 2:
        return model.image(h.unsqueeze(0), kind=N.FIELD_REAL_F32)[0]
    return model.image(h.unsqueeze(0), kind=N.FIELD_COMPLEX_C64, nch=h.shape[2])[0]


def abbe_intensity(source, scatter, projector, numerics, h=None):
    """Abbe image [nFocus, Ny, Nx] float32 on the device (CalculateAerialImage.py:18-92).  h: the field on the
    device, complex64 [Ny, Nx, C] or, for one real channel, float32 [Ny, Nx]."""
    dev = require_cuda()
    if h is None:
        h = _field_on_device(scatter, dev)
    ny, nx = h.shape[0], h.shape[1]
    zs = _focus_list(projector)
    sd = source.Calc_SourceSimple()
    if sd.Value.numel() == 0:   # the reference divides 0 by a zero source weight
        _mode(numerics)
        return torch.full((len(zs), ny, nx), float('nan'), device=dev)
    model = abbe_model(source, projector, numerics, scatter.Period_Y, scatter.Period_X, ny, nx, pack=False)
    if model is None:
        return torch.zeros((len(zs), ny, nx), device=dev)
    return _field_image(model, h)


def CalculateAbbeImage(source, scatter, projector, numerics):
    """Abbe aerial image -> (ImageData, pupilImage) (CalculateAerialImage.py:18-103)."""
    dev = require_cuda()
    fld = _DropInField(scatter, dev)
    inten = abbe_intensity(source, scatter, projector, numerics, h=fld.carrier())
    pim = fld.pupil_image(scatter, projector, source, dev)
    rd = _result_device(scatter)
    inten, pim = _to_host(inten, rd), _to_host(pim, rd)
    _check('CalculateAbbeImage')
    return _image_data(inten, scatter, projector), pim


# ------------------------------------------------------------------------------------------------ TCC
def _tcc_axes(source, xypitch, projector):
    """TCC grid axes exactly as CalculateTCCMatrix.py:17-22 (float32 tensors)."""
    npf = torch.tensor(xypitch[0] / (source.Wavelength / projector.NA))
    npg = torch.tensor(xypitch[1] / (source.Wavelength / projector.NA))
    nf = int(torch.ceil(2 * npf).int())
    ng = int(torch.ceil(2 * npg).int())
    f = (1 / npf) * torch.arange(-nf, nf + 1)
    g = (1 / npg) * torch.arange(-ng, ng + 1)
    return f, g


def tcc_pupil_matrix(source, xypitch, projector, focus, numerics):
    """h [ne, FG, S] complex128 with TCC = sum_e h_e h_e^H, and FG_ValidSize [len g, len f].  With several
    polarisation states (a CoherencyMatrix) their component sets are stacked: ne = 3 x states."""
    vector = _mode(numerics)
    _check_domain(projector)
    dev = require_cuda()
    sd = source.Calc_SourceSimple()
    X, Y, V = (t.reshape(-1).to(torch.float32) for t in (sd.X, sd.Y, sd.Value))
    f, g = _tcc_axes(source, xypitch, projector)
    ne = 3 if vector else 1
    nsrc = X.numel()
    if nsrc == 0:
        h = torch.full((ne, f.numel() * g.numel(), 1), float('nan'), dtype=torch.complex128, device=dev)
        return h, [g.numel(), f.numel()]
    fd, gd, Xd, Yd, Vd = (t.to(dev) for t in (f, g, X, Y, V))   # held until the launch is enqueued
    hs = []
    for st in _pol_states(source, X, Y, vector, dev):   # TCC = sum over states and components of h h^H
        h = torch.empty((ne, f.numel() * g.numel(), nsrc), dtype=torch.complex128, device=dev)
        args = (N.ptr(fd), f.numel(), N.ptr(gd), g.numel(), N.ptr(Xd), N.ptr(Yd), N.ptr(Vd), nsrc,
                float(torch.sum(V)), float(focus), _zernike(projector), int(vector))
        tail = (float(projector.NA), float(projector.Magnification), float(projector.IndexImage),
                float(source.Wavelength), N.ptr(h), N.stream_handle(dev))
        if st is None:
            N.call('oi_tcc_pupils64', *args, _jones(source), *tail)
        else:
            N.call('oi_tcc_pupils64_pol', *args, N.ptr(st), *tail)
        hs.append(h)
    return (hs[0] if len(hs) == 1 else torch.cat(hs, dim=0)), [g.numel(), f.numel()]


def CalculateTCCMatrix(source, xypitch, projector, focus, numerics):
    """TCC [FG, FG] complex128 on the device and FG_ValidSize [len g, len f] (CalculateTCCMatrix.py:9-56)."""
    h, fg = tcc_pupil_matrix(source, xypitch, projector, focus, numerics)
    n = h.shape[1]
    tcc = torch.empty((n, n), dtype=torch.complex128, device=h.device)
    N.call('oi_tcc_assemble64', N.ptr(h), h.shape[0], n, h.shape[2], N.ptr(tcc), N.stream_handle(h.device))
    return tcc, fg


def GetTCCMatrix(sourceData, shiftedPupil):
    """P diag(w) P^H / sum(w) for a [FG, S] pupil matrix (CalculateTCCMatrix.py:58-75), FP64 on the device."""
    dev = require_cuda()
    w = sourceData.Value.reshape(-1).to(torch.float64)
    p = torch.as_tensor(shiftedPupil).to(dev, torch.complex128)
    h = (p * torch.sqrt(w.to(dev) / torch.sum(w).to(dev))).contiguous().unsqueeze(0)
    n = h.shape[1]
    tcc = torch.empty((n, n), dtype=torch.complex128, device=dev)
    N.call('oi_tcc_assemble64', N.ptr(h), 1, n, h.shape[2], N.ptr(tcc), N.stream_handle(dev))
    return tcc


def _socs_count(numerics, evals, size):
    kind = numerics.Hopkins_SettingType.lower()
    if kind == 'order':
        return min(numerics.Hopkins_Order, size - 1)
    if kind == 'threshold':
        c = torch.cumsum(evals, 0)
        k = int(torch.searchsorted(c, numerics.Hopkins_Threshold * c[-1], right=True))
        return min(k, size - 1)
    raise ValueError('Error: Hopkins_SettingType should be order or threshold!')


def _eig_desc(tcc):
    """Every eigenpair of the Hermitian TCC, eigenvalues descending and clamped at zero (FP64, on the device;
    the library's dense solver, for decompositions that keep more kernels than eig_topk covers)."""
    lam, U = torch.linalg.eigh(tcc)
    return torch.clamp(lam.flip(0), min=0), U.flip(1)


TOPK_MAX = 48          # kernels the hand-written solver keeps (its block holds 64 vectors)


def eig_topk(k: int, tcc: torch.Tensor | None = None, h: torch.Tensor | None = None, tol: float = 1e-13,
             max_iter: int = 300):
    """The k leading eigenpairs (eigenvalues descending, clamped at zero; eigenvectors [n, k]) of the Hermitian
    TCC, given densely (`tcc` [n, n] complex128) or as its pupil factor (`h` [ne, n, s] complex128 with
    TCC = sum_e h_e h_e^H, never formed), by the library's FP64 block subspace iteration (oi_eig_topk64):
    Rayleigh-Ritz residuals below tol x the largest eigenvalue.  Returns None when k is out of its range
    (k > TOPK_MAX or a TCC of fewer than 64 rows)."""
    A = tcc if tcc is not None else h
    n = A.shape[0] if tcc is not None else A.shape[1]
    p = 64
    if k > TOPK_MAX or k <= 0 or n < p:
        return None
    dev = A.device
    ne, s_ = (0, 0) if tcc is not None else (A.shape[0], A.shape[2])
    nbytes = ctypes.c_longlong(0)
    N.call('oi_eig_topk64_workspace', n, p, ne, s_, ctypes.byref(nbytes))
    work = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    vecs = torch.empty((n, k), dtype=torch.complex128, device=dev)
    vals = torch.empty(k, dtype=torch.float64, device=dev)
    iters = ctypes.c_int(0)
    A = A.to(torch.complex128).contiguous()
    N.call('oi_eig_topk64', N.ptr(A) if tcc is not None else None, N.ptr(A) if tcc is None else None, ne, n, s_,
           k, p, max_iter, float(tol), N.ptr(vecs), N.ptr(vals), N.ptr(work), nbytes.value, ctypes.byref(iters),
           N.stream_handle(dev))
    if iters.value < 0:
        warnings.warn(f'oi_eig_topk64 did not reach tol={tol} in {max_iter} iterations; using the dense solver',
                      RuntimeWarning, stacklevel=2)
        return None
    return vals, vecs


def _placement(n, length):
    """Frequency of the first kernel row/column as DecomposeTCC_SOCS places it: centred embedding at
    (n - length + 1)//2 then fftshift (DecomposeTCC_SOCS.py:29-31).  For odd n this lands one frequency
    below the centre, and the engine keeps that placement so its images match the reference's."""
    return (n - length + 1) // 2 + n // 2 - n


def socs_kernels_from_tcc(tcc, FG_ValidSize, Nfg, numerics) -> SocsKernels:
    """Top-K SOCS kernels sqrt(lambda_k) u_k in band form, placed as the reference places them."""
    nf, ng = Nfg
    lg, lf = FG_ValidSize
    if lf > ng or lg > nf:
        raise ValueError(f'TCC grid {lf}x{lg} does not fit the {ng}x{nf} image grid')
    top = None
    if numerics.Hopkins_SettingType.lower() == 'order':
        top = eig_topk(min(numerics.Hopkins_Order, tcc.shape[0] - 1), tcc=tcc)
    if top is not None:
        lam, U = top
        k = lam.numel()
    else:
        lam, U = _eig_desc(tcc)
        k = _socs_count(numerics, lam, U.shape[1])
    kb = (U[:, :k] * torch.sqrt(lam[:k])).T.reshape(k, lf, lg)
    band = Band(_placement(ng, lf), lf, _placement(nf, lg), lg)
    return SocsKernels(kb.to(torch.complex64), band, ng, nf)


def socs_kernels_from_pupils(h, FG_ValidSize, Nfg, numerics) -> SocsKernels:
    """Top-K SOCS kernels from the pupil matrix h [ne, FG, S] of TCC = sum_e h_e h_e^H, without forming the TCC
    when its rank bound ne*S is below FG: with H = [h_0 | .. | h_ne-1] (FG x ne*S), the Gram matrix H^H H has the
    TCC's non-zero eigenvalues, and its eigenvectors v give the kernels sqrt(lambda) u = H v (FP64 on the device).
    Kernels equal socs_kernels_from_tcc's up to a phase per kernel (images are unchanged)."""
    ne, fg, s = h.shape
    if ne * s >= fg:
        tcc = torch.empty((fg, fg), dtype=torch.complex128, device=h.device)
        N.call('oi_tcc_assemble64', N.ptr(h), ne, fg, s, N.ptr(tcc), N.stream_handle(h.device))
        return socs_kernels_from_tcc(tcc, FG_ValidSize, Nfg, numerics)
    nf, ng = Nfg
    lg, lf = FG_ValidSize
    if lf > ng or lg > nf:
        raise ValueError(f'TCC grid {lf}x{lg} does not fit the {ng}x{nf} image grid')
    top = None
    if numerics.Hopkins_SettingType.lower() == 'order':   # leading kernels of h h^H, the TCC never formed
        top = eig_topk(min(numerics.Hopkins_Order, fg - 1, ne * s), h=h)
    if top is not None:
        lam, U = top
        k = lam.numel()
        kb = (U * torch.sqrt(lam)).T.reshape(k, lf, lg)
        band = Band(_placement(ng, lf), lf, _placement(nf, lg), lg)
        return SocsKernels(kb.to(torch.complex64).contiguous(), band, ng, nf)
    H = h.permute(1, 0, 2).reshape(fg, ne * s)
    lam, V = torch.linalg.eigh(H.conj().T @ H)
    lam, V = torch.clamp(lam.flip(0), min=0), V.flip(1)
    k = min(_socs_count(numerics, lam, fg), V.shape[1])   # kernels past the rank bound are zero
    kb = (H @ V[:, :k]).T.reshape(k, lf, lg)
    band = Band(_placement(ng, lf), lf, _placement(nf, lg), lg)
    return SocsKernels(kb.to(torch.complex64).contiguous(), band, ng, nf)


def DecomposeTCC_SOCS(TCCMatrix_Stacked, FG_ValidSize, Nfg, numerics):
    """Full-grid SOCS kernels [Ny, Nx, K] complex64 on the device (DecomposeTCC_SOCS.py:3-37)."""
    dev = require_cuda()
    tcc = torch.as_tensor(TCCMatrix_Stacked).to(dev, torch.complex128)
    sk = socs_kernels_from_tcc(tcc, FG_ValidSize, Nfg, numerics)
    nf, ng = Nfg
    full = torch.zeros((ng, nf, sk.count), dtype=torch.complex64, device=dev)
    b = sk.band
    full[:b.br, :b.bc, :] = sk.kernels.permute(1, 2, 0)
    full = torch.roll(full, shifts=(b.m0r, b.m0c), dims=(0, 1))
    _SOCS_CACHE[full] = (full._version, sk)    # CalculateAerialImage_SOCS reuses the band form
    return full


def CalculateAerialImage_SOCS(scatter, TCCMatrix_SOCS, source, projector):
    """SOCS aerial image [Ny, Nx] and pupilImage (CalculateAerialImage_SOCS.py:3-11)."""
    dev = require_cuda()
    sk = _socs_kernels_of(TCCMatrix_SOCS, dev)
    fld = _DropInField(scatter, dev)
    if fld.real is not None:
        # one real channel (a thin mask, the usual ScatterField): the model's real-mask path
        img = sk.image(fld.real.unsqueeze(0), kind=N.FIELD_REAL_F32)[0]
    else:
        h = fld.live_complex()
        img = sk.image(h.unsqueeze(0), kind=N.FIELD_COMPLEX_C64, nch=h.shape[2])[0]
    pim = fld.pupil_image(scatter, projector, source, dev)
    rd = _result_device(scatter)
    img, pim = _to_host(img, rd), _to_host(pim, rd)
    _check('CalculateAerialImage_SOCS')
    return img, pim


def socs_model(source, projector, numerics, period_y, period_x, ny, nx, focus=None, pack=True) -> CoherentModel:
    """SOCS kernels of every focus plane resident on the device: per plane TCC -> FP64 top-K eigenpairs ->
    kernels placed as the reference places them (CalculateAerialImage.py:112-119).  image() gives the Hopkins
    image of a batch of masks, all planes in one pass."""
    zs = _focus_list(projector) if focus is None else [float(z) for z in focus]
    sets = []
    for z in zs:
        h, fg = tcc_pupil_matrix(source, [period_y, period_x], projector, z, numerics)
        sets.append(socs_kernels_from_pupils(h, fg, [nx, ny], numerics))
    k = max(s.count for s in sets)   # 'threshold' may keep a different count per plane: pad with zero kernels
    pupils = torch.zeros((len(zs), k, sets[0].band.br, sets[0].band.bc), dtype=torch.complex64,
                         device=sets[0].kernels.device)
    for i, s in enumerate(sets):
        pupils[i, :s.count] = s.kernels
    return CoherentModel(pupils, torch.ones((len(zs), k), device=pupils.device), sets[0].band, ny, nx, 'socs',
                         pack=pack)


def hopkins_intensity(source, scatter, projector, numerics, h=None):
    """Hopkins image [nFocus, Ny, Nx] on the device: per plane TCC -> top-K kernels -> SOCS image.  h as for
    abbe_intensity."""
    dev = require_cuda()
    if h is None:
        h = _field_on_device(scatter, dev)
    ny, nx = h.shape[0], h.shape[1]
    model = socs_model(source, projector, numerics, scatter.Period_Y, scatter.Period_X, ny, nx, pack=False)
    return _field_image(model, h)


def CalculateHopkinsImage(source, scatter, projector, numerics):
    """Hopkins aerial image -> (ImageData, pupilImage) (CalculateAerialImage.py:105-130)."""
    dev = require_cuda()
    fld = _DropInField(scatter, dev)
    inten = hopkins_intensity(source, scatter, projector, numerics, h=fld.carrier())
    pim = fld.pupil_image(scatter, projector, source, dev)
    rd = _result_device(scatter)
    inten, pim = _to_host(inten, rd), _to_host(pim, rd)
    _check('CalculateHopkinsImage')
    return _image_data(inten, scatter, projector), pim


# ------------------------------------------------------------------------------ Floquet-mode ("optimized")
def CalculateSOCS(FloquetMode, TCCMatrix_SOCS, numerics):
    """Direct-DFT SOCS image [ScatterGrid_X, ScatterGrid_Y] from Floquet modes (CalculateAerialImage_SOCS.py:13-32).

    I[x][y] = sum_{k,c} |sum_o exp(2 pi i (ox (x+1/2)/Gx + oy (y+1/2)/Gy)) FM[o, c] kern_k[o]|^2 over the
    (2 ScatterOrder_X + 1) x (2 ScatterOrder_Y + 1) orders o, with kern_k = ifftshift(transpose(kernels)) paired
    with FM by flat index exactly as the reference reshapes them.  The engine's coherent-sum stages evaluate it:
    each (k, c) is one field on the order band; the half-pixel offset is a phase per order, and the positive
    exponent is the engine's negative one applied to the order-reversed field.
    """
    dev = require_cuda()
    fm = torch.as_tensor(FloquetMode).to(dev, torch.complex64)
    ker = torch.as_tensor(TCCMatrix_SOCS).to(dev, torch.complex64)
    gx, gy = numerics.ScatterGrid_X, numerics.ScatterGrid_Y
    ox, oy = numerics.ScatterOrder_X, numerics.ScatterOrder_Y
    nox, noy = 2 * ox + 1, 2 * oy + 1
    kt = torch.fft.ifftshift(ker.transpose(0, 1), dim=(0, 1))
    if tuple(fm.shape) != (nox, noy, 3) or tuple(kt.shape[:2]) != (nox, noy):
        raise ValueError(f'FloquetMode {tuple(fm.shape)} / kernels {tuple(ker.shape)} do not match the '
                         f'{nox}x{noy} scatter orders')
    k = kt.shape[2]
    qx = torch.arange(-ox, ox + 1, device=dev, dtype=torch.float64)
    qy = torch.arange(-oy, oy + 1, device=dev, dtype=torch.float64)
    half = torch.exp(1j * torch.pi * (qx[:, None] / gx + qy[None, :] / gy)).to(torch.complex64)
    a = fm.permute(2, 0, 1)[None] * kt.permute(2, 0, 1)[:, None] * half    # [K, 3, nox, noy]
    fields = torch.flip(a, dims=(2, 3)).reshape(1, k * 3, nox, noy).contiguous()
    plan = Plan.get(gx, gy, Band(-ox, nox, -oy, noy), dev)
    ones = torch.ones((1, 1, nox, noy), dtype=torch.complex64, device=dev)
    w = torch.ones((1, 1), dtype=torch.float32, device=dev)
    img = coherent_image(fields, ones, w, plan)[0, 0]
    _check('CalculateSOCS')
    return img.to(_tensor_device(FloquetMode))


def _tensor_device(t):
    return t.device if isinstance(t, torch.Tensor) else torch.device('cpu')


def CalculateOptimized(source, scatter, projector, numerics):
    """Floquet-mode SOCS image -> (ImageData, empty tensor) (CalculateAerialImage.py:131-152)."""
    pitchxy = [scatter.Period_Y, scatter.Period_X]
    fm = scatter.FloquetMode
    nfg = [fm.shape[0], fm.shape[1]]
    zs = projector.FocusRange
    out = torch.zeros(len(_focus_list(projector)), numerics.ScatterGrid_X, numerics.ScatterGrid_Y)
    for i, z in enumerate(_focus_list(projector)):
        tcc, fg = CalculateTCCMatrix(source, pitchxy, projector, z, numerics)
        ker = DecomposeTCC_SOCS(tcc, fg, nfg, numerics)
        out[i] = CalculateSOCS(fm, ker, numerics).cpu()
    img = ImageData()
    img.Intensity = out
    img.ImageX = torch.linspace(-scatter.Period_X / 2, scatter.Period_X / 2, numerics.ScatterGrid_X)
    img.ImageY = torch.linspace(-scatter.Period_Y / 2, scatter.Period_Y / 2, numerics.ScatterGrid_Y)
    img.ImageZ = zs
    return img, torch.tensor([])


def CalculateCharacteristicMatrix(f_calc, g_calc, NA, indexImage):
    """Polarisation transfer terms (CalculateCharacteristicMatrix.py:3-17), torch complex on the input's device.

    The engine evaluates this inside its pupil kernels; this host form is the reference's public helper.
    """
    alpha = torch.complex((NA / indexImage) * f_calc, torch.zeros_like(f_calc))
    beta = torch.complex((NA / indexImage) * g_calc, torch.zeros_like(g_calc))
    gamma = torch.sqrt(1 - alpha ** 2 - beta ** 2)
    mxx = 1 - alpha ** 2 / (1 + gamma)
    myx = -alpha * beta / (1 + gamma)
    myy = 1 - beta ** 2 / (1 + gamma)
    return mxx, myx, myx, myy, -alpha, -beta
