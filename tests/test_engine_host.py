"""Host-side logic of the engine (no GPU): band selection, kernel support, field split, coarse sizes."""
import math

import numpy as np
import torch

from opticalimaging_b200 import engine as E
from opticalimaging_b200 import imaging as I


def test_plan_api_shape():
    assert callable(E.Plan.get) and callable(E.Plan.use_fft) and callable(E.Plan.use_coarse_fft)


def test_coarse_size_holds_intensity_band():
    for b in (1, 17, 31, 32, 33, 59, 64, 65, 117, 128):
        m = E.coarse_size(b)
        assert m % 64 == 0 and m >= 2 * b - 1 and m - 64 < max(2 * b - 1, 64)
    assert E.coarse_size(59) == 128 and E.coarse_size(31) == 64 and E.coarse_size(117) == 256


def test_field_split_divides_and_fills():
    assert E.field_split(24, 64, sms=148) == 8   # 64 images x 8 splits >= 3 waves of 148 SMs
    assert E.field_split(24, 1, sms=148) == 24
    assert E.field_split(324, 5, sms=148) == 108
    assert E.field_split(24, 64, sms=132) == 8 and E.field_split(24, 32, sms=132) == 24
    for n, b in ((24, 64), (7, 3), (324, 5), (1, 1)):
        d = E.field_split(n, b)
        assert n % d == 0


def test_cyclic_support_and_centring():
    z = torch.zeros(16, dtype=torch.bool)
    z[[14, 15, 0, 1, 2]] = True
    assert E.cyclic_support(z) == (14, 5)
    assert E.centred(14, 16) == -2 and E.centred(3, 16) == 3 and E.centred(8, 16) == -8
    z = torch.zeros(9, dtype=torch.bool)
    z[[3]] = True
    assert E.cyclic_support(z) == (3, 1)
    assert E.cyclic_support(torch.ones(5, dtype=torch.bool)) == (0, 5)


def test_reference_kernel_placement():
    # centred embedding then fftshift (DecomposeTCC_SOCS.py:29-31): even grids centre the band on 0,
    # odd grids place it one frequency low
    assert I._placement(1024, 59) == -29
    assert I._placement(45, 15) == -8
    assert I._placement(63, 19) == -10
    assert I._placement(40, 13) == -6


def test_abbe_band_covers_every_shifted_pupil():
    sx = torch.tensor([-0.9, 0.3, 0.9])
    sy = torch.tensor([0.0, -0.9, 0.5])
    npy, npx = 7.16, 7.16
    b = E.abbe_band(256, 256, npy, npx, sx, sy)
    # every frequency with (m/np + s)^2 <= 1 for some point lies in the band
    for x, y in zip(sx.tolist(), sy.tolist()):
        lo_r, hi_r = math.ceil(npy * (-1 - x)), math.floor(npy * (1 - x))
        lo_c, hi_c = math.ceil(npx * (-1 - y)), math.floor(npx * (1 - y))
        assert b.m0r <= lo_r and hi_r <= b.m0r + b.br - 1
        assert b.m0c <= lo_c and hi_c <= b.m0c + b.bc - 1
    # clipped to the grid's frequencies
    b = E.abbe_band(16, 16, 20.0, 20.0, sx, sy)
    assert b.m0r >= -8 and b.m0r + b.br - 1 <= 7


def test_require_cuda_resolves_a_bare_cuda_device(monkeypatch):
    """'cuda' without an index means the current device (a scheduler thread calls torch.cuda.set_device with
    it, which needs an index); no GPU needed: CUDA availability is faked."""
    import torch
    from opticalimaging_b200 import engine as E, _native as N
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: True)
    monkeypatch.setattr(torch.cuda, 'current_device', lambda: 3)
    monkeypatch.setattr(N, 'load', lambda *a, **k: None)
    assert E.require_cuda(torch.device('cuda')) == torch.device('cuda', 3)
    assert E.require_cuda('cuda') == torch.device('cuda', 3)
    assert E.require_cuda(None) == torch.device('cuda', 3)
    assert E.require_cuda('cuda:1') == torch.device('cuda', 1)


def test_field_split_sm_minimises_waves_times_fields():
    """The field split of the one-block-per-SM coherent kernel (256 x 256 coarse grid): the d in [1, nfields]
    minimising ceil(blocks d / SMs) * (ceil(nfields / d) + 1/2), the smallest d on ties."""
    from opticalimaging_b200.engine import field_split_sm
    SMS = 148

    def cost(nf, b, d):
        return -(-b * d // SMS) * (-(-nf // d) + 0.5)

    assert field_split_sm(324, 8, SMS) == 18   # vector Abbe 2048^2 at batch 8: 144 blocks of 18 fields, one wave
    assert field_split_sm(24, 8, SMS) == 12    # SOCS-24: 96 blocks of 2 fields (18 ties, more partial sums)
    assert field_split_sm(1, 1, SMS) == 1
    for nf in (1, 5, 24, 72, 324):
        for b in (1, 2, 8, 64, 200):
            d = field_split_sm(nf, b, SMS)
            assert 1 <= d <= nf
            best = min(cost(nf, b, e) for e in range(1, nf + 1))
            assert cost(nf, b, d) == best
            assert all(cost(nf, b, e) > best for e in range(1, d))


def test_sm_count_without_a_device_is_the_b200s():
    if not torch.cuda.is_available():
        assert E.sm_count() == E.B200_SMS == 148


def test_plan_cache_is_bounded_lru(monkeypatch):
    made = []

    class FakePlan(E.Plan):
        def __init__(self, ny, nx, band, device, coarse=None):   # no device work: record the key only
            made.append((ny, nx))

    monkeypatch.setattr(E.Plan, '_cache', E.collections.OrderedDict())
    monkeypatch.setattr(E.Plan, 'CACHE_SIZE', 4)
    band = E.Band(-2, 5, -2, 5)
    first = FakePlan.get(8, 8, band, 'cpu')
    for n in range(9, 14):
        FakePlan.get(n, n, band, 'cpu')
        FakePlan.get(8, 8, band, 'cpu')             # kept in use: stays cached
    assert len(E.Plan._cache) == 4
    assert FakePlan.get(8, 8, band, 'cpu') is first
    FakePlan.get(9, 9, band, 'cpu')                 # evicted earlier: built again
    assert made.count((9, 9)) == 2 and made.count((8, 8)) == 1


def _coherent_sum_fp64(pupils, weights, band, mask):
    """sum_k w_k |IDFT(P_k .* c)|^2 on the mask's grid in FP64, c the band of the mask's DFT (numpy)."""
    ny, nx = mask.shape
    spec = np.fft.fft2(mask) / (ny * nx)
    rows = (band.m0r + np.arange(band.br)) % ny
    cols = (band.m0c + np.arange(band.bc)) % nx
    c = spec[np.ix_(rows, cols)]
    out = np.zeros((pupils.shape[0], ny, nx))
    for z in range(pupils.shape[0]):
        for k in range(pupils.shape[1]):
            full = np.zeros((ny, nx), dtype=np.complex128)
            full[np.ix_(rows, cols)] = pupils[z, k] * c
            out[z] += weights[z, k] * np.abs(np.fft.ifft2(full) * ny * nx) ** 2
    return out


def test_packed_real_fields_give_the_same_images():
    """For a real mask, kernels that are Hermitian up to a phase pack two to a transform and generic complex
    kernels split into two real fields each; the packed set gives the same sum of |IDFT|^2 in FP64."""
    import torch
    from opticalimaging_b200.engine import Band, pack_real_fields
    rng = np.random.default_rng(5)
    band = Band(-7, 15, -5, 11)
    herm = []
    for _ in range(6):                 # Hermitian kernels times a random phase
        h = rng.normal(size=(15, 11)) + 1j * rng.normal(size=(15, 11))
        h = (h + np.conj(h[::-1, ::-1])) / 2
        herm.append(h * np.exp(1j * rng.uniform(0, 2 * np.pi)))
    generic = [rng.normal(size=(15, 11)) + 1j * rng.normal(size=(15, 11)) for _ in range(3)]
    P = np.stack(herm + generic)[None]
    w = rng.uniform(0.2, 2.0, size=(1, 9))
    packed = pack_real_fields(torch.from_numpy(P), torch.from_numpy(w), band)
    assert packed is not None
    Q, wq = packed
    assert Q.shape == (1, 6, 15, 11)           # J = 6 + 2 * 3 = 12 real fields -> 6 transforms instead of 9
    assert torch.equal(wq, torch.ones((1, 6)))
    for seed in range(3):
        mask = (np.random.default_rng(seed).uniform(size=(40, 36)) > 0.6).astype(np.float64)
        a = _coherent_sum_fp64(P, w, band, mask)
        b = _coherent_sum_fp64(Q.numpy().astype(np.complex128), wq.numpy(), band, mask)
        assert np.max(np.abs(a - b)) / np.max(a) < 1e-6     # the packed set is stored as complex64


def test_packing_declines_what_it_cannot_use():
    """No packing for an off-centre band, a negative weight, or fields that gain nothing (all generic)."""
    import torch
    from opticalimaging_b200.engine import Band, pack_real_fields
    rng = np.random.default_rng(6)
    P = torch.from_numpy(rng.normal(size=(1, 4, 9, 9)) + 1j * rng.normal(size=(1, 4, 9, 9)))
    w = torch.ones((1, 4), dtype=torch.float64)
    assert pack_real_fields(P, w, Band(-3, 9, -4, 9)) is None          # not centred on frequency 0
    assert pack_real_fields(P, w, Band(-4, 9, -4, 9)) is None          # 8 real fields: 4 transforms again
    h = (P + torch.flip(P, dims=(-2, -1)).conj()) / 2
    assert pack_real_fields(h, w, Band(-4, 9, -4, 9)) is not None
    assert pack_real_fields(h, -w, Band(-4, 9, -4, 9)) is None


def test_packing_sees_through_degenerate_mixtures():
    """Kernels that are unitary mixtures of Hermitian ones ((A + iB) / sqrt 2, (A - iB) / sqrt 2: what an
    eigensolver may return for a degenerate pair) span two real dimensions: two kernels, one transform."""
    import torch
    from opticalimaging_b200.engine import Band, pack_real_fields
    rng = np.random.default_rng(8)
    band = Band(-6, 13, -6, 13)
    herm = []
    for _ in range(4):
        a = rng.normal(size=(13, 13)) + 1j * rng.normal(size=(13, 13))
        herm.append((a + np.conj(a[::-1, ::-1])) / 2)
    mix = [(herm[0] + 1j * herm[1]) / np.sqrt(2), (herm[0] - 1j * herm[1]) / np.sqrt(2),
           (herm[2] + 1j * herm[3]) * np.exp(0.7j) / np.sqrt(2), (herm[2] - 1j * herm[3]) * np.exp(-1.1j) / np.sqrt(2)]
    P = np.stack(mix)[None]
    w = np.ones((1, 4))
    Q, wq = pack_real_fields(torch.from_numpy(P), torch.from_numpy(w), band)
    assert Q.shape == (1, 2, 13, 13)
    mask = (np.random.default_rng(1).uniform(size=(30, 34)) > 0.5).astype(np.float64)
    a = _coherent_sum_fp64(P, w, band, mask)
    b = _coherent_sum_fp64(Q.numpy().astype(np.complex128), wq.numpy(), band, mask)
    assert np.max(np.abs(a - b)) / np.max(a) < 1e-6


def _field(f):
    from opticalimaging_b200.params import Scatter
    sc = Scatter()
    sc.ScatterField = torch.from_numpy(f)
    return sc


def test_drop_in_field_classifies_channels():
    """The drop-in's one reduction (run here on a small host field) finds the live channels and whether the field
    is one real channel: -0 counts as zero, NaN as non-zero, an all-zero field keeps channel 0."""
    dev = torch.device('cpu')
    rng = np.random.default_rng(3)
    m = (rng.random((12, 10)) > 0.5).astype(np.float32)
    f = np.zeros((12, 10, 3), np.complex64)
    f[:, :, 0] = m
    d = I._DropInField(_field(f), dev)
    assert d.live == [0] and d.real is not None
    np.testing.assert_array_equal(d.real.numpy(), m)
    assert d.live_complex().shape == (12, 10, 1)

    g = f.copy()
    g.imag[:, :, 0] = np.float32(-0.0)                    # negative zero imaginary parts: still one real channel
    d = I._DropInField(_field(g), dev)
    assert d.real is not None and d.live == [0]

    g = f.copy()
    g[3, 4, 2] = 0.5j                                     # a second, complex channel
    d = I._DropInField(_field(g), dev)
    assert d.real is None and d.live == [0, 2]
    np.testing.assert_array_equal(d.live_complex().numpy(), g[:, :, [0, 2]])

    g = f.copy()
    g[0, 0, 1] = np.nan                                   # NaN is non-zero
    d = I._DropInField(_field(g), dev)
    assert d.real is None and d.live == [0, 1]

    g = f.copy()
    g[5, 5, 0] += 1e-30j                                  # one imaginary part makes channel 0 complex
    d = I._DropInField(_field(g), dev)
    assert d.real is None and d.live == [0]

    d = I._DropInField(_field(np.zeros((12, 10, 3), np.complex64)), dev)
    assert d.live == [0] and d.real is not None and not d.real.any()

    d = I._DropInField(_field(np.zeros((12, 10, 3), np.complex64)[:, :, :2].copy()), dev)
    assert d.nch == 2 and d.live == [0]
    import pytest
    with pytest.raises(ValueError):
        I._DropInField(_field(np.zeros((12, 10), np.complex64)), dev)
