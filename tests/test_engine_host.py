"""Host-side logic of the engine (no GPU): band selection, kernel support, field split, coarse sizes."""
import math

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
