"""Split-BF16x3 coherent contraction on the tensor cores (oi_coherent_coarse_tc) against the FP64 oracle, the
reference's own outputs and the FP32 forms.

Stated bound of the split form: 1e-4 of the peak of the FP64 image (each real operand carries ~16 significant
bits as bf16 hi + lo; products hi*hi + hi*lo + lo*hi in FP32).  Every case also reports max and RMS error.
"""
import numpy as np
import pytest
import torch

from oracle import optics64 as O
from tests.fixtures import build, load, rel_err

pytestmark = pytest.mark.gpu

BF16X3_VS_FP64 = 1e-4


def rms_rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.max(np.abs(b)))


@pytest.fixture(scope='module')
def oi():
    import opticalimaging_b200.imaging as imaging
    from opticalimaging_b200 import _native
    _native.load()
    _native.device_status(reset=True)
    return imaging


def test_tc_layout_and_range_errors(oi):
    from opticalimaging_b200 import _native as N
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert N.tc_layout(64, 24) == (sms, N.tc_layout(64, 24)[1])
    assert N.tc_layout(2, 3) == (6, 3)                     # fewer tasks than SMs: one task per CTA
    dev = torch.device('cuda')
    band = torch.zeros((1, 1, 8, 8), dtype=torch.complex64, device=dev)
    pup = torch.zeros((1, 4, 8, 8), dtype=torch.complex64, device=dev)
    w = torch.ones((1, 4), device=dev)
    consts = torch.zeros(98304, dtype=torch.uint8, device=dev)
    coarse = torch.zeros((4, 1, 1, 128, 128), device=dev)
    s = N.stream_handle(dev)
    with pytest.raises(N.NativeError, match='partial slots'):
        N.call('oi_coherent_coarse_tc', N.ptr(band), 1, 1, -4, 8, -4, 8, N.ptr(pup), 0, N.ptr(w), 1, 4,
               N.ptr(consts), 4, 3, N.ptr(coarse), s)
    big = torch.zeros((1, 1, 65, 8), dtype=torch.complex64, device=dev)
    with pytest.raises(N.NativeError, match='exceeds 64x64'):
        N.call('oi_coherent_coarse_tc', N.ptr(big), 1, 1, -32, 65, -4, 8, N.ptr(pup), 0, N.ptr(w), 1, 4,
               N.ptr(consts), 4, 4, N.ptr(coarse), s)
    tw = torch.zeros(128, dtype=torch.complex64, device=dev)
    with pytest.raises(N.NativeError, match='bytes given'):
        N.call('oi_tc_constants', -4, -3, N.ptr(tw), N.ptr(tw), N.ptr(consts), 98304, s)


@pytest.mark.parametrize('name', ['cfg1', 'vec_small', 'odd_scalar'])
def test_abbe_bf16x3_vs_fp64(oi, name):
    from opticalimaging_b200 import _native as N
    meta, a = load(name)
    sr, sc, po, nm = build(meta, a)
    h = torch.from_numpy(a['field']).cuda().to(torch.complex64)
    ny, nx = h.shape[0], h.shape[1]
    model = oi.abbe_model(sr, po, nm, sc.Period_Y, sc.Period_X, ny, nx)
    got = model.image(h.unsqueeze(0), kind=N.FIELD_COMPLEX_C64, nch=3, form='bf16x3')[0].cpu().numpy()
    fp32 = model.image(h.unsqueeze(0), kind=N.FIELD_COMPLEX_C64, nch=3)[0].cpu().numpy()
    want = O.abbe(sr, sc, po, nm)
    err, rms = rel_err(got, want), rms_rel(got, want)
    print(f'{name}: bf16x3 vs FP64 max {err:.2e} rms {rms:.2e}; fp32 vs FP64 max {rel_err(fp32, want):.2e}')
    assert err < BF16X3_VS_FP64
    assert rel_err(got, a['abbe']) < BF16X3_VS_FP64
    assert N.device_status() == 0


@pytest.mark.parametrize('name', ['vec_small', 'odd_scalar', 'cfg3_small'])
def test_hopkins_bf16x3_vs_reference(oi, name):
    from opticalimaging_b200 import _native as N
    meta, a = load(name)
    sr, sc, po, nm = build(meta, a)
    h = torch.from_numpy(a['field']).cuda().to(torch.complex64)
    ny, nx = h.shape[0], h.shape[1]
    model = oi.socs_model(sr, po, nm, sc.Period_Y, sc.Period_X, ny, nx)
    got = model.image(h.unsqueeze(0), kind=N.FIELD_COMPLEX_C64, nch=3, form='bf16x3')[0].cpu().numpy()
    fp32 = model.image(h.unsqueeze(0), kind=N.FIELD_COMPLEX_C64, nch=3)[0].cpu().numpy()
    print(f'{name}: bf16x3 vs fp32 max {rel_err(got, fp32):.2e} rms {rms_rel(got, fp32):.2e}; '
          f'vs reference max {rel_err(got, a["hopkins"]):.2e}')
    assert rel_err(got, fp32) < BF16X3_VS_FP64
    assert rel_err(got, a['hopkins']) < BF16X3_VS_FP64


def test_socs24_1024_bf16x3_vs_fp64(oi):
    """The headline workload: SOCS-24 from the vector annular TCC at 1024 x 1024 (2 nm pixels)."""
    from opticalimaging_b200 import workloads as W
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=24)
    T, fg = oi.CalculateTCCMatrix(sr, [2048.0, 2048.0], po, 0.0, nm)
    sk = oi.socs_kernels_from_tcc(T, fg, [1024, 1024], nm)
    masks = W.config3_masks(4, seed=11)
    md = torch.from_numpy(masks).cuda()
    got = sk.image(md, form='bf16x3').cpu().numpy()
    fp32 = sk.image(md, form='fft').cpu().numpy()
    assert rel_err(got, fp32) < BF16X3_VS_FP64
    s = Scatter()
    s.Period_X = s.Period_Y = 2048.0
    s.ScatterField = W.thin_field(masks[0])
    K = oi.DecomposeTCC_SOCS(T, fg, [1024, 1024], nm).cpu().numpy().astype(np.complex128)
    want = O.socs(s, K, sr, po)
    err, rms = rel_err(got[0], want), rms_rel(got[0], want)
    print(f'SOCS-24 1024^2: bf16x3 vs FP64 max {err:.2e} rms {rms:.2e}; fp32 max {rel_err(fp32[0], want):.2e}')
    assert err < BF16X3_VS_FP64


@pytest.mark.parametrize('batch', [3, 7])
def test_tc_ranges_cross_images_deterministic(oi, batch):
    """Two planes x 5 fields x 3 channels: task ranges that start and end inside images, partial slots
    zero-filled; the result is bit-identical run to run and matches the FP32 form."""
    from opticalimaging_b200 import _native as N
    from opticalimaging_b200.engine import Band, CoherentModel
    g = torch.Generator().manual_seed(batch)
    band = Band(-20, 41, -13, 27)
    pupils = torch.randn((2, 5, band.br, band.bc), dtype=torch.complex64, generator=g)
    weights = torch.rand((2, 5), generator=g) + 0.5
    model = CoherentModel(pupils.cuda(), weights.cuda(), band, 256, 256)
    field = (torch.rand((batch, 256, 256, 3), generator=g) > 0.5).to(torch.complex64).cuda()
    field[..., 1] *= 0.3j
    one = model.image(field, kind=N.FIELD_COMPLEX_C64, nch=3, form='bf16x3')
    two = model.image(field, kind=N.FIELD_COMPLEX_C64, nch=3, form='bf16x3')
    ref = model.image(field, kind=N.FIELD_COMPLEX_C64, nch=3, form='fft')
    assert torch.equal(one, two)
    assert rel_err(one.cpu().numpy(), ref.cpu().numpy()) < BF16X3_VS_FP64
    for b in range(batch):   # every image on its own gives the same result as in the batch
        solo = model.image(field[b:b + 1].contiguous(), kind=N.FIELD_COMPLEX_C64, nch=3, form='bf16x3')
        assert rel_err(solo.cpu().numpy(), ref[b:b + 1].cpu().numpy()) < BF16X3_VS_FP64
    assert N.device_status() == 0


@pytest.mark.parametrize('band', [(-29, 59, -29, 59), (-20, 41, -13, 27)])
@pytest.mark.parametrize('ctas', [1, 3, 7])
def test_coherent_tc_long_ranges_vs_fp64(oi, band, ctas):
    """Few CTAs, so each runs tens of fields through its pipeline (two operand slots for the symmetric band, one
    for the asymmetric band), against the coarse intensity evaluated in FP64 by torch; the partial sums of any
    cut add up to the same image."""
    from opticalimaging_b200 import _native as N
    from opticalimaging_b200.engine import Band, Plan, TC_COARSE
    dev = torch.device('cuda')
    b = Band(*band)
    batch, nk = 3, 9
    g = torch.Generator().manual_seed(ctas + b.bc)
    spec = torch.randn((batch, 1, b.br, b.bc), dtype=torch.complex64, generator=g)
    pup = torch.randn((1, nk, b.br, b.bc), dtype=torch.complex64, generator=g)
    w = torch.rand((1, nk), generator=g) + 0.5
    plan = Plan.get(256, 256, b, dev, coarse=TC_COARSE)
    s = N.stream_handle(dev)
    specd, pupd, wd = spec.to(dev), pup.to(dev), w.to(dev)

    def run(c, nparts):
        coarse = torch.full((nparts, batch, 1, 128, 128), float('nan'), device=dev)
        N.call('oi_coherent_coarse_tc', N.ptr(specd), batch, 1, b.m0r, b.br, b.m0c, b.bc, N.ptr(pupd), 0, N.ptr(wd),
               1, nk, N.ptr(plan.tc_constants()), c, nparts, N.ptr(coarse), s)
        return coarse.double().sum(dim=0)[:, 0].cpu()

    got = run(ctas, ctas + 1)            # slots past the cut's own are zero-filled
    default = run(*N.tc_layout(batch, nk))
    # FP64: E[sr][sc] = sum_ir sum_ic exp(-2 pi i ((m0r+ir) sr + (m0c+ic) sc) / 128) P[ir][ic] band[ir][ic]
    s128 = torch.arange(128, dtype=torch.float64)
    cr = torch.exp(-2j * np.pi * torch.outer(s128, b.m0r + torch.arange(b.br, dtype=torch.float64)) / 128)
    cc = torch.exp(-2j * np.pi * torch.outer(s128, b.m0c + torch.arange(b.bc, dtype=torch.float64)) / 128)
    a = spec[:, 0, None].to(torch.complex128) * pup[0, None].to(torch.complex128)   # [batch][nk][br][bc]
    e = torch.einsum('ri,bkij,cj->bkrc', cr, a, cc)
    ref = torch.einsum('k,bkrc->brc', w[0].double(), e.abs() ** 2)
    assert rel_err(got.numpy(), ref.numpy()) < BF16X3_VS_FP64
    assert rel_err(got.numpy(), default.numpy()) < 1e-6
    assert N.device_status() == 0


@pytest.mark.parametrize('ny,nx,band', [
    (256, 256, (-15, 31, -15, 31)),
    (512, 1024, (-29, 59, -29, 59)),
    (1024, 1024, (-29, 59, -20, 41)),
    (2048, 512, (-31, 63, 0, 64)),
])
def test_tc_row_passes_vs_fft(oi, ny, nx, band):
    """Band spectrum (tensor-core row pass + FFT columns) of float32 and uint8 masks, and the synthesis
    (FFT columns + tensor-core row pass), against the FP32 FFT form."""
    from opticalimaging_b200 import _native as N
    from opticalimaging_b200.engine import Band, CoherentModel, Plan, band_spectrum
    dev = torch.device('cuda')
    b = Band(*band)
    plan = Plan.get(ny, nx, b, dev)
    assert plan.tc_rows('bf16x3')
    rng = np.random.default_rng(ny + nx)
    m = (rng.random((3, ny, nx)) > 0.6).astype(np.float32)
    m[1] *= rng.random((ny, nx)).astype(np.float32)          # a grey mask too
    md = torch.from_numpy(m).to(dev)
    want = band_spectrum(md, N.FIELD_REAL_F32, plan, form='fft').cpu().numpy()
    got = band_spectrum(md, N.FIELD_REAL_F32, plan, form='bf16x3').cpu().numpy()
    assert rel_err(got, want) < 2e-5
    u8 = torch.from_numpy((m[[0, 2]] > 0).astype(np.uint8)).to(dev)
    got8 = band_spectrum(u8, N.FIELD_U8, plan, form='bf16x3').cpu().numpy()
    assert rel_err(got8, want[[0, 2]]) < 2e-5
    g = torch.Generator().manual_seed(ny)
    pupils = torch.randn((1, 3, b.br, b.bc), dtype=torch.complex64, generator=g)
    model = CoherentModel(pupils.to(dev), torch.ones((1, 3), device=dev), b, ny, nx)
    img = model.image(md, form='bf16x3').cpu().numpy()
    ref = model.image(md, form='fft').cpu().numpy()
    print(f'{ny}x{nx}: band max {rel_err(got, want):.2e}, image max {rel_err(img, ref):.2e} rms {rms_rel(img, ref):.2e}')
    assert rel_err(img, ref) < BF16X3_VS_FP64
    assert N.device_status() == 0


@pytest.mark.parametrize('count,ny,nx,bc', [(1, 128, 256, 40), (7, 640, 2048, 33), (5, 1024, 1024, 59),
                                            (3, 384, 384, 21), (64, 1024, 1024, 59), (2, 256, 512, 64)])
def test_rows_inv_tc_direct(oi, count, ny, nx, bc):
    """The inverse tensor-core row pass through the C ABI against an FP64 evaluation of
    out[i][y][x] = sum_qc Re(v[i][qc][y] exp(-2 pi i qc x / nx)): one item, ranges crossing x tiles and images,
    the 64-clip benchmark shape, a full 64-column band, nx = 384 and odd numbers of 128-row blocks (the last pair
    half empty); columns 0, nx/2 and nx - 1 checked on their own."""
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    g = torch.Generator().manual_seed(count * ny + nx)
    v = torch.randn((count, bc, ny), dtype=torch.complex64, generator=g)
    s = N.stream_handle(dev)
    consts = torch.empty((nx // 128) * 65536, dtype=torch.uint8, device=dev)
    N.call('oi_rows_tc_constants', 1, nx, 0, bc, N.ptr(consts), consts.numel(), s)
    vd = v.to(dev)
    tiles = torch.empty(count * ny * 512, dtype=torch.uint8, device=dev)
    out = torch.full((count, ny, nx), float('nan'), device=dev)
    N.call('oi_rows_inv_tc', N.ptr(vd), count, ny, nx, bc, N.ptr(consts), N.ptr(tiles), N.ptr(out), s)
    got = out.cpu().numpy()
    E = np.exp(-2j * np.pi * np.outer(np.arange(bc), np.arange(nx)) / nx)
    vv = v.numpy().astype(np.complex128)
    want = np.stack([np.real(vv[i].T @ E) for i in range(count)])
    err, rms = rel_err(got, want), rms_rel(got, want)
    print(f'inverse rows {count}x{ny}x{nx} bc {bc}: max {err:.2e} rms {rms:.2e}')
    assert not np.isnan(got).any()
    assert err < BF16X3_VS_FP64
    peak = np.max(np.abs(want))
    for col in (0, nx // 2, nx - 1):
        assert np.max(np.abs(got[:, :, col] - want[:, :, col])) < BF16X3_VS_FP64 * peak, col
    assert N.device_status() == 0


def test_kernels_wait_for_the_preceding_torch_kernel(oi):
    """The split form's kernels may start before the previous kernel on the stream has finished (programmatic
    dependent launch) but wait for it before reading: masks written by a torch kernel right before the call give
    bit-identical images to masks that were synchronised first, and a torch kernel right after sees the images."""
    from opticalimaging_b200 import workloads as W
    sr, po, nm = W.config3_optics(order=24)
    T, fg = oi.CalculateTCCMatrix(sr, [512.0, 512.0], po, 0.0, nm)
    sk = oi.socs_kernels_from_tcc(T, fg, [256, 256], nm)
    torch.manual_seed(7)
    base = torch.rand((8, 256, 256), device='cuda')
    want = sk.image((base > 0.5).float(), form='bf16x3').clone()
    torch.cuda.synchronize()
    for _ in range(3):
        masks = (base > 0.5).float()                  # a torch kernel, not synchronised
        got = sk.image(masks, form='bf16x3')
        total = got.sum()                             # a torch kernel reading the images right away
        assert torch.equal(got, want)
        assert torch.isclose(total, want.sum(), rtol=1e-6)


@pytest.mark.parametrize('count,ny,nx,m0c,bc,u8', [(1, 384, 256, -7, 15, False), (3, 640, 512, -29, 59, False),
                                                   (2, 256, 1024, 0, 64, True), (5, 1024, 1024, -29, 59, False)])
def test_rows_fwd_tc_direct(oi, count, ny, nx, m0c, bc, u8):
    """The forward tensor-core row pass through the C ABI against an FP64 evaluation of
    t[b][ic][y] = sum_x mask[b][y][x] exp(+2 pi i (m0c+ic) x / nx): an odd number of 128-row blocks (the last
    pair of blocks half empty), grey float32 masks and uint8 masks, more pairs than CTAs."""
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    rng = np.random.default_rng(count * ny + nx)
    if u8:
        m = (rng.random((count, ny, nx)) > 0.5).astype(np.uint8) * rng.integers(1, 255, (count, ny, nx)).astype(np.uint8)
    else:
        m = (rng.random((count, ny, nx)) > 0.6).astype(np.float32) * rng.random((count, ny, nx)).astype(np.float32)
    s = N.stream_handle(dev)
    nbytes = (nx // 64) * 32768
    consts = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    N.call('oi_rows_tc_constants', 0, nx, m0c, bc, N.ptr(consts), nbytes, s)
    md = torch.from_numpy(m).to(dev)
    t = torch.full((count, bc, ny), complex(float('nan'), 0.0), dtype=torch.complex64, device=dev)
    N.call('oi_rows_fwd_tc', N.ptr(md), N.FIELD_U8 if u8 else N.FIELD_REAL_F32, count, ny, nx, m0c, bc,
           N.ptr(consts), N.ptr(t), s)
    got = t.cpu().numpy()
    E = np.exp(2j * np.pi * np.outer(np.arange(nx), m0c + np.arange(bc)) / nx)     # [nx][bc]
    want = np.stack([(m[i].astype(np.float64) @ E).T for i in range(count)])       # [count][bc][ny]
    err = rel_err(got, want)
    print(f'forward rows {count}x{ny}x{nx} bc {bc} u8={u8}: max {err:.2e}')
    assert err < 2e-5
    assert N.device_status() == 0


@pytest.mark.parametrize('count,ny,nx,bc,u8', [(1, 384, 256, 15, False), (3, 640, 512, 59, False),
                                               (2, 256, 1024, 63, True), (5, 1024, 1024, 59, False)])
def test_rows_fwd_tc_half_direct(oi, count, ny, nx, bc, u8):
    """The Hermitian-half forward row pass (oi_rows_fwd_tc_half, constants of oi_rows_tc_constants(2, ...)) against
    FP64 t[b][kx][y] = sum_x mask[b][y][x] exp(+2 pi i kx x / nx), kx = 0 .. (bc-1)/2: odd block counts, the widest
    half (32 columns), uint8 masks."""
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    rng = np.random.default_rng(count * ny + nx + 1)
    if u8:
        m = (rng.random((count, ny, nx)) > 0.5).astype(np.uint8) * rng.integers(1, 255, (count, ny, nx)).astype(np.uint8)
    else:
        m = (rng.random((count, ny, nx)) > 0.6).astype(np.float32) * rng.random((count, ny, nx)).astype(np.float32)
    s = N.stream_handle(dev)
    bch = (bc + 1) // 2
    nbytes = (nx // 64) * 16384
    consts = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    N.call('oi_rows_tc_constants', 2, nx, -(bc - 1) // 2, bc, N.ptr(consts), nbytes, s)
    md = torch.from_numpy(m).to(dev)
    t = torch.full((count, bch + 1, ny), complex(float('nan'), 0.0), dtype=torch.complex64, device=dev)
    N.call('oi_rows_fwd_tc_half', N.ptr(md), N.FIELD_U8 if u8 else N.FIELD_REAL_F32, count, ny, nx, bch,
           N.ptr(consts), N.ptr(t), s)
    got = t.cpu().numpy().reshape(-1)[:count * bch * ny].reshape(count, bch, ny)
    assert np.isnan(t.cpu().numpy().reshape(-1)[count * bch * ny:]).all()     # nothing written past the output
    E = np.exp(2j * np.pi * np.outer(np.arange(nx), np.arange(bch)) / nx)        # [nx][bch]
    want = np.stack([(m[i].astype(np.float64) @ E).T for i in range(count)])    # [count][bch][ny]
    err = rel_err(got, want)
    print(f'forward half rows {count}x{ny}x{nx} bch {bch} u8={u8}: max {err:.2e}')
    assert err < 2e-5
    assert N.device_status() == 0


def test_rows_tc_constants_half_rejects_asymmetric_band(oi):
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    c = torch.empty(4 * 16384, dtype=torch.uint8, device=dev)
    for m0c, bc in ((-6, 15), (-7, 16), (-32, 65)):
        with pytest.raises(N.NativeError):
            N.call('oi_rows_tc_constants', 2, 256, m0c, bc, N.ptr(c), c.numel(), N.stream_handle(dev))


@pytest.mark.parametrize('batch,n,b', [(3, 256, 15), (2, 1024, 59), (1, 512, 63)])
def test_band_spectrum_tc_sym_matches_full(oi, batch, n, b):
    """The symmetric-band spectrum (half row pass + mirrored column pass) against the full tensor-core row pass
    and against FP64, float32 masks."""
    from opticalimaging_b200 import engine as E, _native as N
    dev = torch.device('cuda')
    band = E.Band(-(b - 1) // 2, b, -(b - 1) // 2, b)
    plan = E.Plan.get(n, n, band, dev)
    assert plan.symmetric_band()
    rng = np.random.default_rng(n + b)
    m = ((rng.random((batch, n, n)) > 0.6) * rng.random((batch, n, n))).astype(np.float32)
    md = torch.from_numpy(m).to(dev)
    s = N.stream_handle(dev)
    scratch = torch.empty(batch * n * b, dtype=torch.complex64, device=dev)
    full = torch.empty((batch, 1, b, b), dtype=torch.complex64, device=dev)
    half = torch.full((batch, 1, b, b), complex(float('nan'), 0.0), dtype=torch.complex64, device=dev)
    N.call('oi_band_spectrum_tc', N.ptr(md), N.FIELD_REAL_F32, batch, n, n, band.m0r, b, band.m0c, b,
           N.ptr(plan.rows_consts(0)), N.ptr(plan.wn_y), 1.0 / (n * n), N.ptr(scratch), N.ptr(full), s)
    N.call('oi_band_spectrum_tc_sym', N.ptr(md), N.FIELD_REAL_F32, batch, n, n, b, b, N.ptr(plan.rows_consts(2)),
           N.ptr(plan.wn_y), 1.0 / (n * n), N.ptr(scratch), N.ptr(half), s)
    h, f = half.cpu().numpy(), full.cpu().numpy()
    assert not np.isnan(h).any()
    k = np.arange(b) - (b - 1) // 2
    Ey = np.exp(2j * np.pi * np.outer(k, np.arange(n)) / n)       # [ky][y]
    Ex = np.exp(2j * np.pi * np.outer(np.arange(n), k) / n)       # [x][kx]
    want = np.stack([Ey @ m[i].astype(np.float64) @ Ex for i in range(batch)])[:, None] / (n * n)
    assert rel_err(h, want) < 2e-5
    assert rel_err(h, f) < 2e-5
    assert N.device_status() == 0


def decode_v_tiles(tiles: np.ndarray, count: int, ny: int) -> np.ndarray:
    """v [count, 64, ny] complex from V operand tiles ([count*ny/128][hi re | hi im | lo re | lo im][128 y][64 qc] bf16,
    128-byte swizzled): hi + lo of each part."""
    t = tiles.reshape(count * ny // 128, 4, 128, 128)                     # bytes: [tile][block][row][128 B]
    r = np.arange(128)[:, None]
    k = np.arange(64)[None, :]
    off = ((k // 8) ^ (r % 8)) * 16 + (k % 8) * 2
    lo_b = np.take_along_axis(t, np.broadcast_to(off, (t.shape[0], 4, 128, 64)), axis=3).astype(np.uint32)
    hi_b = np.take_along_axis(t, np.broadcast_to(off + 1, (t.shape[0], 4, 128, 64)), axis=3).astype(np.uint32)
    f = ((hi_b << 24) | (lo_b << 16)).view(np.float32).astype(np.float64)   # bf16 -> float32 bits
    re, im = f[:, 0] + f[:, 2], f[:, 1] + f[:, 3]                          # [tile][y][qc]
    v = (re + 1j * im).reshape(count, ny, 64)
    return v.transpose(0, 2, 1)


@pytest.mark.parametrize('count,nparts,ny,br,bc', [(3, 3, 256, 59, 59), (64, 2, 1024, 59, 59), (5, 1, 512, 30, 17)])
def test_synth_tiles_tc_direct(oi, count, nparts, ny, br, bc):
    """The tensor-core synthesis preparation through the C ABI against FP64: the V tiles (hi + lo) of
    v[qc][y] = sum_|qr|<br Ihat[qr][qc] exp(-2 pi i qr y / ny), Ihat the (qc > 0 doubled) coarse spectrum of the
    sum of the partial coarse images; zero beyond bc."""
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    g = np.random.default_rng(count * ny + br)
    coarse = g.random((nparts, count, 128, 128)).astype(np.float32)
    c = coarse.astype(np.float64).sum(axis=0)
    consts = torch.empty((1 + ny // 128) * 65536, dtype=torch.uint8, device=dev)
    s = N.stream_handle(dev)
    N.call('oi_synth_tc_constants', ny, br, bc, N.ptr(consts), consts.numel(), s)
    cd = torch.from_numpy(coarse).to(dev)
    tiles = torch.zeros(count * ny * 512, dtype=torch.uint8, device=dev)
    N.call('oi_synth_tiles_tc', N.ptr(cd), nparts, count, br, bc, N.ptr(consts), ny, N.ptr(tiles), s)
    got = decode_v_tiles(tiles.cpu().numpy(), count, ny)
    qr = np.arange(-(br - 1), br)
    qc = np.arange(bc)
    s128 = np.arange(128)
    Er = np.exp(2j * np.pi * np.outer(qr, s128) / 128)
    Ec = np.exp(2j * np.pi * np.outer(s128, qc) / 128)
    ih = np.einsum('ra,iab,bc->irc', Er, c, Ec) / 128 ** 2
    ih[:, :, 1:] *= 2
    Sy = np.exp(-2j * np.pi * np.outer(qr, np.arange(ny)) / ny)            # [nq, ny]
    want = np.einsum('irc,ry->icy', ih, Sy)
    err = np.max(np.abs(got[:, :bc] - want)) / np.max(np.abs(want))
    print(f'synth tiles {count}x{ny} br {br} bc {bc} parts {nparts}: max {err:.2e}')
    assert err < BF16X3_VS_FP64
    assert np.all(got[:, bc:] == 0)
    assert N.device_status() == 0


def test_bounded_wait_expiry_reports_and_recovers(oi):
    """The tensor-core kernels' failure path, made to happen without a fault: a bounded wait (10 ms here) on a
    barrier that nothing completes sets the device status and releases tensor memory (all 512 columns), the
    status is read and cleared on the host, and the next calls -- which allocate all 512 columns again -- run
    normally with bit-identical results."""
    from opticalimaging_b200 import _native as N, workloads as W
    sr, po, nm = W.config3_optics(order=8)
    T, fg = oi.CalculateTCCMatrix(sr, [512.0, 512.0], po, 0.0, nm)
    sk = oi.socs_kernels_from_tcc(T, fg, [256, 256], nm)
    g = torch.Generator(device='cuda').manual_seed(3)
    masks = (torch.rand((4, 256, 256), device='cuda', generator=g) > 0.5).float()
    before = sk.image(masks, form='bf16x3').clone()
    N.device_status(reset=True)
    N.call('oi_wait_probe', 10_000_000, 512, N.stream_handle())
    torch.cuda.synchronize()
    assert N.device_status() == 1
    with pytest.raises(N.DeviceWaitError):
        N.check_device_status('wait probe')
    assert N.device_status() == 0
    after = sk.image(masks, form='bf16x3')
    torch.cuda.synchronize()
    assert torch.equal(before, after)
    assert N.device_status() == 0
    with pytest.raises(N.NativeError, match='outside'):
        N.call('oi_wait_probe', 10 ** 9, 512, N.stream_handle())      # limits above 100 ms are refused
