"""FFT form of the two N-point stages vs numpy and vs the DFT form, on every supported grid size."""
import numpy as np
import pytest
import torch

from oracle import optics64 as O
from tests.fixtures import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def eng():
    from opticalimaging_b200 import engine
    return engine


@pytest.mark.parametrize('ny,nx,band', [
    (256, 256, (-15, 31, -15, 31)),
    (512, 256, (-20, 29, -7, 30)),      # asymmetric column band: the mirror range is wider than the band
    (1024, 1024, (-29, 59, -29, 59)),
    (256, 2048, (-3, 7, -100, 201)),
    (2048, 512, (-60, 121, -1, 3)),
])
def test_band_spectrum_fft(eng, ny, nx, band):
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    b = eng.Band(*band)
    plan = eng.Plan.get(ny, nx, b, dev)
    assert plan.fft
    rng = np.random.default_rng(ny + nx)
    m = (rng.random((3, ny, nx)) > 0.6).astype(np.float32)
    m[1] *= rng.random((ny, nx)).astype(np.float32)          # a grey mask too
    want = np.fft.ifft2(m.astype(np.float64), axes=(1, 2))
    rows = np.arange(b.m0r, b.m0r + b.br) % ny
    cols = np.arange(b.m0c, b.m0c + b.bc) % nx
    want = want[:, rows][:, :, cols]
    md = torch.from_numpy(m).to(dev)
    got = eng.band_spectrum(md, N.FIELD_REAL_F32, plan, form='fft')[:, 0].cpu().numpy()
    dft = eng.band_spectrum(md, N.FIELD_REAL_F32, plan, form='dft')[:, 0].cpu().numpy()
    assert rel_err(got, want) < 3e-6
    assert rel_err(dft, want) < 3e-6
    u8 = torch.from_numpy((m[[0, 2]] > 0).astype(np.uint8)).to(dev)
    got8 = eng.band_spectrum(u8, N.FIELD_U8, plan, form='fft')[:, 0].cpu().numpy()
    assert rel_err(got8, want[[0, 2]]) < 3e-6


@pytest.mark.parametrize('ny,nx,order', [(256, 256, 8), (512, 1024, 12), (1024, 1024, 24), (2048, 256, 6)])
def test_socs_fft_matches_dft_and_oracle(eng, ny, nx, order):
    from opticalimaging_b200 import imaging, workloads as W
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=order)
    T, fg = imaging.CalculateTCCMatrix(sr, [2048.0 * ny / 1024, 2048.0 * nx / 1024], po, 0.0, nm)
    sk = imaging.socs_kernels_from_tcc(T, fg, [nx, ny], nm)
    assert sk.plan.fft
    rng = np.random.default_rng(order)
    masks = np.stack([W.rect_mask(ny, nx, 2.0 * ny, 2.0 * nx, 40, 30, 400, rng) for _ in range(2)])
    md = torch.from_numpy(masks).cuda()
    fft = sk.image(md, form='fft').cpu().numpy()
    dft = sk.image(md, form='dft').cpu().numpy()
    assert rel_err(fft, dft) < 5e-6
    if ny * nx <= 512 * 1024:
        sc = Scatter()
        sc.Period_X, sc.Period_Y = 2.0 * nx, 2.0 * ny
        sc.ScatterField = W.thin_field(masks[0])
        K = imaging.DecomposeTCC_SOCS(T, fg, [nx, ny], nm).cpu().numpy().astype(np.complex128)
        assert rel_err(fft[0], O.socs(sc, K, sr, po)) < 1e-5


def test_fft_rejects_unsupported_grid(eng):
    from opticalimaging_b200 import _native as N
    lib = N.load()
    assert lib.oi_fft_supported(1024, 1024) == 1
    assert lib.oi_fft_supported(1000, 1024) == 0
    assert lib.oi_fft_supported(128, 1024) == 0
    plan = eng.Plan.get(45, 63, eng.Band(-5, 11, -5, 11), torch.device('cuda'))
    assert not plan.fft   # odd grids take the DFT form


def test_large_band_coarse_256_fft_vs_dft_and_oracle(eng):
    """Band 117 (> 64): coarse grid 256 x 256, DFT coherent sum split over fields, coarse spectrum by the FFT
    band pass and FFT synthesis; against the all-DFT form and the FP64 oracle (kernels from the Gram path)."""
    from opticalimaging_b200 import imaging, workloads as W, _native as N
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=8)
    model = imaging.socs_model(sr, po, nm, 4096.0, 4096.0, 1024, 1024)
    assert model.band.br > 64 and model.plan.mr == 256 and model.plan.big_coarse_fft(None)
    rng = np.random.default_rng(9)
    masks = np.stack([W.rect_mask(1024, 1024, 4096.0, 4096.0, 30, 40, 600, rng) for _ in range(3)])
    md = torch.from_numpy(masks).cuda()
    fft = model.image(md)[:, 0].cpu().numpy()
    dft = model.image(md, form='dft')[:, 0].cpu().numpy()
    assert rel_err(fft, dft) < 5e-6
    b = model.band
    full = torch.zeros((1024, 1024, model.count), dtype=torch.complex64, device=model.device)
    full[:b.br, :b.bc, :] = model.pupils[0].permute(1, 2, 0)
    K = torch.roll(full, shifts=(b.m0r, b.m0c), dims=(0, 1)).cpu().numpy().astype(np.complex128)
    sc = Scatter()
    sc.Period_X = sc.Period_Y = 4096.0
    sc.ScatterField = W.thin_field(masks[0])
    assert rel_err(fft[0], O.socs(sc, K, sr, po)) < 1e-5
    assert N.device_status() == 0


def test_clip_2048_large_band_vs_oracle(eng):
    """A 2048 x 2048 clip at 2 nm per pixel (4096 nm period, band 117 > 64: coarse grid 256 x 256, the FP32 FFT
    form the served 2048-point clips take) against the FP64 oracle with the same SOCS kernels, at the FP32
    forms' bound of 1e-5 of peak."""
    from opticalimaging_b200 import imaging, workloads as W, _native as N
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=8)
    model = imaging.socs_model(sr, po, nm, 4096.0, 4096.0, 2048, 2048)
    assert model.band.br > 64 and model.plan.mr == 256 and model.plan.fft
    rng = np.random.default_rng(21)
    masks = np.stack([W.rect_mask(2048, 2048, 4096.0, 4096.0, 30, 40, 600, rng) for _ in range(2)])
    img = model.image(torch.from_numpy(masks).cuda())[:, 0].cpu().numpy()
    b = model.band
    full = torch.zeros((2048, 2048, model.count), dtype=torch.complex64, device=model.device)
    full[:b.br, :b.bc, :] = model.pupils[0].permute(1, 2, 0)
    K = torch.roll(full, shifts=(b.m0r, b.m0c), dims=(0, 1)).cpu().numpy().astype(np.complex128)
    del full
    sc = Scatter()
    sc.Period_X = sc.Period_Y = 4096.0
    for i in range(2):
        sc.ScatterField = W.thin_field(masks[i])
        err = rel_err(img[i], O.socs(sc, K, sr, po))
        print(f'2048 x 2048 clip {i}: max error {err:.2e} of peak')
        assert err < 1e-5
    assert N.device_status() == 0


@pytest.mark.parametrize('nparts,count,m,br,bc', [(3, 2, 256, 117, 59), (1, 3, 256, 70, 66), (2, 1, 512, 128, 128)])
def test_coarse_half_spectrum_fft(eng, nparts, count, m, br, bc):
    """oi_coarse_half_spectrum_fft (parts summed in the row pass, columns qc > 0 doubled) against FP64
    ihat[qr][qc] = w(qc) / m^2 sum_{y,x} c[y][x] exp(+2 pi i (qr y + qc x) / m)."""
    from opticalimaging_b200 import _native as N
    dev = torch.device('cuda')
    rng = np.random.default_rng(nparts * 100 + br)
    coarse = rng.random((nparts, count, m, m)).astype(np.float32)
    c = coarse.astype(np.float64).sum(axis=0)
    tables = eng.fft_tables(m, dev)
    cd = torch.from_numpy(coarse).to(dev)
    t = torch.empty(count * m * bc, dtype=torch.complex64, device=dev)
    ihat = torch.empty((count, 2 * br - 1, bc), dtype=torch.complex64, device=dev)
    N.call('oi_coarse_half_spectrum_fft', N.ptr(cd), nparts, count, m, m, br, bc, N.ptr(tables), N.ptr(tables),
           N.ptr(t), N.ptr(ihat), N.stream_handle(dev))
    qr = np.arange(-(br - 1), br)
    E = np.exp(2j * np.pi * np.arange(m) / m)
    Er = E[np.outer(qr, np.arange(m)) % m]                  # [nq][y]
    Ec = E[np.outer(np.arange(m), np.arange(bc)) % m]       # [x][qc]
    want = np.einsum('ry,iyx,xc->irc', Er, c, Ec) / m ** 2
    want[:, :, 1:] *= 2
    err = rel_err(ihat.cpu().numpy(), want)
    print(f'coarse half spectrum {nparts} parts {count}x{m}^2 band {br}x{bc}: {err:.2e}')
    assert err < 2e-6
    assert N.device_status() == 0


@pytest.mark.parametrize('batch,nch,nz,nk,br,bc,m0r,m0c,nsplit,per_image', [
    (2, 2, 2, 3, 70, 66, -35, -30, 4, False),     # 12 fields over 4 splits, two planes, two channels
    (2, 1, 1, 5, 128, 128, -64, -64, 2, True),    # the largest band; pupils per image
    (1, 1, 1, 2, 117, 65, -58, 5, 1, False),      # asymmetric band, offset column band
])
def test_coherent_coarse_fft_256(eng, batch, nch, nz, nk, br, bc, m0r, m0c, nsplit, per_image):
    """The 256 x 256 coarse grid (tensor-memory accumulator) against an FP64 numpy evaluation of
    sum_{k,c} w |sum A[ir][ic] exp(-2 pi i ((m0r+ir) sr + (m0c+ic) sc) / 256)|^2, A = P[z][k] .* band[b][c]."""
    from opticalimaging_b200 import _native as N
    rng = np.random.default_rng(br * 1000 + bc)
    cplx = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s))  # noqa: E731
    band = cplx(batch, nch, br, bc)
    pup = cplx(batch if per_image else 1, nz, nk, br, bc)
    w = rng.random((nz, nk)) + 0.1
    j = np.arange(256)
    cr = np.exp(-2j * np.pi * np.outer(j, m0r + np.arange(br)) / 256)     # [sr][ir]
    cc = np.exp(-2j * np.pi * np.outer(m0c + np.arange(bc), j) / 256)     # [ic][sc]
    want = np.zeros((batch, nz, 256, 256))
    for b in range(batch):
        for z in range(nz):
            for k in range(nk):
                for c in range(nch):
                    e = cr @ (pup[b if per_image else 0, z, k] * band[b, c]) @ cc
                    want[b, z] += w[z, k] * np.abs(e) ** 2
    dev = torch.device('cuda')
    tb = torch.from_numpy(band.astype(np.complex64)).to(dev)
    tp = torch.from_numpy(pup.astype(np.complex64)).to(dev)
    tw = torch.from_numpy(w.astype(np.float32)).to(dev)
    tab = torch.from_numpy(np.exp(2j * np.pi * j / 256).astype(np.complex64)).to(dev)
    coarse = torch.full((nsplit, batch, nz, 256, 256), float('nan'), device=dev)
    stride = nz * nk * br * bc if per_image else 0
    N.call('oi_coherent_coarse_fft', N.ptr(tb), batch, nch, m0r, br, m0c, bc, N.ptr(tp), stride, N.ptr(tw), nz, nk,
           256, 256, N.ptr(tab), N.ptr(tab), nsplit, N.ptr(coarse), N.stream_handle(dev))
    got = coarse.sum(dim=0).cpu().numpy()
    assert rel_err(got, want) < 5e-6
    assert N.device_status() == 0
