"""Parity of the CUDA engine with the FP64 oracle and with the reference's own outputs (golden fixtures).

Tolerances are relative to the peak of the reference image: the FP32 engine form must agree with the FP64
oracle and with the complex64 reference to 1e-5 of peak.  (The reference's own rounding on these fixtures is
1.2e-6 to 2.5e-6 of peak against FP64, pinned in tests/test_oracle_golden.py; the engine's is of the same size,
so the two stay well inside 1e-5 of each other.  Each test records its measured errors.)
"""
import warnings

import numpy as np
import pytest
import torch

from oracle import optics64 as O
from tests.fixtures import build, load, rel_err

pytestmark = pytest.mark.gpu

FP32_VS_FP64 = 1e-5
FP32_VS_REF = 1e-5


@pytest.fixture(scope='module')
def oi():
    import opticalimaging_b200.imaging as imaging
    from opticalimaging_b200 import _native
    _native.load()
    return imaging


def test_band_spectrum_matches_numpy(oi):
    from opticalimaging_b200 import engine as E, _native as N
    dev = torch.device('cuda')
    rng = np.random.default_rng(0)
    for ny, nx, band in ((64, 48, E.Band(-7, 15, -5, 11)), (45, 63, E.Band(-22, 45, -31, 63)),
                         (17, 23, E.Band(-3, 4, 2, 5))):
        h = (rng.standard_normal((2, ny, nx, 3)) + 1j * rng.standard_normal((2, ny, nx, 3))).astype(np.complex64)
        plan = E.Plan.get(ny, nx, band, dev)
        got = E.band_spectrum(torch.from_numpy(h).to(dev), N.FIELD_COMPLEX_C64, plan, nch=3).cpu().numpy()
        # header definition: c(m) = 1/(ny nx) sum h exp(+2 pi i m.y/N), origin at pixel 0 (= ifft2 at m mod N)
        full = np.fft.ifft2(h.astype(np.complex128), axes=(1, 2))
        rows = np.arange(band.m0r, band.m0r + band.br) % ny
        cols = np.arange(band.m0c, band.m0c + band.bc) % nx
        want = full[:, rows][:, :, cols].transpose(0, 3, 1, 2)
        assert rel_err(got, want) < 2e-6
        # real and uint8 kinds of the same data
        r = (rng.random((3, ny, nx)) > 0.5)
        want_r = np.fft.ifft2(r.astype(np.float64), axes=(1, 2))[:, rows][:, :, cols]
        got_f = E.band_spectrum(torch.from_numpy(r.astype(np.float32)).to(dev), N.FIELD_REAL_F32, plan)
        got_u = E.band_spectrum(torch.from_numpy(r.astype(np.uint8)).to(dev), N.FIELD_U8, plan)
        assert rel_err(got_f[:, 0].cpu().numpy(), want_r) < 2e-6
        assert rel_err(got_u[:, 0].cpu().numpy(), want_r) < 2e-6


@pytest.mark.parametrize('name', ['cfg1', 'vec_small', 'odd_scalar', 'cfg2_small'])
def test_abbe_parity(oi, name, report):
    meta, a = load(name)
    sr, sc, po, nm = build(meta, a)
    img, pim = oi.CalculateAbbeImage(sr, sc, po, nm)
    got = img.Intensity.numpy()
    assert got.shape == a['abbe'].shape
    o = O.abbe(sr, sc, po, nm)
    report(f'abbe_{name}', engine_vs_fp64=rel_err(got, o), engine_vs_reference=rel_err(got, a['abbe']),
           reference_vs_fp64=rel_err(a['abbe'], o))
    assert rel_err(got, o) < FP32_VS_FP64
    assert rel_err(got, a['abbe']) < FP32_VS_REF
    np.testing.assert_array_equal(np.isnan(pim.numpy()), np.isnan(a['abbe_pupil']))
    ok = ~np.isnan(a['abbe_pupil'])
    assert rel_err(pim.numpy()[ok], a['abbe_pupil'][ok]) < 1e-5


def test_socs_with_reference_kernels(oi, report):
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    got, _ = oi.CalculateAerialImage_SOCS(sc, torch.from_numpy(a['kernels']), sr, po)
    o = O.socs(sc, a['kernels'].astype(np.complex128), sr, po)
    report('socs_vec_small', engine_vs_fp64=rel_err(got.numpy(), o), engine_vs_reference=rel_err(got.numpy(), a['socs']),
           reference_vs_fp64=rel_err(a['socs'], o))
    assert rel_err(got.numpy(), a['socs']) < FP32_VS_REF
    assert rel_err(got.numpy(), o) < FP32_VS_FP64


@pytest.mark.parametrize('name', ['vec_small', 'odd_scalar', 'cfg3_small'])
def test_hopkins_parity(oi, name, report):
    meta, a = load(name)
    sr, sc, po, nm = build(meta, a)
    img, _ = oi.CalculateHopkinsImage(sr, sc, po, nm)
    report(f'hopkins_{name}', engine_vs_reference=rel_err(img.Intensity.numpy(), a['hopkins']))
    assert rel_err(img.Intensity.numpy(), a['hopkins']) < FP32_VS_REF


def test_tcc_fp64(oi):
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    T, fg = oi.CalculateTCCMatrix(sr, [meta['Period_Y'], meta['Period_X']], po, meta['focus'][0], nm)
    assert T.dtype == torch.complex128 and list(fg) == list(a['fg'])
    To, _ = O.tcc(sr, [meta['Period_Y'], meta['Period_X']], po, meta['focus'][0], nm)
    assert rel_err(T.cpu().numpy(), To) < 1e-12
    assert rel_err(T.cpu().numpy(), a['tcc']) < 2e-6
    K = oi.DecomposeTCC_SOCS(T, fg, [sc.ScatterField.shape[1], sc.ScatterField.shape[0]], nm)
    Ko = O.decompose(To, fg, [sc.ScatterField.shape[1], sc.ScatterField.shape[0]], nm)
    assert K.shape == Ko.shape
    # same subspace: the rank-K TCC sum_k K_k K_k^H agrees (kernel phases are arbitrary)
    kg, ko = K.cpu().numpy().reshape(-1, K.shape[2]), Ko.reshape(-1, Ko.shape[2])
    assert rel_err(kg @ kg.conj().T, ko @ ko.conj().T) < 1e-6


def test_tcc_cfg3_spectrum(oi):
    from opticalimaging_b200 import workloads as W
    meta, a = load('cfg3_tcc')
    sr, po, nm = W.config3_optics()
    T, fg = oi.CalculateTCCMatrix(sr, [2048, 2048], po, 0.0, nm)
    lam = torch.linalg.eigvalsh(T).flip(0)[:64].cpu().numpy()
    np.testing.assert_allclose(lam, a['sv'], rtol=0, atol=1e-5 * lam[0])
    assert abs(float(torch.real(torch.trace(T))) - meta['trace']) < 1e-5 * meta['trace']


def test_floquet_optimized_form(oi, report):
    meta, a = load('floquet')

    class Nm:
        pass
    nm = Nm()
    for k in ('ScatterOrder_X', 'ScatterOrder_Y', 'ScatterGrid_X', 'ScatterGrid_Y'):
        setattr(nm, k, meta[k])
    got = oi.CalculateSOCS(torch.from_numpy(a['floquet']), torch.from_numpy(a['kernels']), nm)
    report('floquet', engine_vs_reference=rel_err(got.numpy(), a['image']))
    assert rel_err(got.numpy(), a['image']) < FP32_VS_REF


def test_spectrum_api(oi):
    from opticalimaging_b200.params import Projection, Scatter, Source
    meta, a = load('spectrum')
    sc, po, sr = Scatter(), Projection(), Source()
    sc.Period_X, sc.Period_Y, sc.ScatterField = meta['Period_X'], meta['Period_Y'], torch.from_numpy(a['field'])
    po.NA, sr.Wavelength = meta['NA'], meta['Wavelength']
    hk, f, g, pim = sc.CalculateSpectrum(po, sr)
    assert rel_err(hk.numpy(), a['hk']) < 2e-6
    np.testing.assert_array_equal(f.numpy(), a['f'])
    np.testing.assert_array_equal(np.isnan(pim.numpy()), np.isnan(a['pupil']))


def test_raw_optics_nan_with_warning(oi):
    meta, a = load('raw_nan')
    sr, sc, po, nm = build(meta, a)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter('always')
        img, _ = oi.CalculateAbbeImage(sr, sc, po, nm)
    assert np.isnan(img.Intensity.numpy()).all()
    assert any(issubclass(x.category, RuntimeWarning) for x in w)


def test_batched_socs_matches_single(oi):
    """SocsKernels.image on a batch (float32 and uint8 masks) equals the per-clip drop-in call."""
    from opticalimaging_b200 import workloads as W
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=8)
    T, fg = oi.CalculateTCCMatrix(sr, [2048, 2048], po, 0.0, nm)
    sk = oi.socs_kernels_from_tcc(T, fg, [256, 256], nm)
    masks = W.manhattan_masks(5, 256, 2048.0, seed=9)
    md = torch.from_numpy(masks).cuda()
    batch = sk.image(md)
    batch_u8 = sk.image(md.to(torch.uint8))
    for i in range(5):
        sc = Scatter()
        sc.Period_X = sc.Period_Y = 2048
        sc.ScatterField = W.thin_field(masks[i])
        one, _ = oi.CalculateAerialImage_SOCS(sc, sk, sr, po)
        assert rel_err(batch[i].cpu().numpy(), one.numpy()) < 5e-6   # FFT form vs the drop-in DFT form
        assert rel_err(batch_u8[i].cpu().numpy(), one.numpy()) < 5e-6
        if i == 0:
            ref = O.socs(sc, oi.DecomposeTCC_SOCS(T, fg, [256, 256], nm).cpu().numpy().astype(np.complex128), sr, po)
            assert rel_err(one.numpy(), ref) < FP32_VS_FP64


@pytest.mark.parametrize('form', ['fft', 'dft', 'bf16x3'])
def test_packed_real_fields_match_the_kernels(oi, form):
    """Configuration-3 optics (SOCS-24, centred 59 x 59 band): the model packs the 24 kernels into 12 real-field
    pairs for real masks; float32 masks (packed fields) and the same masks as complex64 (the model's own 24
    kernels) give the same images, and both match FP64."""
    from opticalimaging_b200 import workloads as W, _native as N
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=24)
    T, fg = oi.CalculateTCCMatrix(sr, [2048, 2048], po, 0.0, nm)
    sk = oi.socs_kernels_from_tcc(T, fg, [256, 256], nm)
    assert sk.packed is not None and sk.packed[0].shape[1] == 12
    assert sk.fields_for(N.FIELD_COMPLEX_C64)[0] is sk.pupils
    masks = W.manhattan_masks(3, 256, 2048.0, seed=4)
    md = torch.from_numpy(masks).cuda()
    packed = sk.image(md, form=form).cpu().numpy()
    own = sk.image(md.to(torch.complex64).unsqueeze(-1), form=form).cpu().numpy()
    bound = FP32_VS_FP64 if form != 'bf16x3' else 1e-4
    assert rel_err(packed, own) < bound
    sc = Scatter()
    sc.Period_X = sc.Period_Y = 2048
    sc.ScatterField = W.thin_field(masks[0])
    ref = O.socs(sc, oi.DecomposeTCC_SOCS(T, fg, [256, 256], nm).cpu().numpy().astype(np.complex128), sr, po)
    assert rel_err(packed[0], ref) < bound
    assert N.device_status() == 0


@pytest.mark.parametrize('ny,nx', [(17, 23), (64, 64), (33, 40)])
def test_small_and_odd_grids_single_point(oi, ny, nx):
    """Edge cases: tiny odd grids, a single source point on axis (ideal low-pass), K=1."""
    from opticalimaging_b200.params import Numerics, Projection, Scatter, Source
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    sr.Shape, sr.PntNum = 'pixel', 3
    c = torch.linspace(-1, 1, 3)
    sr.SPointX, sr.SPointY = torch.meshgrid(c, c, indexing='ij')
    v = torch.zeros(3, 3)
    v[0, 1] = 1.0   # one off-centre point (the centre is always zeroed)
    sr.SPointValue = v
    po.NA, po.IndexImage, po.Magnification = 0.8, 1.0, 1.0
    sr.Wavelength = 200.0
    nm.ImageCalculationMode = 'scalar'
    sc.Period_X, sc.Period_Y = 10.0 * nx, 10.0 * ny
    rng = np.random.default_rng(ny * nx)
    f = np.zeros((ny, nx, 3), np.complex64)
    f[:, :, 0] = rng.random((ny, nx)) > 0.5
    sc.ScatterField = torch.from_numpy(f)
    img, _ = oi.CalculateAbbeImage(sr, sc, po, nm)
    assert rel_err(img.Intensity.numpy(), O.abbe(sr, sc, po, nm)) < FP32_VS_FP64
    nm.Hopkins_SettingType, nm.Hopkins_Order = 'order', 1
    h, _ = oi.CalculateHopkinsImage(sr, sc, po, nm)
    assert rel_err(h.Intensity.numpy(), O.hopkins(sr, sc, po, nm)) < FP32_VS_FP64


def test_clear_field_is_uniform(oi):
    """Known answer: a clear mask (h = 1) gives the uniform intensity n * sum_j w_j |P_j(0)|^2 / sum w = n."""
    from opticalimaging_b200 import workloads as W
    sr, sc, po, nm = W.config1()
    sc.ScatterField = W.thin_field(np.ones((256, 256), np.float32))
    img, _ = oi.CalculateAbbeImage(sr, sc, po, nm)
    np.testing.assert_allclose(img.Intensity.numpy(), 1.0, rtol=0, atol=5e-6)


@pytest.mark.parametrize('order,threshold', [(24, None), (None, 0.99)])
def test_gram_kernels_match_tcc_kernels(oi, order, threshold):
    """SOCS kernels from the Gram matrix of the pupil matrix (rank 3S < FG) give the same images as the
    eigendecomposition of the assembled TCC, for 'order' and 'threshold' truncation."""
    from opticalimaging_b200 import _native as N, workloads as W
    sr, po, nm = W.config3_optics(order=order or 24)
    if threshold is not None:
        nm.Hopkins_SettingType, nm.Hopkins_Threshold = 'threshold', threshold
    h, fg = oi.tcc_pupil_matrix(sr, [2048.0, 2048.0], po, 0.0, nm)   # FG = 59^2 > 3 S = 1560
    assert h.shape[0] * h.shape[2] < h.shape[1]          # the Gram path is taken
    gram = oi.socs_kernels_from_pupils(h, fg, [256, 256], nm)
    T, fg2 = oi.CalculateTCCMatrix(sr, [2048.0, 2048.0], po, 0.0, nm)
    full = oi.socs_kernels_from_tcc(T, fg2, [256, 256], nm)
    assert gram.count == full.count and gram.band == full.band
    rng = np.random.default_rng(5)
    masks = torch.from_numpy(np.stack([W.rect_mask(256, 256, 2048.0, 2048.0, 20, 30, 400, rng)
                                       for _ in range(2)])).cuda()
    a = gram.image(masks).cpu().numpy()
    b = full.image(masks).cpu().numpy()
    assert rel_err(a, b) < 2e-6
    assert N.device_status() == 0


@pytest.mark.parametrize('form,tol', [('fft', 1e-6), ('bf16x3', 5e-5)])
def test_image_host_matches_device_image(oi, form, tol):
    """image_host (pinned host masks in, pinned host images out, chunked over three streams) gives the images
    of image() on device masks: bit-identical per image for the FFT form up to float rounding of the batch split,
    within the split form's batch-composition tolerance for BF16x3; twice in a row (rotating buffer slots), with
    a ragged last chunk."""
    from opticalimaging_b200 import workloads as W
    sr, po, nm = W.config3_optics(order=24)
    T, fg = oi.CalculateTCCMatrix(sr, [512.0, 512.0], po, 0.0, nm)
    sk = oi.socs_kernels_from_tcc(T, fg, [256, 256], nm)
    masks = (np.random.default_rng(5).random((11, 256, 256)) > 0.6).astype(np.uint8)
    want = sk.image(torch.from_numpy(masks).cuda(), form=form).cpu().numpy()
    host_in = torch.from_numpy(masks).pin_memory()
    for _ in range(2):
        host_out = torch.full((11, 256, 256), float('nan')).pin_memory()
        sk.image_host(host_in, host_out, chunk=4, form=form)
        torch.cuda.current_stream().synchronize()
        got = host_out.numpy()
        assert np.isfinite(got).all()
        assert rel_err(got, want) < tol
    with pytest.raises(ValueError, match='pinned'):
        sk.image_host(torch.from_numpy(masks), torch.empty((11, 256, 256)), form=form)


def test_dropin_socs_reuses_band_form_of_reference_layout_kernels(oi):
    """CalculateAerialImage_SOCS with the [Ny, Nx, K] kernels DecomposeTCC_SOCS returned finds their band form
    once per tensor (no full-grid scan per call); an in-place change of the tensor is seen; the image is the
    same as through the band-form kernels."""
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    T, fg = oi.CalculateTCCMatrix(sr, [meta['Period_Y'], meta['Period_X']], po, meta['focus'][0], nm)
    K = oi.DecomposeTCC_SOCS(T, fg, [sc.ScatterField.shape[1], sc.ScatterField.shape[0]], nm)
    sk0 = oi._SOCS_CACHE[K][1]
    img1, _ = oi.CalculateAerialImage_SOCS(sc, K, sr, po)
    assert oi._SOCS_CACHE[K][1] is sk0
    img2, _ = oi.CalculateAerialImage_SOCS(sc, sk0, sr, po)
    np.testing.assert_array_equal(img1.numpy(), img2.numpy())
    K.mul_(2.0)                                   # the kernels change in place: the band form is found again
    img3, _ = oi.CalculateAerialImage_SOCS(sc, K, sr, po)
    assert oi._SOCS_CACHE[K][1] is not sk0
    assert rel_err(img3.numpy(), 4.0 * img1.numpy()) < 1e-6
    host = K.cpu()                                # a host copy: its own entry, scanned once
    img4, _ = oi.CalculateAerialImage_SOCS(sc, host, sr, po)
    assert host in oi._SOCS_CACHE and rel_err(img4.numpy(), img3.numpy()) < 1e-6


@pytest.mark.parametrize('form', ['dense', 'factored'])
def test_eig_topk_matches_dense_eigh(oi, form, report):
    """The library's FP64 top-K solver (oi_eig_topk64) on the configuration-3 TCC (3481 x 3481, K = 24): the
    rank-24 projector and eigenvalues against torch.linalg.eigh of the same FP64 matrix -- from the dense TCC
    and from its pupil factor h (the TCC never formed)."""
    from opticalimaging_b200 import workloads as W
    sr, po, nm = W.config3_optics(order=24)
    h, fg = oi.tcc_pupil_matrix(sr, [2048.0, 2048.0], po, 0.0, nm)
    T = torch.einsum('eps,eqs->pq', h, h.conj())
    lam, U = torch.linalg.eigh(T)
    lam, U = lam.flip(0)[:24], U.flip(1)[:, :24]
    got = oi.eig_topk(24, tcc=T) if form == 'dense' else oi.eig_topk(24, h=h)
    assert got is not None
    gl, gU = got
    P = (U @ U.conj().T).cpu().numpy()
    Pg = (gU @ gU.conj().T).cpu().numpy()
    perr = float(np.max(np.abs(Pg - P)) / np.max(np.abs(P)))
    lerr = float(torch.max(torch.abs(gl - lam)) / lam[0])
    orth = float(torch.max(torch.abs(gU.conj().T @ gU - torch.eye(24, dtype=gU.dtype, device=gU.device))))
    report(f'eig_topk_{form}', projector=perr, eigenvalues=lerr, orthonormality=orth)
    assert perr < 1e-10 and lerr < 1e-12 and orth < 1e-12


def test_eig_topk_small_and_edge_cases(oi):
    """A small TCC (vec_small, three live channels' optics), K = 12: kernels from the solver give the reference's
    SOCS image; k above the solver's range returns None (the caller takes the dense solver)."""
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    T, fg = oi.CalculateTCCMatrix(sr, [meta['Period_Y'], meta['Period_X']], po, meta['focus'][0], nm)
    if T.shape[0] >= 64:
        vals, vecs = oi.eig_topk(12, tcc=T)
        lam = torch.linalg.eigvalsh(T).flip(0)[:12]
        assert float(torch.max(torch.abs(vals - lam)) / lam[0]) < 1e-12
    assert oi.eig_topk(oi.TOPK_MAX + 1, tcc=T) is None
    img, _ = oi.CalculateHopkinsImage(sr, sc, po, nm)
    assert rel_err(img.Intensity.numpy(), a['hopkins']) < FP32_VS_REF


def test_dropin_large_host_field_through_pinned_staging(oi):
    """A 1024 x 1024 x 3 complex64 host ScatterField (24 MiB, pageable) goes through the pinned staging.  As one real
    channel it takes the real-mask path: the drop-in image is the resident kernels' image of the same mask, bit for
    bit, and the pupil image comes from the real channel's band pass; with an imaginary part in another channel
    the live channels take the complex path.  Images and pupil images come back as host tensors."""
    from opticalimaging_b200 import _native as N, workloads as W
    from opticalimaging_b200.params import Scatter
    sr, po, nm = W.config3_optics(order=8)
    T, fg = oi.CalculateTCCMatrix(sr, [2048.0, 2048.0], po, 0.0, nm)
    K = oi.DecomposeTCC_SOCS(T, fg, [1024, 1024], nm)
    mask = W.config3_masks(count=1, n=1024, seed=77)[0]
    sc = Scatter()
    sc.Period_X = sc.Period_Y = 2048.0
    sc.ScatterField = W.thin_field(mask)
    assert not sc.ScatterField.is_pinned() and sc.ScatterField.numel() * 8 >= (4 << 20)
    img, pim = oi.CalculateAerialImage_SOCS(sc, K, sr, po)
    assert img.device.type == 'cpu' and img.shape == (1024, 1024)
    sk = oi._SOCS_CACHE[K][1]
    want = sk.image(torch.from_numpy(mask).cuda()[None])[0].cpu().numpy()
    # one real channel: the image is the real-mask path's
    assert np.array_equal(img.numpy(), want)
    # the pupil image from the real channel's FFT band pass against the complex field's DFT band pass
    full = sc.ScatterField.cuda()
    ref = oi._pupil_image(sc, po, sr, full, torch.device('cuda')).cpu().numpy()
    assert pim.shape == ref.shape and pim.device.type == 'cpu'
    np.testing.assert_array_equal(np.isnan(pim.numpy()), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert rel_err(pim.numpy()[ok], ref[ok]) < 1e-5
    assert not np.any(pim.numpy()[..., 1:][ok[..., 1:]])      # the zero channels stay exactly zero
    # a field that is not one real channel (an imaginary part in channel 2): channels 0 and 2 in the complex path
    f2 = sc.ScatterField.clone()
    f2[:, :, 2] = 0.25j * f2[:, :, 0]
    sc.ScatterField = f2
    img2, pim2 = oi.CalculateAerialImage_SOCS(sc, K, sr, po)
    h2 = f2.cuda()[:, :, [0, 2]].contiguous()
    want2 = sk.image(h2[None], kind=N.FIELD_COMPLEX_C64, nch=2)[0].cpu().numpy()
    assert np.array_equal(img2.numpy(), want2)
    ref2 = oi._pupil_image(sc, po, sr, f2.cuda(), torch.device('cuda')).cpu().numpy()
    ok2 = ~np.isnan(ref2)
    np.testing.assert_array_equal(np.isnan(pim2.numpy()), ~ok2)
    assert rel_err(pim2.numpy()[ok2], ref2[ok2]) < 1e-6
    assert rel_err(img2.numpy(), 1.0625 * want) < 1e-5        # |m|^2 (1 + 1/16): the same mask, scaled intensity
