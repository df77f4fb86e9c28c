"""Pin the FP64 oracle (and the host-side parameter objects) to outputs of the reference itself.

The fixtures under tests/golden were produced by running the reference (complex64, CPU) on these inputs;
the oracle is its float64 restatement, so they agree to about the reference's own float32 rounding.
"""
import math

import numpy as np
import pytest
import torch

from oracle import optics64 as O
from opticalimaging_b200.params import Projection, Source
from tests.fixtures import build, load, make_source, rel_err

SOURCE_CASES = ['annular21', 'quasar31', 'annular41', 'dipole25', 'multipole25', 'annular21_psf', 'default81']


@pytest.mark.parametrize('name', SOURCE_CASES)
def test_source_points_bit_exact(name):
    meta, a = load('sources')
    sr = make_source(meta[name])
    X, Y, V = O.source_points(sr)
    np.testing.assert_array_equal(X, a[name + '_X'])
    np.testing.assert_array_equal(Y, a[name + '_Y'])
    np.testing.assert_allclose(V, a[name + '_V'], rtol=2e-7, atol=0)
    # the engine's host-side Source is bit-identical to the reference
    d = sr.Calc_SourceSimple()
    np.testing.assert_array_equal(d.X.numpy(), a[name + '_X'])
    np.testing.assert_array_equal(d.Y.numpy(), a[name + '_Y'])
    np.testing.assert_array_equal(d.Value.numpy(), a[name + '_V'])


def test_pixel_source():
    meta, a = load('sources')
    sr = make_source(meta['pixel9'])
    c = torch.linspace(-1, 1, 9)
    sr.SPointX, sr.SPointY = torch.meshgrid(c, c, indexing='ij')
    sr.SPointValue = torch.from_numpy(a['pixel9_SPointValue'])
    d = sr.Calc_SourceSimple()
    np.testing.assert_array_equal(d.X.numpy(), a['pixel9_X'])
    np.testing.assert_array_equal(d.Value.numpy(), a['pixel9_V'])
    X, Y, V = O.source_points(sr)
    np.testing.assert_array_equal(X, a['pixel9_X'])
    np.testing.assert_array_equal(V, a['pixel9_V'])


def test_source_errors_match_reference():
    sr = Source()
    sr.Shape = 'hexapole'
    with pytest.raises(ValueError, match='unsupported illumination'):
        sr.Calc_SourceSimple()
    sr.Shape, sr.OpenAngle = 'quasar', 2.0
    with pytest.raises(ValueError, match='open angle'):
        sr.Calc_SourceSimple()
    sr.Shape, sr.PntNum = 'pixel', 5
    with pytest.raises(ValueError, match='Matrix Size X'):
        sr.Calc_SourceSimple()


def test_zernike_and_char_matrix():
    _, a = load('zernike_char')
    ab = O.aberration(a['coef'], a['rho'].astype(np.float64), a['theta'].astype(np.float64))
    np.testing.assert_allclose(ab, a["aberration"], rtol=0, atol=1e-5)  # fp32 cancellation in Z37
    po = Projection()
    po.Aberration_Zernike = torch.from_numpy(a['coef'])
    host = po.CalculateAberrationFast(torch.from_numpy(a['rho']), torch.from_numpy(a['theta']), 0)
    np.testing.assert_allclose(host.numpy(), a['aberration'], rtol=0, atol=1e-5)
    np.testing.assert_allclose(Projection.RotateAngle(torch.from_numpy(a['coef']), 0.4).numpy(), a['rotated'],
                               rtol=0, atol=1e-6)
    m = O.char_matrix(a['f'].astype(np.float64), a['g'].astype(np.float64), 0.9375, 1.0)
    for got, key in zip((m[0], m[1], m[3], m[4], m[5]), ('mxx', 'myx', 'myy', 'mxz', 'myz')):
        np.testing.assert_allclose(got, a[key], rtol=0, atol=2e-6)


def test_spectrum():
    meta, a = load('spectrum')

    class P:
        pass
    sc, po, sr = P(), P(), P()
    sc.ScatterField, sc.Period_X, sc.Period_Y = a['field'], meta['Period_X'], meta['Period_Y']
    po.NA, sr.Wavelength = meta['NA'], meta['Wavelength']
    hk, f, g = O.spectrum(sc, po, sr)
    assert rel_err(hk, a['hk']) < 2e-6
    np.testing.assert_array_equal(f, a['f'])
    np.testing.assert_array_equal(g, a['g'])
    _, _, npx, npy = O.freq_axes(sc, po, sr)
    pim = O.pupil_image(hk, f, g, npx, npy)
    np.testing.assert_array_equal(np.isnan(pim), np.isnan(a['pupil']))
    ok = ~np.isnan(a['pupil'])
    assert np.max(np.abs(pim[ok] - a['pupil'][ok])) < 2e-6 * np.max(np.abs(a['pupil'][ok]))


@pytest.mark.parametrize('name', ['cfg1', 'vec_small', 'odd_scalar', 'cfg2_small'])
def test_abbe(name):
    meta, a = load(name)
    sr, sc, po, nm = build(meta, a)
    img = O.abbe(sr, sc, po, nm)
    assert img.shape == a['abbe'].shape
    assert rel_err(img, a['abbe']) < 1e-5
    for z in range(img.shape[0]):   # every focus plane on its own
        assert rel_err(img[z], a['abbe'][z]) < 1e-5


def test_raw_optics_are_nan_in_reference_and_oracle():
    meta, a = load('raw_nan')
    assert np.isnan(a['abbe']).all()
    sr, sc, po, nm = build(meta, a)
    assert np.isnan(O.abbe(sr, sc, po, nm)).all()


def test_tcc_and_socs_vector():
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    T, fg = O.tcc(sr, [meta['Period_Y'], meta['Period_X']], po, meta['focus'][0], nm)
    assert list(fg) == list(a['fg'])
    assert rel_err(T, a['tcc']) < 2e-6
    lam = np.linalg.eigvalsh(T)[::-1]
    np.testing.assert_allclose(lam[:40], a['tcc_sv'][:40], rtol=0, atol=2e-6 * lam[0])
    # SOCS image from the reference's own kernels: isolates the imaging step from the eigensolver
    I_ref_kernels = O.socs(sc, a['kernels'].astype(np.complex128), sr, po)
    assert rel_err(I_ref_kernels, a['socs']) < 1e-5
    # and from the oracle's FP64 kernels: same image, since K=12 sits at an eigenvalue gap
    K = O.decompose(T, fg, [sc.ScatterField.shape[1], sc.ScatterField.shape[0]], nm)
    assert K.shape == a['kernels'].shape
    assert rel_err(O.socs(sc, K, sr, po), a['socs']) < 1e-5
    assert rel_err(O.hopkins(sr, sc, po, nm), a['hopkins']) < 1e-5


def test_hopkins_odd_grid_matches_reference_quirk():
    """On odd grids the reference embeds SOCS kernels with fftshift (DecomposeTCC_SOCS.py:31), which puts
    frequency k at index k-1; its Hopkins image then differs from its Abbe image.  The oracle follows it."""
    meta, a = load('odd_scalar')
    sr, sc, po, nm = build(meta, a)
    h = O.hopkins(sr, sc, po, nm)
    assert rel_err(h, a['hopkins']) < 1e-5
    assert rel_err(a['hopkins'], a['abbe']) > 1e-2


@pytest.mark.parametrize('ny,nx,py,px', [(44, 62, 440, 620), (40, 48, 400, 480)])
def test_hopkins_full_order_equals_abbe_even_grid(ny, nx, py, px):
    meta, a = load('odd_scalar')
    sr, sc, po, nm = build(meta, a)
    nm.Hopkins_Order = 10 ** 6
    f = np.zeros((ny, nx, 3), np.complex64)
    f[:, :, 0] = np.random.default_rng(0).random((ny, nx)) > 0.5
    sc.ScatterField, sc.Period_Y, sc.Period_X = torch.from_numpy(f), py, px
    assert rel_err(O.hopkins(sr, sc, po, nm), O.abbe(sr, sc, po, nm)) < 1e-6  # order caps at FG-1


@pytest.mark.slow
def test_cfg3_small_socs24():
    meta, a = load('cfg3_small')
    sr, sc, po, nm = build(meta, a)
    T, fg = O.tcc(sr, [meta['Period_Y'], meta['Period_X']], po, 0.0, nm)
    lam = np.linalg.eigvalsh(T)[::-1]
    np.testing.assert_allclose(lam[:64], a["tcc_sv"][:64], rtol=0, atol=1e-5 * lam[0])  # complex64 SVD
    K = O.decompose(T, fg, [256, 256], nm)
    assert rel_err(O.socs(sc, K, sr, po), a['socs']) < 1e-5


def test_cfg3_tcc_spectrum_pinned():
    meta, a = load('cfg3_tcc')
    assert list(meta['fg']) == [59, 59]
    assert a['sv'][23] / a['sv'][0] > 1.02 * a['sv'][24] / a['sv'][0]  # the K=24 cut sits at a gap


def test_socs_floquet():
    meta, a = load('floquet')

    class N:
        pass
    nm = N()
    for k in ('ScatterOrder_X', 'ScatterOrder_Y', 'ScatterGrid_X', 'ScatterGrid_Y'):
        setattr(nm, k, meta[k])
    I = O.socs_floquet(a['floquet'], a['kernels'].astype(np.complex128), nm)
    assert rel_err(I, a['image']) < 1e-5


def test_threshold_mode_counts_energy():
    class N:
        Hopkins_SettingType, Hopkins_Threshold = 'threshold', 0.9
    lam = np.array([5.0, 3.0, 1.0, 0.5, 0.5])
    assert O.socs_count(N, lam, 5) == 3   # 5+3+1 = 9 >= 0.9*10
    N.Hopkins_SettingType = 'bogus'
    with pytest.raises(ValueError):
        O.socs_count(N, lam, 5)
    assert math.isclose(float(np.sum(lam)), 10.0)


def test_cfg4_resist_gradient_matches_reference_autograd():
    """Configuration 4 at its own size (1024^2, the reference's SOCS-16 kernels, sigmoid(N(0,1)) mask, a = 50
    resist loss): the FP64 image, loss and exact gradient against the reference's complex64 forward and its
    torch-autograd gradient at 4096 seeded pixels.  The bounds are the reference's own complex64 rounding at
    this size (measured: image 5.7e-5 of peak, loss 1.8e-4 relative, gradient 4.4e-4 of its maximum)."""
    from opticalimaging_b200 import workloads as W
    from tests.fixtures import cfg4_kernels
    meta, a = load('autograd_cfg4')
    _, _, _, logits, target = W.config4(seed=meta['seed'], n=meta['n'], order=meta['order'])
    I, L, G = O.socs_resist(logits, target, cfg4_kernels(meta, a), meta['a'], meta['thr'])
    px = a['pixels']
    assert np.max(np.abs(I[px[:, 0], px[:, 1]] - a['image_at'])) < 1e-4 * float(a['image_peak'])
    assert abs(L - float(a['loss'])) < 5e-4 * float(a['loss'])
    assert np.max(np.abs(G[px[:, 0], px[:, 1]] - a['grad_at'])) < 1e-3 * float(a['grad_maxabs'])


def test_cfg4_gradient_matches_central_differences():
    """The FP64 gradient against central finite differences (h = 1e-3) of the FP64 loss on 8 pixels, each
    difference from the exact single-pixel update of the SOCS fields (socs_pixel_fields)."""
    from opticalimaging_b200 import workloads as W
    from tests.fixtures import cfg4_kernels
    meta, a = load('autograd_cfg4')
    n, A, thr = meta['n'], meta['a'], meta['thr']
    _, _, _, logits, target = W.config4(seed=meta['seed'], n=n, order=meta['order'])
    K = cfg4_kernels(meta, a)
    _, _, G = O.socs_resist(logits, target, K, A, thr)
    fd = cfg4_central_differences(logits, target, K, A, thr, [tuple(p) for p in a['pixels'][:8]])
    got = np.array([G[tuple(p)] for p in a['pixels'][:8]])
    assert np.max(np.abs(got - fd)) < 1e-6 * np.max(np.abs(G))


def cfg4_central_differences(logits, target, K, A, thr, pixels, h=1e-3):
    """Central differences (h in the logits) of the FP64 resist loss at `pixels`, from the single-pixel field
    update E_k + delta roll(F_k, q), q the ifftshift image of the pixel."""
    n = logits.shape[0]
    lg = logits.astype(np.float64)
    t = 1.0 / (1.0 + np.exp(-lg))
    d = O._ifft2(np.fft.ifftshift(t))
    E = [O._fft2(K[:, :, k] * d) for k in range(K.shape[2])]
    F = O.socs_pixel_fields(K)

    def loss(p, dl):
        dt = 1.0 / (1.0 + np.exp(-(lg[p] + dl))) - t[p]
        q = ((p[0] + n // 2) % n, (p[1] + n // 2) % n)
        acc = np.zeros((n, n))
        for e, f in zip(E, F):
            x = e + dt * np.roll(f, q, axis=(0, 1))
            acc += x.real ** 2 + x.imag ** 2
        s = 1.0 / (1.0 + np.exp(-A * (np.fft.fftshift(acc) - thr)))
        return float(np.sum((s - target) ** 2))
    return np.array([(loss(p, h) - loss(p, -h)) / (2 * h) for p in pixels])


def test_cpu_reference_arm_matches_the_reference():
    """The reference arm of the benchmark (oracle/cpu_reference.socs_clip: the reference's SOCS algorithm with
    torch's CPU FFTs on complex64) reproduces the reference's own SOCS image from the reference's kernels, and
    its host-built kernels (socs_kernels) give the reference's configuration-3 image at 256^2."""
    from oracle import cpu_reference as R
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    npx = meta['Period_X'] / (sr.Wavelength / po.NA)
    npy = meta['Period_Y'] / (sr.Wavelength / po.NA)
    img = R.socs_clip(a['field'], a['kernels'], npx, npy, 2)
    assert rel_err(img, a['socs']) < 2e-6
    meta, a = load('cfg3_small')
    sr, sc, po, nm = build(meta, a)
    K = R.socs_kernels(sr, po, nm, [meta['Period_Y'], meta['Period_X']], [256, 256])
    assert K.shape == (256, 256, 24) and K.dtype == np.complex64
    npx = meta['Period_X'] / (sr.Wavelength / po.NA)
    img = R.socs_clip(a['field'], K, npx, npx, 2)
    assert rel_err(img, a['socs']) < 2e-5
