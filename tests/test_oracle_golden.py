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


@pytest.mark.parametrize('name', ['cfg1', 'vec_small', 'odd_scalar'])
def test_abbe(name):
    meta, a = load(name)
    sr, sc, po, nm = build(meta, a)
    img = O.abbe(sr, sc, po, nm)
    assert img.shape == a['abbe'].shape
    assert rel_err(img, a['abbe']) < 1e-5


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
