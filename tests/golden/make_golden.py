"""Generate golden fixtures by running the reference implementation itself.

Run in a container that holds the reference sources (it imports them from ``REFERENCE_DIR``):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [REFERENCE_DIR [CASE ...]]

Writes ``tests/golden/ref_<case>.npz`` (every case, or only the CASEs named) plus ``manifest.json``.  Each fixture stores the inputs and the
reference's outputs, so the tests replay the same inputs through the oracle and the engine without needing
the reference at run time.  The reference's matplotlib-importing drivers are not imported, and its RCWA
solver is not constructed.

Optics: every imaging case uses the immersion-mapped optics (wavelength/n, NA/n, IndexImage 1,
Magnification 1), because the reference returns NaN at the literal immersion optics; one case records that
NaN behaviour.
"""
import json
import math
import os
import sys
import time

import numpy as np
import torch

REF = sys.argv[1] if len(sys.argv) > 1 else '/root/reference'
sys.path.insert(0, REF)
sys.dont_write_bytecode = True

from Source import Source  # noqa: E402
from Projection import Projection  # noqa: E402
from Numerics import Numerics  # noqa: E402
from Scatter import Scatter  # noqa: E402
from CalculateAerialImage import CalculateAbbeImage, CalculateHopkinsImage  # noqa: E402
from CalculateTCCMatrix import CalculateTCCMatrix  # noqa: E402
from DecomposeTCC_SOCS import DecomposeTCC_SOCS  # noqa: E402
from CalculateAerialImage_SOCS import CalculateAerialImage_SOCS, CalculateSOCS  # noqa: E402
from CalculateCharacteristicMatrix import CalculateCharacteristicMatrix  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
LAM, NA, N_IMG = 193.0, 1.35, 1.44
torch.set_num_threads(min(8, os.cpu_count() or 1))


def mapped(po, sr):
    sr.Wavelength = LAM / N_IMG
    po.NA = NA / N_IMG
    po.IndexImage = 1.0
    po.Magnification = 1.0


def rect_mask(ny, nx, period_y, period_x, nrect, lo, hi, seed):
    """Binary mask from seeded axis-aligned rectangles (sizes in nm, positions uniform over the period)."""
    g = np.random.default_rng(seed)
    t = np.zeros((ny, nx), dtype=np.float32)
    yy = (np.arange(ny) + 0.5) * period_y / ny
    xx = (np.arange(nx) + 0.5) * period_x / nx
    for _ in range(nrect):
        w, h = g.uniform(lo, hi, 2)
        x0, y0 = g.uniform(0, period_x), g.uniform(0, period_y)
        t[np.ix_((yy >= y0) & (yy < y0 + h), (xx >= x0) & (xx < x0 + w))] = 1
    return t


def src_arrays(sr):
    d = sr.Calc_SourceSimple()
    return d.X.numpy().copy(), d.Y.numpy().copy(), d.Value.numpy().copy()


def src_params(sr):
    keys = ['PntNum', 'Wavelength', 'Shape', 'SigmaOut', 'SigmaIn', 'SigmaCenter', 'SigmaRadius', 'OpenAngle',
            'RotateAngle', 'PoleNumber', 'PSFEnable', 'PSFSigma']
    d = {k: getattr(sr, k) for k in keys}
    d['PolarizationVector'] = [complex(v) for v in sr.PolarizationVector]
    return d


def save(name, meta, **arrays):
    np.savez_compressed(os.path.join(OUT, f'ref_{name}.npz'), meta=json.dumps(meta, default=str), **arrays)
    print(f'  {name}: ' + ', '.join(f'{k}{tuple(np.shape(v))}' for k, v in arrays.items()))


def case_sources():
    specs = {
        'annular21': dict(Shape='annular', PntNum=21, SigmaIn=0.6, SigmaOut=0.9),
        'quasar31': dict(Shape='quasar', PntNum=31, SigmaIn=0.5, SigmaOut=0.85, OpenAngle=math.pi / 6),
        'annular41': dict(Shape='annular', PntNum=41, SigmaIn=0.7, SigmaOut=0.95),
        'dipole25': dict(Shape='dipolecirc', PntNum=25, SigmaIn=0.3, SigmaOut=0.8, OpenAngle=math.pi / 4,
                         RotateAngle=0.3),
        'multipole25': dict(Shape='multipole', PntNum=25, SigmaCenter=0.6, SigmaRadius=0.15, PoleNumber=4,
                            RotateAngle=0.2),
        'annular21_psf': dict(Shape='annular', PntNum=21, SigmaIn=0.3, SigmaOut=0.7, PSFEnable=True,
                              PSFSigma=0.05),
        'default81': dict(),
    }
    out = {}
    for name, kw in specs.items():
        sr = Source()
        for k, v in kw.items():
            setattr(sr, k, v)
        X, Y, V = src_arrays(sr)
        out[name] = (src_params(sr), X, Y, V)
    arrays = {}
    meta = {}
    for name, (p, X, Y, V) in out.items():
        meta[name] = p
        arrays[name + '_X'], arrays[name + '_Y'], arrays[name + '_V'] = X, Y, V
    # a pixel source given as a 2-D map
    sr = Source()
    sr.Shape = 'pixel'
    sr.PntNum = 9
    c = torch.linspace(-1, 1, 9)
    sr.SPointX, sr.SPointY = torch.meshgrid(c, c, indexing='ij')
    sr.SPointValue = torch.rand(9, 9, generator=torch.Generator().manual_seed(5))
    X, Y, V = src_arrays(sr)
    meta['pixel9'] = src_params(sr)
    arrays.update(pixel9_X=X, pixel9_Y=Y, pixel9_V=V, pixel9_SPointValue=sr.SPointValue.numpy())
    save('sources', meta, **arrays)


def case_zernike_char():
    g = torch.Generator().manual_seed(11)
    po = Projection()
    po.Aberration_Zernike = 0.05 * torch.randn(37, generator=g)
    rho = torch.rand(200, generator=g)
    theta = (torch.rand(200, generator=g) * 2 - 1) * math.pi
    ab = po.CalculateAberrationFast(rho, theta, 0)
    rot = Projection.RotateAngle(po.Aberration_Zernike, 0.4)
    f = (torch.rand(64, generator=g) * 2 - 1) * 1.3
    gg = (torch.rand(64, generator=g) * 2 - 1) * 1.3
    m = CalculateCharacteristicMatrix(f, gg, 0.9375, 1.0)
    save('zernike_char', {}, coef=po.Aberration_Zernike.numpy(), rho=rho.numpy(), theta=theta.numpy(),
         aberration=ab.numpy(), rotated=rot.numpy(), f=f.numpy(), g=gg.numpy(),
         mxx=m[0].numpy(), myx=m[1].numpy(), myy=m[3].numpy(), mxz=m[4].numpy(), myz=m[5].numpy())


def case_spectrum():
    g = torch.Generator().manual_seed(3)
    h = torch.complex(torch.randn(21, 16, 3, generator=g), torch.randn(21, 16, 3, generator=g))
    sc, po, sr = Scatter(), Projection(), Source()
    mapped(po, sr)
    sc.Period_X, sc.Period_Y, sc.ScatterField = 320, 420, h
    hk, f, gg, pim = sc.CalculateSpectrum(po, sr)
    save('spectrum', dict(Period_X=320, Period_Y=420, Wavelength=sr.Wavelength, NA=po.NA),
         field=h.numpy(), hk=hk.numpy(), f=f.numpy(), g=gg.numpy(), pupil=pim.numpy())


def imaging_case(name, *, ny, nx, period_y, period_x, src, vector, focus, zernike_sigma, channels, seed,
                 hopkins_order=None, pol=(1.0, 0.0), raw=False, abbe=True, keep_tcc=False, keep_kernels=False,
                 rects=None):
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    for k, v in src.items():
        setattr(sr, k, v)
    if raw:
        sr.Wavelength, po.NA, po.IndexImage, po.Magnification = LAM, NA, N_IMG, 0.25
    else:
        mapped(po, sr)
    sr.PolarizationVector = list(pol)
    nm.ImageCalculationMode = 'vector' if vector else 'scalar'
    po.FocusRange = torch.tensor(focus)
    gz = torch.Generator().manual_seed(seed + 100)
    z = torch.zeros(37)
    if zernike_sigma:
        z[4:] = zernike_sigma * torch.randn(33, generator=gz)
    po.Aberration_Zernike = z
    nrect, lo, hi = rects or (10, 0.05 * min(period_x, period_y), 0.4 * min(period_x, period_y))
    t = rect_mask(ny, nx, period_y, period_x, nrect, lo, hi, seed)
    field = np.zeros((ny, nx, 3), dtype=np.complex64)
    field[:, :, 0] = t
    if channels > 1:
        rng = np.random.default_rng(seed + 7)
        for c in range(1, channels):
            field[:, :, c] = (0.3 * rng.standard_normal((ny, nx)) + 0.2j * rng.standard_normal((ny, nx))) * t
    sc.Period_X, sc.Period_Y, sc.ScatterField = period_x, period_y, torch.from_numpy(field)
    meta = dict(src=src_params(sr), Period_X=period_x, Period_Y=period_y, vector=vector, focus=list(focus),
                NA=po.NA, IndexImage=po.IndexImage, Magnification=po.Magnification, raw=raw)
    arrays = dict(field=field, zernike=z.numpy())
    t0 = time.time()
    if abbe:
        img, pim = CalculateAbbeImage(sr, sc, po, nm)
        arrays['abbe'] = img.Intensity.numpy()
        arrays['abbe_pupil'] = pim.numpy()
    if hopkins_order is not None:
        nm.Hopkins_SettingType = 'order'
        nm.Hopkins_Order = hopkins_order
        meta['hopkins_order'] = hopkins_order
        T, fg = CalculateTCCMatrix(sr, [period_y, period_x], po, float(focus[0]), nm)
        K = DecomposeTCC_SOCS(T, fg, [nx, ny], nm)
        I, _ = CalculateAerialImage_SOCS(sc, K, sr, po)
        S = torch.linalg.svdvals(T)
        arrays.update(socs=I.numpy(), tcc_sv=S.numpy(), fg=np.array(fg))
        if keep_kernels:
            arrays['kernels'] = K.numpy()
        if keep_tcc:
            arrays['tcc'] = T.numpy()
        hk = CalculateHopkinsImage(sr, sc, po, nm)[0].Intensity
        arrays['hopkins'] = hk.numpy()
    meta['seconds'] = time.time() - t0
    save(name, meta, **arrays)


def case_autograd():
    """d loss / d logits through the reference's SOCS image, by torch autograd."""
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut = 'annular', 11, 0.6, 0.9
    mapped(po, sr)
    nm.ImageCalculationMode = 'vector'
    nm.Hopkins_SettingType, nm.Hopkins_Order = 'order', 8
    ny, nx, py, px = 40, 48, 400, 480
    T, fg = CalculateTCCMatrix(sr, [py, px], po, 0.0, nm)
    K = DecomposeTCC_SOCS(T, fg, [nx, ny], nm)
    g = torch.Generator().manual_seed(21)
    logits = torch.randn(ny, nx, generator=g, requires_grad=True)
    target = torch.from_numpy(rect_mask(ny, nx, py, px, 6, 40, 160, 22))
    mask = torch.sigmoid(logits)
    z = torch.zeros_like(mask)
    sc.Period_X, sc.Period_Y = px, py
    sc.ScatterField = torch.stack((mask, z, z), 2)
    I, _ = CalculateAerialImage_SOCS(sc, K, sr, po)
    loss = torch.sum((torch.sigmoid(50.0 * (I - 0.25)) - target) ** 2)
    loss.backward()
    save('autograd', dict(src=src_params(sr), Period_X=px, Period_Y=py, a=50.0, thr=0.25, order=8),
         logits=logits.detach().numpy(), target=target.numpy(), kernels=K.detach().numpy(),
         image=I.detach().numpy(), loss=np.array(loss.item()), grad=logits.grad.numpy())


def case_floquet():
    sr, po, nm = Source(), Projection(), Numerics()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut = 'annular', 11, 0.5, 0.8
    mapped(po, sr)
    nm.ImageCalculationMode = 'scalar'
    nm.Hopkins_SettingType, nm.Hopkins_Order = 'order', 6
    nm.ScatterOrder_X, nm.ScatterOrder_Y, nm.ScatterGrid_X, nm.ScatterGrid_Y = 8, 7, 24, 20
    g = torch.Generator().manual_seed(31)
    fm = torch.complex(torch.randn(17, 15, 3, generator=g), torch.randn(17, 15, 3, generator=g))
    T, fg = CalculateTCCMatrix(sr, [400, 480], po, 0.0, nm)
    K = DecomposeTCC_SOCS(T, fg, [17, 15], nm)
    I = CalculateSOCS(fm, K, nm)
    save('floquet', dict(src=src_params(sr), Period_X=480, Period_Y=400, ScatterOrder_X=8, ScatterOrder_Y=7,
                         ScatterGrid_X=24, ScatterGrid_Y=20, order=6),
         floquet=fm.numpy(), kernels=K.numpy(), image=I.numpy())


def case_cfg3_tcc_spectrum():
    """Leading TCC singular values of the 2048 nm vector annular 0.7/0.95 (PntNum 41) system."""
    sr, po, nm = Source(), Projection(), Numerics()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut = 'annular', 41, 0.7, 0.95
    mapped(po, sr)
    nm.ImageCalculationMode = 'vector'
    T, fg = CalculateTCCMatrix(sr, [2048, 2048], po, 0.0, nm)
    S = torch.linalg.svdvals(T)
    save('cfg3_tcc', dict(src=src_params(sr), Period=2048, fg=fg, trace=float(torch.real(torch.trace(T)))),
         sv=S[:64].numpy(), diag=torch.real(torch.diagonal(T)).numpy())


def line_space_mask(n, period, seed, line=45.0, pitch=90.0, ncuts=3):
    """Vertical lines (`line` nm at `pitch` nm) with `ncuts` seeded rectangular cuts of 40-200 nm."""
    g = np.random.default_rng(seed)
    xx = (np.arange(n) + 0.5) * period / n
    t = np.repeat(((xx % pitch) < line).astype(np.float32)[None, :], n, axis=0)
    yy = (np.arange(n) + 0.5) * period / n
    for _ in range(ncuts):
        w, h = g.uniform(40.0, 200.0, 2)
        x0, y0 = g.uniform(0, period, 2)
        t[np.ix_((yy >= y0) & (yy < y0 + h), (xx >= x0) & (xx < x0 + w))] = 0
    return t


def case_cfg2_small():
    """Configuration 2 at a quarter of its period (512 nm at its 4 nm/pixel, 128 x 128): vector Abbe, x_pol,
    quasar 0.5/0.85/30 deg PntNum 31, five focus planes -60..60 nm, Zernike Z5-Z37 ~ N(0, 0.01) waves, 45/90 nm
    lines with seeded cuts."""
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut, sr.OpenAngle = 'quasar', 31, 0.5, 0.85, math.pi / 6
    sr.PolarizationVector = [1.0, 0.0]
    mapped(po, sr)
    nm.ImageCalculationMode = 'vector'
    focus = [-60.0, -30.0, 0.0, 30.0, 60.0]
    po.FocusRange = torch.tensor(focus)
    z = torch.zeros(37)
    z[4:] = 0.01 * torch.randn(33, generator=torch.Generator().manual_seed(1202))
    po.Aberration_Zernike = z
    n, period = 128, 512
    field = np.zeros((n, n, 3), dtype=np.complex64)
    field[:, :, 0] = line_space_mask(n, period, 202)
    sc.Period_X = sc.Period_Y = period
    sc.ScatterField = torch.from_numpy(field)
    t0 = time.time()
    img, pim = CalculateAbbeImage(sr, sc, po, nm)
    meta = dict(src=src_params(sr), Period_X=period, Period_Y=period, vector=True, focus=focus, NA=po.NA,
                IndexImage=po.IndexImage, Magnification=po.Magnification, raw=False, seconds=time.time() - t0)
    save('cfg2_small', meta, field=field, zernike=z.numpy(), abbe=img.Intensity.numpy(), abbe_pupil=pim.numpy())


def case_autograd_cfg4():
    """Configuration 4 at its own size through the reference, by torch autograd: SOCS-16 kernels of the vector
    annular 0.7/0.95 (PntNum 41) system at 2048 nm, a 1024 x 1024 mask sigmoid(logits) with seeded N(0, 1)
    logits, loss ||sigmoid(50 (I - 0.25)) - target||^2 against a seeded rectangle target.  Inputs come from
    opticalimaging_b200.workloads.config4 (regenerated by the tests from the seed); the fixture keeps the
    reference's kernels on their band, its loss, and its image and gradient at 4096 seeded pixels."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(OUT)))
    from opticalimaging_b200 import workloads as Wl
    _, _, _, logits_np, target_np = Wl.config4()
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut = 'annular', 41, 0.7, 0.95
    mapped(po, sr)
    nm.ImageCalculationMode = 'vector'
    nm.Hopkins_SettingType, nm.Hopkins_Order = 'order', 16
    n, period = 1024, 2048
    t0 = time.time()
    T, fg = CalculateTCCMatrix(sr, [period, period], po, 0.0, nm)
    K = DecomposeTCC_SOCS(T, fg, [n, n], nm)
    logits = torch.from_numpy(logits_np).requires_grad_(True)
    target = torch.from_numpy(target_np)
    mask = torch.sigmoid(logits)
    zz = torch.zeros_like(mask)
    sc.Period_X = sc.Period_Y = period
    sc.ScatterField = torch.stack((mask, zz, zz), 2)
    I, _ = CalculateAerialImage_SOCS(sc, K, sr, po)
    loss = torch.sum((torch.sigmoid(50.0 * (I - 0.25)) - target) ** 2)
    loss.backward()
    nz = (K != 0).any(dim=2)
    rows = torch.nonzero(nz.any(dim=1)).flatten().numpy()
    cols = torch.nonzero(nz.any(dim=0)).flatten().numpy()
    kb = K.detach()[rows][:, cols]                          # [len rows, len cols, 16] (cyclic index lists kept)
    pix = np.random.default_rng(404).integers(0, n, size=(4096, 2))
    img = I.detach().numpy()
    grad = logits.grad.numpy()
    save('autograd_cfg4', dict(src=src_params(sr), Period_X=period, Period_Y=period, a=50.0, thr=0.25, order=16,
                               n=n, seed=4, seconds=time.time() - t0),
         kernel_rows=rows, kernel_cols=cols, kernels_band=kb.numpy(), loss=np.array(loss.item()),
         pixels=pix, image_at=img[pix[:, 0], pix[:, 1]], grad_at=grad[pix[:, 0], pix[:, 1]],
         image_peak=np.array(float(img.max())), grad_maxabs=np.array(float(np.abs(grad).max())))


CASES = ('sources', 'zernike_char', 'spectrum', 'cfg1', 'vec_small', 'odd_scalar', 'cfg3_small', 'raw_nan',
         'autograd', 'floquet', 'cfg3_tcc', 'cfg2_small', 'autograd_cfg4')


def main(only=None):
    t0 = time.time()
    print('reference fixtures ->', OUT)
    want = set(CASES if not only else only)
    if 'cfg2_small' in want:
        case_cfg2_small()
    if 'autograd_cfg4' in want:
        case_autograd_cfg4()
    if want <= {'cfg2_small', 'autograd_cfg4'}:
        print('done in %.1f s' % (time.time() - t0))
        return
    case_sources()
    case_zernike_char()
    case_spectrum()
    # configuration 1 at its own size: scalar Abbe, 1024 nm, 256x256, annular 0.6/0.9, PntNum 21
    imaging_case('cfg1', ny=256, nx=256, period_y=1024, period_x=1024,
                 src=dict(Shape='annular', PntNum=21, SigmaIn=0.6, SigmaOut=0.9), vector=False, focus=[0.0],
                 zernike_sigma=0.0, channels=1, seed=1, rects=(12, 40.0, 300.0))
    # small non-square vector Abbe + Hopkins with three live channels, focus planes, Zernike, complex Jones
    imaging_case('vec_small', ny=40, nx=48, period_y=400, period_x=480,
                 src=dict(Shape='quasar', PntNum=15, SigmaIn=0.5, SigmaOut=0.85, OpenAngle=math.pi / 6),
                 vector=True, focus=[-60.0, 0.0, 60.0], zernike_sigma=0.01, channels=3, seed=2,
                 hopkins_order=12, pol=(0.6, 0.8j), keep_tcc=True, keep_kernels=True)
    # odd-sized scalar case with defocus: Abbe and Hopkins, full order
    imaging_case('odd_scalar', ny=45, nx=63, period_y=450, period_x=630,
                 src=dict(Shape='annular', PntNum=13, SigmaIn=0.3, SigmaOut=0.8), vector=False, focus=[40.0],
                 zernike_sigma=0.02, channels=1, seed=3, hopkins_order=10000)
    # configuration-3 optics on a coarser grid (2048 nm at 8 nm/pixel): SOCS-24 with the reference's kernels
    imaging_case('cfg3_small', ny=256, nx=256, period_y=2048, period_x=2048,
                 src=dict(Shape='annular', PntNum=41, SigmaIn=0.7, SigmaOut=0.95), vector=True, focus=[0.0],
                 zernike_sigma=0.0, channels=1, seed=4, hopkins_order=24, abbe=False)
    # the literal immersion optics: the reference returns NaN
    imaging_case('raw_nan', ny=64, nx=64, period_y=512, period_x=512,
                 src=dict(Shape='annular', PntNum=11, SigmaIn=0.6, SigmaOut=0.9), vector=False, focus=[0.0],
                 zernike_sigma=0.0, channels=1, seed=5, raw=True)
    case_autograd()
    case_floquet()
    case_cfg3_tcc_spectrum()
    with open(os.path.join(OUT, 'manifest.json'), 'w') as fh:
        json.dump(dict(torch=torch.__version__, numpy=np.__version__, threads=torch.get_num_threads(),
                       seconds=round(time.time() - t0, 1)), fh, indent=1)
    print('done in %.1f s' % (time.time() - t0))


if __name__ == '__main__':
    main([a for a in sys.argv[2:]])
