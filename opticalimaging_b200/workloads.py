"""Seeded synthetic workloads with the shapes of the five benchmark configurations.

No public dataset is involved: every mask is generated from a seed.  Optics use the immersion mapping
(wavelength/n, NA/n, IndexImage 1, Magnification 1) because the reference's formulas return NaN at the
literal immersion values (NA 1.35 > 1); the mapping keeps the normalised pitch P*NA/lambda, hence the pupil
support, the band sizes and the cost, and gives the physical in-medium defocus phase and direction cosines.

  config 1  scalar Abbe, 1024 nm / 256^2, annular 0.6/0.9 PntNum 21, 12 rectangles 40-300 nm
  config 2  vector Abbe x_pol, 2048 nm / 512^2, quasar 0.5/0.85/30deg PntNum 31, 45/90 nm lines + 20 cuts,
            focus -60..60 nm (5 planes), Zernike Z5-Z37 ~ N(0, 0.01)
  config 3  SOCS-24 from the vector TCC of annular 0.7/0.95 PntNum 41, 64 clips of 1024^2 at 2 nm/pixel,
            Manhattan rectangles 30-400 nm to ~35 % fill
  config 4  SOCS-16 adjoint, 1024^2 continuous mask sigmoid(N(0,1)), rectangle target
  config 5  serving stream: Poisson arrivals, clip sizes {256,512,1024,2048}^2 at 2 nm/pixel
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .params import Numerics, Projection, Scatter, Source

LAMBDA, NA, INDEX = 193.0, 1.35, 1.44


def mapped_optics(projector: Projection, source: Source, raw: bool = False):
    """Set the immersion-mapped optics (or, with raw=True, the literal ones that the reference turns to NaN)."""
    if raw:
        source.Wavelength, projector.NA, projector.IndexImage, projector.Magnification = LAMBDA, NA, INDEX, 0.25
    else:
        source.Wavelength = LAMBDA / INDEX
        projector.NA = NA / INDEX
        projector.IndexImage = 1.0
        projector.Magnification = 1.0


def rect_mask(ny, nx, period_y, period_x, nrect, lo, hi, rng):
    """Binary mask [ny, nx] float32 from `nrect` axis-aligned rectangles (sizes U[lo, hi] nm, uniform corners)."""
    t = np.zeros((ny, nx), dtype=np.float32)
    yy = (np.arange(ny) + 0.5) * period_y / ny
    xx = (np.arange(nx) + 0.5) * period_x / nx
    for _ in range(nrect):
        w, h = rng.uniform(lo, hi, 2)
        x0, y0 = rng.uniform(0, period_x), rng.uniform(0, period_y)
        t[np.ix_((yy >= y0) & (yy < y0 + h), (xx >= x0) & (xx < x0 + w))] = 1
    return t


def manhattan_mask(n, period, lo, hi, fill, rng):
    """Binary [n, n] mask of random rectangles (sides U[lo, hi] nm) added until the fill fraction is reached."""
    t = np.zeros((n, n), dtype=np.float32)
    px = period / n
    while t.mean() < fill:
        w, h = rng.uniform(lo, hi, 2)
        x0, y0 = rng.integers(0, n, 2)
        t[y0:y0 + max(1, int(round(h / px))), x0:x0 + max(1, int(round(w / px)))] = 1
    return t


def manhattan_masks(count, n, period, seed, lo=30.0, hi=400.0, fill=0.35):
    rng = np.random.default_rng(seed)
    return np.stack([manhattan_mask(n, period, lo, hi, fill, rng) for _ in range(count)])


def line_space_mask(n, period, rng, line=45.0, pitch=90.0, ncuts=20):
    """Vertical 45 nm lines at 90 nm pitch with `ncuts` seeded rectangular cuts."""
    xx = (np.arange(n) + 0.5) * period / n
    t = np.repeat(((xx % pitch) < line).astype(np.float32)[None, :], n, axis=0)
    yy = (np.arange(n) + 0.5) * period / n
    for _ in range(ncuts):
        w, h = rng.uniform(40.0, 200.0, 2)
        x0, y0 = rng.uniform(0, period, 2)
        t[np.ix_((yy >= y0) & (yy < y0 + h), (xx >= x0) & (xx < x0 + w))] = 0
    return t


def thin_field(mask):
    """Reference ScatterField [Ny, Nx, 3] for a thin mask: channel 0 carries the transmission."""
    m = torch.as_tensor(mask, dtype=torch.float32)
    z = torch.zeros_like(m)
    return torch.stack((m, z, z), 2).to(torch.complex64)


def config1(seed=1):
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut = 'annular', 21, 0.6, 0.9
    mapped_optics(po, sr)
    nm.ImageCalculationMode, nm.ImageCalculationMethod = 'scalar', 'abbe'
    po.FocusRange = torch.tensor([0.0])
    sc.Period_X = sc.Period_Y = 1024
    sc.ScatterField = thin_field(rect_mask(256, 256, 1024, 1024, 12, 40.0, 300.0, np.random.default_rng(seed)))
    return sr, sc, po, nm


def config2(seed=2, n=512):
    sr, po, nm, sc = Source(), Projection(), Numerics(), Scatter()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut, sr.OpenAngle = 'quasar', 31, 0.5, 0.85, math.pi / 6
    sr.PolarizationVector = [1.0, 0.0]
    mapped_optics(po, sr)
    nm.ImageCalculationMode, nm.ImageCalculationMethod = 'vector', 'abbe'
    po.FocusRange = torch.tensor([-60.0, -30.0, 0.0, 30.0, 60.0])
    g = torch.Generator().manual_seed(seed + 1000)
    z = torch.zeros(37)
    z[4:] = 0.01 * torch.randn(33, generator=g)
    po.Aberration_Zernike = z
    sc.Period_X = sc.Period_Y = 2048
    sc.ScatterField = thin_field(line_space_mask(n, 2048, np.random.default_rng(seed)))
    return sr, sc, po, nm


def config3_optics(order=24):
    """Vector TCC optics of configuration 3: annular 0.7/0.95, PntNum 41, 2048 nm period, focus 0."""
    sr, po, nm = Source(), Projection(), Numerics()
    sr.Shape, sr.PntNum, sr.SigmaIn, sr.SigmaOut = 'annular', 41, 0.7, 0.95
    mapped_optics(po, sr)
    nm.ImageCalculationMode, nm.ImageCalculationMethod = 'vector', 'hopkins'
    nm.Hopkins_SettingType, nm.Hopkins_Order = 'order', order
    po.FocusRange = torch.tensor([0.0])
    return sr, po, nm


def config3_masks(count=64, n=1024, seed=3):
    """`count` binary Manhattan clips [count, n, n] float32 at 2048/n nm per pixel."""
    return manhattan_masks(count, n, 2048.0, seed)


def config4(seed=4, n=1024, order=16):
    sr, po, nm = config3_optics(order)
    rng = np.random.default_rng(seed)
    logits = rng.standard_normal((n, n)).astype(np.float32)
    target = rect_mask(n, n, 2048, 2048, 40, 60.0, 400.0, rng)
    return sr, po, nm, logits, target


CONFIG5_SIZES = (256, 512, 1024, 2048)


def config5_specs(form='bf16x3'):
    """The resident models of the serving stream, keyed (kind, n): SOCS-24 (annular 0.7/0.95 PntNum 41 vector
    TCC), vector Abbe (quasar 0.5/0.85/30deg PntNum 31, x_pol) and SOCS-24 at three focus planes (-40, 0, 40 nm),
    each for clips n x n at 2 nm/pixel (period 2n nm).  `form` is the serving form ('bf16x3' where the band
    allows it, FP32 FFT otherwise; None for the plain FP32 path)."""
    from . import serve
    sr, po, nm = config3_optics(order=24)
    q, qp, qn = Source(), Projection(), Numerics()
    q.Shape, q.PntNum, q.SigmaIn, q.SigmaOut, q.OpenAngle = 'quasar', 31, 0.5, 0.85, math.pi / 6
    q.PolarizationVector = [1.0, 0.0]
    mapped_optics(qp, q)
    qn.ImageCalculationMode, qn.ImageCalculationMethod = 'vector', 'abbe'
    specs = {}
    for n in CONFIG5_SIZES:
        period = 2.0 * n
        specs[('socs24', n)] = serve.socs_spec(sr, po, nm, period, n, name='socs24', form=form)
        specs[('abbe', n)] = serve.abbe_spec(q, qp, qn, period, n, name='abbe-quasar', form=form)
        specs[('socs24x3', n)] = serve.socs_spec(sr, po, nm, period, n, focus=(-40.0, 0.0, 40.0), name='socs24x3',
                                                 form=form)
    return specs


def config5_stream(count, seed=5):
    """`count` requests (kind, n, mask index): sizes uniform over CONFIG5_SIZES, kinds 50 % SOCS-24, 30 % Abbe,
    20 % three-plane SOCS."""
    rng = np.random.default_rng(seed)
    kinds = rng.choice(['socs24', 'abbe', 'socs24x3'], size=count, p=[0.5, 0.3, 0.2])
    sizes = rng.choice(CONFIG5_SIZES, size=count)
    return [(str(k), int(n), i) for i, (k, n) in enumerate(zip(kinds, sizes))]
