"""Adjoint kernel (inverse lithography): mask gradient vs torch autograd through the reference and vs FP64
central finite differences; source-weight gradient of the Abbe image vs FP64 finite differences."""
import numpy as np
import pytest
import torch

from oracle import optics64 as O
from tests.fixtures import load, make_source, rel_err

pytestmark = pytest.mark.gpu


def _setup():
    from opticalimaging_b200.engine import SocsKernels
    from opticalimaging_b200.params import Projection, Scatter
    from opticalimaging_b200 import workloads as W
    meta, a = load('autograd')
    sr = make_source(meta['src'])
    po = Projection()
    W.mapped_optics(po, sr)
    model = SocsKernels.from_full_grid(torch.from_numpy(a['kernels']).cuda())
    return meta, a, sr, po, model


def _loss_torch(I, target, a, thr):
    return torch.sum((torch.sigmoid(a * (I - thr)) - target) ** 2)


def test_gradient_matches_reference_autograd():
    from opticalimaging_b200.autograd import aerial_image
    meta, a, sr, po, model = _setup()
    logits = torch.from_numpy(a['logits']).cuda().requires_grad_(True)
    target = torch.from_numpy(a['target']).cuda()
    I = aerial_image(model, torch.sigmoid(logits)[None])[0, 0]
    assert rel_err(I.detach().cpu().numpy(), a['image']) < 2e-5
    loss = _loss_torch(I, target, meta['a'], meta['thr'])
    loss.backward()
    assert abs(loss.item() - float(a['loss'])) < 1e-4 * abs(float(a['loss']))
    assert rel_err(logits.grad.cpu().numpy(), a['grad']) < 1e-4


def test_gradient_matches_fp64_finite_differences():
    from opticalimaging_b200.autograd import aerial_image
    from opticalimaging_b200.params import Scatter
    meta, a, sr, po, model = _setup()
    logits = torch.from_numpy(a['logits']).cuda().requires_grad_(True)
    target = torch.from_numpy(a['target']).cuda()
    loss = _loss_torch(aerial_image(model, torch.sigmoid(logits)[None])[0, 0], target, meta['a'], meta['thr'])
    loss.backward()
    grad = logits.grad.cpu().numpy()
    K = a['kernels'].astype(np.complex128)
    lg = a['logits'].astype(np.float64)
    tg = a['target'].astype(np.float64)

    def loss64(l):
        sc = Scatter()
        sc.Period_X, sc.Period_Y = meta['Period_X'], meta['Period_Y']
        t = 1.0 / (1.0 + np.exp(-l))
        z = np.zeros_like(t)
        sc.ScatterField = np.stack((t, z, z), 2)
        I = O.socs(sc, K, sr, po)
        return float(np.sum((1.0 / (1.0 + np.exp(-meta['a'] * (I - meta['thr']))) - tg) ** 2))

    rng = np.random.default_rng(32)
    h = 1e-3
    idx = [tuple(rng.integers(0, s) for s in lg.shape) for _ in range(32)]
    fd = []
    for p in idx:
        lp, lm = lg.copy(), lg.copy()
        lp[p] += h
        lm[p] -= h
        fd.append((loss64(lp) - loss64(lm)) / (2 * h))
    fd = np.array(fd)
    got = np.array([grad[p] for p in idx])
    assert np.max(np.abs(got - fd)) / np.max(np.abs(grad)) < 1e-3


def test_source_weight_gradient_matches_fp64_finite_differences():
    from opticalimaging_b200.autograd import aerial_image, source_weight_gradient
    from opticalimaging_b200.imaging import abbe_model
    from opticalimaging_b200.params import Numerics, Projection, Scatter, Source
    from opticalimaging_b200 import workloads as W
    ny, nx, py, px = 40, 48, 400.0, 480.0
    sr, po, nm = Source(), Projection(), Numerics()
    W.mapped_optics(po, sr)
    nm.ImageCalculationMode = 'vector'
    sr.Shape, sr.PntNum = 'pixel', 7
    c = torch.linspace(-1, 1, 7)
    sr.SPointX, sr.SPointY = torch.meshgrid(c, c, indexing='ij')
    rng = np.random.default_rng(11)
    vals = (0.2 + rng.random((7, 7))).astype(np.float32)
    sr.SPointValue = torch.from_numpy(vals.copy())
    sd = sr.Calc_SourceSimple()
    keep = np.argwhere(((sr.SPointX ** 2 + sr.SPointY ** 2) <= 1).numpy() & (np.arange(49).reshape(7, 7) != 24))
    assert len(keep) == sd.Value.numel()
    mask = W.rect_mask(ny, nx, py, px, 8, 40, 160, rng)
    g0 = rng.standard_normal((ny, nx))
    model = abbe_model(sr, po, nm, py, px, ny, nx)
    mt = torch.from_numpy(mask).cuda()[None]
    I = aerial_image(model, mt)                      # linear loss L = <g0, I>
    got = source_weight_gradient(model, mt, torch.from_numpy(g0).float().cuda()[None, None], sd.Value,
                                 po.IndexImage)[0].cpu().numpy()

    def loss64(v):
        s2 = Source()
        W.mapped_optics(Projection(), s2)
        s2.Wavelength, s2.Shape, s2.PntNum = sr.Wavelength, 'pixel', 7
        s2.SPointX, s2.SPointY, s2.SPointValue = sr.SPointX, sr.SPointY, torch.from_numpy(v.astype(np.float32))
        sc = Scatter()
        sc.Period_X, sc.Period_Y = px, py
        z = np.zeros_like(mask)
        sc.ScatterField = np.stack((mask, z, z), 2)
        return float(np.sum(g0 * O.abbe(s2, sc, po, nm)[0]))

    h = 1e-3
    for j in rng.choice(len(keep), 6, replace=False):
        r, cc = keep[j]
        vp, vm = vals.copy(), vals.copy()
        vp[r, cc] += h
        vm[r, cc] -= h
        fd = (loss64(vp) - loss64(vm)) / (2 * h)
        assert abs(got[j] - fd) < 1e-3 * np.max(np.abs(got)) + 1e-6, (j, got[j], fd)
