"""Benchmark configurations 2 and 4 at their own sizes on the GPU, against the FP64 oracle and the reference.

Configuration 2 (CalculateAerialImage.py:18-103): vector Abbe, x_pol, quasar 0.5/0.85/30 deg PntNum 31 (108
points), 512 x 512 over 2048 nm of 45/90 nm lines with 20 cuts, five focus planes -60..60 nm, Zernike Z5-Z37 ~
N(0, 0.01) waves.  Every plane of the FP32 form (through the drop-in CalculateAbbeImage) is held to 1e-5 of the
FP64 image's peak, and of the split-BF16x3 form to 1e-4; per-plane max and RMS are recorded.

Configuration 4 (CalculateAerialImage_SOCS.py:3-11 under the resist loss): the reference's SOCS-16 kernels of the
vector annular 0.7/0.95 PntNum 41 system at 2048 nm, a 1024 x 1024 mask sigmoid(logits), logits ~ N(0, 1),
loss ||sigmoid(50 (I - 0.25)) - target||^2.  The adjoint's gradient is held to 1e-3 of its maximum against:
the exact FP64 gradient at every pixel, central finite differences (h = 1e-3, FP64) on 32 seeded pixels, and the
reference's torch-autograd gradient at 4096 pixels.  The source-weight gradient (the Abbe identity
dI/dv_j = (n I_j - I) / sum v, for the untruncated image of the same source, 520 points) is held to 1e-3 of its
maximum against FP64 central differences on 6 points.
"""
import numpy as np
import pytest
import torch

from oracle import optics64 as O
from tests.fixtures import build, cfg4_kernels, load, rel_err

pytestmark = pytest.mark.gpu

A, THR, H = 50.0, 0.25, 1e-3


def _rms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.max(np.abs(b)))


# -------------------------------------------------------------------------------------- configuration 2
@pytest.fixture(scope='module')
def cfg2():
    from opticalimaging_b200 import workloads as W
    sr, sc, po, nm = W.config2()
    return sr, sc, po, nm, O.abbe(sr, sc, po, nm)


def test_config2_fp32_every_plane(cfg2, report):
    from opticalimaging_b200 import imaging
    sr, sc, po, nm, ref = cfg2
    img, _ = imaging.CalculateAbbeImage(sr, sc, po, nm)
    got = img.Intensity.numpy()
    assert got.shape == (5, 512, 512)
    per = {f'plane{z}_max': rel_err(got[z], ref[z]) for z in range(5)}
    per.update({f'plane{z}_rms': _rms(got[z], ref[z]) for z in range(5)})
    report('config2_fp32', **per)
    for z in range(5):
        assert rel_err(got[z], ref[z]) < 1e-5, z


def test_config2_split_form_every_plane(cfg2, report):
    from opticalimaging_b200 import imaging
    sr, sc, po, nm, ref = cfg2
    model = imaging.abbe_model(sr, po, nm, sc.Period_Y, sc.Period_X, 512, 512)
    mask = sc.ScatterField[:, :, 0].real.contiguous().cuda()[None]
    got = model.image(mask, form='bf16x3')[0].cpu().numpy()
    per = {f'plane{z}_max': rel_err(got[z], ref[z]) for z in range(5)}
    per.update({f'plane{z}_rms': _rms(got[z], ref[z]) for z in range(5)})
    report('config2_bf16x3', **per)
    for z in range(5):
        assert rel_err(got[z], ref[z]) < 1e-4, z


# -------------------------------------------------------------------------------------- configuration 4
@pytest.fixture(scope='module')
def cfg4():
    from opticalimaging_b200 import workloads as W
    meta, a = load('autograd_cfg4')
    _, _, _, logits, target = W.config4(seed=meta['seed'], n=meta['n'], order=meta['order'])
    K = cfg4_kernels(meta, a)
    I64, L64, G64 = O.socs_resist(logits, target, K, A, THR)
    return meta, a, logits, target, K, I64, L64, G64


def _engine_gradient(K, logits, target):
    from opticalimaging_b200.autograd import aerial_image
    from opticalimaging_b200.engine import SocsKernels
    model = SocsKernels.from_full_grid(torch.from_numpy(K.astype(np.complex64)).cuda())
    lt = torch.from_numpy(logits).cuda().requires_grad_(True)
    tg = torch.from_numpy(target).cuda()
    I = aerial_image(model, torch.sigmoid(lt)[None])[0, 0]
    loss = torch.sum((torch.sigmoid(A * (I - THR)) - tg) ** 2)
    loss.backward()
    torch.cuda.synchronize()
    return model, I.detach().cpu().numpy(), float(loss.item()), lt.grad.cpu().numpy()


def test_config4_adjoint_full_size(cfg4, report):
    from tests.test_oracle_golden import cfg4_central_differences
    meta, a, logits, target, K, I64, L64, G64 = cfg4
    model, I, loss, grad = _engine_gradient(K, logits, target)
    assert model.count == 16 and grad.shape == (1024, 1024)
    px = a['pixels']
    pk = float(np.max(np.abs(G64)))
    fd_pix = [tuple(p) for p in px[:32]]
    fd = cfg4_central_differences(logits, target, K, A, THR, fd_pix, h=H)
    got = np.array([grad[p] for p in fd_pix])
    err = dict(image_vs_fp64=rel_err(I, I64),
               image_vs_reference=float(np.max(np.abs(I[px[:, 0], px[:, 1]] - a['image_at'])) / a['image_peak']),
               loss_vs_fp64=abs(loss - L64) / L64, loss_vs_reference=abs(loss - float(a['loss'])) / float(a['loss']),
               grad_vs_fp64_max=float(np.max(np.abs(grad - G64)) / pk), grad_vs_fp64_rms=_rms(grad, G64),
               grad_vs_fd32=float(np.max(np.abs(got - fd)) / pk),
               grad_vs_reference_autograd=float(np.max(np.abs(grad[px[:, 0], px[:, 1]] - a['grad_at']))
                                                / a['grad_maxabs']))
    report('config4_adjoint', **err)
    assert err['image_vs_fp64'] < 1e-5
    assert err['image_vs_reference'] < 1e-4           # the reference's own rounding here: 5.7e-5
    assert err['loss_vs_fp64'] < 1e-4
    assert err['grad_vs_fp64_max'] < 1e-3
    assert err['grad_vs_fd32'] < 1e-3
    assert err['grad_vs_reference_autograd'] < 1e-3   # the reference's own rounding here: 4.4e-4


def test_config4_source_weight_gradient(cfg4, report):
    """dL/dv over the 520 source points of the configuration-4 source, through the Abbe identity (the gradient
    of the untruncated image), against FP64 central differences of the loss on the FP64 Abbe image."""
    from opticalimaging_b200 import workloads as W
    from opticalimaging_b200.autograd import aerial_image, source_weight_gradient
    from opticalimaging_b200.imaging import abbe_model
    from opticalimaging_b200.params import Scatter
    meta, a, logits, target, K, *_ = cfg4
    sr, po, nm = W.config3_optics(order=16)
    nm.ImageCalculationMethod = 'abbe'
    sd = sr.Calc_SourceSimple()
    S = sd.Value.numel()
    assert S == 520
    t = (1.0 / (1.0 + np.exp(-logits.astype(np.float64))))
    mask = torch.from_numpy(t.astype(np.float32)).cuda()[None]
    model = abbe_model(sr, po, nm, 2048.0, 2048.0, 1024, 1024)
    with torch.no_grad():
        I = aerial_image(model, mask)[0, 0]
        s = torch.sigmoid(A * (I - THR))
        gI = 2.0 * (s - torch.from_numpy(target).cuda()) * A * s * (1.0 - s)
    got = source_weight_gradient(model, mask, gI[None, None], sd.Value, po.IndexImage)[0].cpu().numpy()
    assert got.shape == (S,)
    # FP64: the Abbe image and the unweighted intensities A_j of the sampled points
    sc = Scatter()
    sc.Period_X = sc.Period_Y = 2048.0
    z = np.zeros_like(t)
    sc.ScatterField = np.stack((t, z, z), 2)
    js = [int(j) for j in np.random.default_rng(41).choice(S, 6, replace=False)]
    I64, Aj = O.abbe(sr, sc, po, nm, points=js)
    I64 = I64[0]
    v = sd.Value.numpy().astype(np.float64)
    W_, n = float(v.sum()), float(po.IndexImage)

    def loss64(img):
        s64 = 1.0 / (1.0 + np.exp(-A * (img - THR)))
        return float(np.sum((s64 - target) ** 2))
    fd = []
    for j in js:   # I(v + d e_j) = (W I + n d A_j) / (W + d)
        fd.append((loss64((W_ * I64 + n * H * Aj[j][0]) / (W_ + H))
                   - loss64((W_ * I64 - n * H * Aj[j][0]) / (W_ - H))) / (2 * H))
    fd = np.array(fd)
    err = float(np.max(np.abs(got[js] - fd)) / np.max(np.abs(got)))
    report('config4_source_weights', grad_vs_fd6=err, image_vs_fp64=rel_err(I.cpu().numpy(), I64), points=S)
    assert rel_err(I.cpu().numpy(), I64) < 1e-5
    assert err < 1e-3
