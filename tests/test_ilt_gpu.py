"""ILT and source-mask optimisation around the adjoint: the loop's first loss is the reference's (autograd
fixture), optimisation lowers it, a source re-weighting equals rebuilding the Abbe model from the new source,
and SMO keeps the weights positive while lowering the loss."""
import numpy as np
import pytest
import torch

from tests.fixtures import load, rel_err

pytestmark = pytest.mark.gpu


def test_optimize_mask_lowers_the_reference_loss():
    from opticalimaging_b200.engine import SocsKernels
    from opticalimaging_b200.ilt import ResistModel, optimize_mask
    meta, a = load('autograd')
    model = SocsKernels.from_full_grid(torch.from_numpy(a['kernels']).cuda())
    target = torch.from_numpy(a['target']).cuda()[None]
    logits = torch.from_numpy(a['logits']).cuda()[None]
    resist = ResistModel(meta['a'], meta['thr'])
    mask, losses = optimize_mask(model, target, logits=logits, steps=25, lr=0.1, resist=resist)
    print('ILT losses', losses[0], losses[-1])
    assert abs(losses[0] - float(a['loss'])) < 1e-4 * abs(float(a['loss']))
    assert losses[-1] < 0.5 * losses[0]
    assert torch.isfinite(mask).all() and (mask >= 0).all() and (mask <= 1).all()


def _small_abbe(values):
    from opticalimaging_b200.imaging import abbe_model
    from opticalimaging_b200.params import Numerics, Projection, Source
    from opticalimaging_b200 import workloads as W
    sr, po, nm = Source(), Projection(), Numerics()
    W.mapped_optics(po, sr)
    nm.ImageCalculationMode = 'vector'
    sr.Shape, sr.PntNum = 'pixel', 7
    c = torch.linspace(-1, 1, 7)
    sr.SPointX, sr.SPointY = torch.meshgrid(c, c, indexing='ij')
    sr.SPointValue = torch.from_numpy(values.astype(np.float32))
    return sr, po, abbe_model(sr, po, nm, 400.0, 480.0, 40, 48)


def test_set_source_weights_matches_rebuilt_model():
    from opticalimaging_b200.ilt import set_source_weights
    from opticalimaging_b200 import workloads as W
    rng = np.random.default_rng(3)
    v1 = 0.2 + rng.random((7, 7))
    v2 = 0.2 + rng.random((7, 7))
    sr1, po, m1 = _small_abbe(v1)
    sr2, _, m2 = _small_abbe(v2)
    mask = torch.from_numpy(W.rect_mask(40, 48, 400.0, 480.0, 8, 40, 160, rng)).cuda()[None]
    set_source_weights(m1, sr2.Calc_SourceSimple().Value, po.IndexImage)
    assert rel_err(m1.weights.cpu().numpy(), m2.weights.cpu().numpy()) < 1e-6
    assert rel_err(m1.image(mask).cpu().numpy(), m2.image(mask).cpu().numpy()) < 1e-6


def test_reweighting_drops_the_packed_fields():
    """A centrosymmetric source's Abbe fields pack two real fields to a transform for real masks; re-weighting
    the model for another source drops that packed set, and the images follow the new weights."""
    from opticalimaging_b200.ilt import set_source_weights
    from opticalimaging_b200 import workloads as W
    rng = np.random.default_rng(11)
    v = 0.2 + rng.random((7, 7))
    v1 = (v + v[::-1, ::-1]) / 2                    # symmetric under s -> -s
    v2 = 0.2 + rng.random((7, 7))
    sr1, po, m1 = _small_abbe(v1)
    sr2, _, m2 = _small_abbe(v2)
    assert m1.packed is not None and m1.packed[0].shape[1] < m1.count
    mask = torch.from_numpy(W.rect_mask(40, 48, 400.0, 480.0, 8, 40, 160, rng)).cuda()[None]
    own = m1.image(mask.to(torch.complex64).unsqueeze(-1)).cpu().numpy()
    assert rel_err(m1.image(mask).cpu().numpy(), own) < 1e-5
    set_source_weights(m1, sr2.Calc_SourceSimple().Value, po.IndexImage)
    assert m1.packed is None
    assert rel_err(m1.image(mask).cpu().numpy(), m2.image(mask).cpu().numpy()) < 1e-6


def test_source_mask_optimisation_lowers_the_loss():
    from opticalimaging_b200.ilt import ResistModel, optimize_source_mask
    from opticalimaging_b200 import workloads as W
    rng = np.random.default_rng(8)
    sr, po, model = _small_abbe(0.2 + rng.random((7, 7)))
    v0 = sr.Calc_SourceSimple().Value
    target = torch.from_numpy(W.rect_mask(40, 48, 400.0, 480.0, 6, 60, 160, rng)).cuda()[None]
    mask, v, losses = optimize_source_mask(model, v0, po.IndexImage, target, steps=20, lr_mask=0.1, lr_source=0.05,
                                           resist=ResistModel(20.0, 0.3))
    print('SMO losses', losses[0], losses[-1])
    assert losses[-1] < 0.75 * losses[0]
    assert torch.isfinite(v).all() and (v > 0).all()
    assert not torch.allclose(v.cpu(), v0.float().cpu())      # the source moved
