"""Inverse lithography (ILT) and source-mask optimisation (SMO) around the adjoint kernel.

* ``ResistModel``: the sigmoid threshold resist R(I) = sigmoid(a (I - threshold)) of the inverse-lithography
  study (steepness a = 50, threshold 0.25).
* ``optimize_mask``: pixel-based ILT.  The mask transmission is m = sigmoid(logits); the loss is
  ||R(I(m)) - target||^2 summed over pixels and focus planes; Adam steps on the logits, the gradient through
  ``autograd.aerial_image`` (the hand-written adjoint, no stored per-field arrays).  Works with SOCS kernels and
  with Abbe models.
* ``optimize_source_mask``: source-mask co-optimisation on an Abbe model.  Source weights are v = exp(s) (kept
  positive); each iteration takes one Adam step on the mask logits and one on s, both gradients at the same
  point: the mask's through the adjoint, the source's from ``source_weight_gradient`` (dI/dv_j =
  (n I_j - I) / sum v, CalculateAerialImage.py:89-92).  A source update only rescales the model's field weights
  (``set_source_weights``, weight of point j = n v_j / sum v); the pupils stay resident.

The reference has no optimisation loop; it differentiates its SOCS image by torch autograd
(CalculateAerialImage_SOCS.py:3-11), which the adjoint reproduces (tests/test_adjoint_gpu.py).
"""
from __future__ import annotations

import torch

from .autograd import aerial_image, source_weight_gradient
from .engine import CoherentModel


class ResistModel:
    """Sigmoid threshold resist: R(I) = sigmoid(steepness (I - threshold))."""

    def __init__(self, steepness: float = 50.0, threshold: float = 0.25):
        self.steepness, self.threshold = float(steepness), float(threshold)

    def __call__(self, image: torch.Tensor) -> torch.Tensor:
        return torch.sigmoid(self.steepness * (image - self.threshold))


def ilt_loss(model: CoherentModel, mask: torch.Tensor, target: torch.Tensor, resist: ResistModel):
    """(loss, image): ||R(I(mask)) - target||^2 over pixels and planes; mask [B, ny, nx], target [B, ny, nx]."""
    image = aerial_image(model, mask)                        # [B, Z, ny, nx]
    loss = torch.sum((resist(image) - target[:, None]) ** 2)
    return loss, image


def _check_target(model: CoherentModel, target: torch.Tensor) -> torch.Tensor:
    if target.dim() != 3 or target.shape[1:] != (model.ny, model.nx):
        raise ValueError(f'target must be [B, {model.ny}, {model.nx}]')
    return target.to(model.device, torch.float32).contiguous()


def optimize_mask(model: CoherentModel, target: torch.Tensor, logits: torch.Tensor | None = None, steps: int = 50,
                  lr: float = 0.1, resist: ResistModel | None = None):
    """Pixel-based ILT: Adam on the mask logits for `steps` iterations.  Returns (mask, losses), mask =
    sigmoid(logits) [B, ny, nx] and the loss before each step.  Default start: logits = 4 (target - 1/2)."""
    resist = resist or ResistModel()
    target = _check_target(model, target)
    if logits is None:
        logits = 4.0 * (target - 0.5)
    logits = logits.to(model.device, torch.float32).detach().clone().requires_grad_(True)
    opt = torch.optim.Adam([logits], lr=lr)
    losses = []
    for _ in range(steps):
        opt.zero_grad()
        loss, _ = ilt_loss(model, torch.sigmoid(logits), target, resist)
        loss.backward()
        opt.step()
        losses.append(loss.item())
    return torch.sigmoid(logits).detach(), losses


def set_source_weights(model: CoherentModel, values: torch.Tensor, index_image: float) -> None:
    """Re-weight an Abbe model for source weights `values` [S] (the order of Calc_SourceSimple's Value): field
    (point j, component e) of every plane gets n v_j / sum v.  The pupils do not depend on the weights."""
    if model.kind != 'abbe':
        raise ValueError('source weights belong to an Abbe model (abbe_model)')
    Z, K = model.weights.shape
    v = values.to(model.device, torch.float64).reshape(-1)
    if K % v.numel():
        raise ValueError(f'{v.numel()} source weights do not divide the model\'s {K} fields')
    w = (index_image / v.sum()) * v
    P = getattr(model, 'pol_states', 1)          # fields are [polarisation state][point][component]
    per = w.repeat_interleave(K // (P * v.numel())).repeat(P)
    model.weights.copy_(per.to(torch.float32)[None].expand(Z, K))
    model.packed = None   # packed for the previous weights


def optimize_source_mask(model: CoherentModel, values: torch.Tensor, index_image: float, target: torch.Tensor,
                         logits: torch.Tensor | None = None, steps: int = 30, lr_mask: float = 0.1,
                         lr_source: float = 0.05, resist: ResistModel | None = None):
    """SMO on an Abbe model: per iteration one Adam step on the mask logits and one on the source log-weights,
    both gradients taken at the same point.  Returns (mask, source weights [S], losses).  The model's weights are
    left set to the returned source."""
    if model.kind != 'abbe':
        raise ValueError('source-mask optimisation needs an Abbe model (abbe_model)')
    resist = resist or ResistModel()
    target = _check_target(model, target)
    if logits is None:
        logits = 4.0 * (target - 0.5)
    logits = logits.to(model.device, torch.float32).detach().clone().requires_grad_(True)
    s = torch.log(values.to(model.device, torch.float64).reshape(-1).clamp_min(1e-12)).requires_grad_(True)
    opt_m = torch.optim.Adam([logits], lr=lr_mask)
    opt_s = torch.optim.Adam([s], lr=lr_source)
    losses = []
    for _ in range(steps):
        v = torch.exp(s.detach())
        set_source_weights(model, v, index_image)
        opt_m.zero_grad()
        opt_s.zero_grad()
        mask = torch.sigmoid(logits)
        loss, image = ilt_loss(model, mask, target, resist)
        image.retain_grad()
        loss.backward()                                       # dL/dlogits and dL/dI
        gv = source_weight_gradient(model, mask.detach(), image.grad, v, index_image)   # [B, S]
        s.grad = gv.sum(dim=0).to(torch.float64) * v          # dL/ds = dL/dv * v
        opt_m.step()
        opt_s.step()
        losses.append(loss.item())
    v = torch.exp(s.detach())
    set_source_weights(model, v, index_image)
    return torch.sigmoid(logits).detach(), v.float(), losses
