"""Differentiable aerial images for inverse lithography.

``aerial_image(model, mask)`` is the batched image of a resident ``CoherentModel`` (SOCS kernels or Abbe
pupils) as a ``torch.autograd.Function``: its backward runs the hand-written adjoint (``oi_coherent_adjoint``),
so a loss on the image -- e.g. a sigmoid resist model against a target -- differentiates into the mask
transmission without storing any per-field array (the forward is recomputed inside the adjoint).

``source_weight_gradient(...)`` gives dL/dv_j for the source-point weights v_j of an Abbe model through the
linear Abbe identity dI/dv_j = (n I_j - I) / sum(v) (CalculateAerialImage.py:89-92): the gradient of the
untruncated image.  For a SOCS model the truncated kernels depend on the source through the eigenvectors,
so its source gradient is taken as that of the untruncated (Abbe) image, which is what it approximates.

The reference obtains gradients by torch autograd through its FFTs (CalculateAerialImage_SOCS.py:3-11); the
tests compare both, and central finite differences in FP64.
"""
from __future__ import annotations

import torch

from . import _native as N
from .engine import Band, CoherentModel, Plan, band_spectrum, field_split


def _half_spectrum_to_image(ihat: torch.Tensor, br: int, bc: int, ny: int, nx: int) -> torch.Tensor:
    """Real images [count, ny, nx] from Hermitian halves ihat [count, 2br-1, bc] (qc > 0 already doubled)."""
    dev = ihat.device
    count = ihat.shape[0]
    plan = Plan.get(ny, nx, Band(-(br - 1), br, 0, bc), dev)
    out = torch.empty((count, ny, nx), dtype=torch.float32, device=dev)
    ih = ihat.contiguous()
    s = N.stream_handle(dev)
    if plan.fft:
        v = torch.empty(count * bc * ny, dtype=torch.complex64, device=dev)
        N.call('oi_spectrum_to_image_fft', N.ptr(ih), count, br, bc, N.ptr(plan.wn_y), N.ptr(plan.wn_x), ny, nx,
               N.ptr(v), N.ptr(out), s)
    else:
        N.call('oi_spectrum_to_image', N.ptr(ih), count, br, bc, N.ptr(plan.sy), N.ptr(plan.sx), ny, nx, N.ptr(out), s)
    return out


ADJOINT_COARSE = (128, 128)


def adjoint_plan(model: CoherentModel) -> Plan:
    """The model's plan on the 128 x 128 coarse grid the adjoint kernel works on (exact for bands up to 64)."""
    b = model.band
    if 2 * b.br - 1 > ADJOINT_COARSE[0] or 2 * b.bc - 1 > ADJOINT_COARSE[1]:
        raise NotImplementedError(f'the adjoint covers bands up to 64 x 64 (this one is {b.br} x {b.bc})')
    return Plan.get(model.ny, model.nx, b, model.device, coarse=ADJOINT_COARSE)


def coarse_gradient(model: CoherentModel, g: torch.Tensor) -> torch.Tensor:
    """The band-limited coarse copy g^c [B, Z, Mr, Mc] of g = dL/dI [B, Z, ny, nx]:
    g^c(s) = 1/(Mr Mc) sum_{|qr|<br, |qc|<bc} ghat(q) exp(-2 pi i q.s/M), ghat(q) = sum_r g(r) exp(+2 pi i q.r/N)."""
    b, plan = model.band, adjoint_plan(model)
    B, Z = g.shape[0], g.shape[1]
    ib = Band(-(b.br - 1), 2 * b.br - 1, 0, b.bc)                     # image band, Hermitian half in x
    gplan = Plan.get(model.ny, model.nx, ib, model.device)
    gh = band_spectrum(g.reshape(B * Z, model.ny, model.nx).contiguous(), N.FIELD_REAL_F32, gplan,
                       scale=float(model.ny * model.nx))[:, 0]          # [B*Z, 2br-1, bc], ghat(q)
    gh = gh * (1.0 / (plan.mr * plan.mc))
    gh[:, :, 1:] *= 2.0
    return _half_spectrum_to_image(gh, b.br, b.bc, plan.mr, plan.mc).view(B, Z, plan.mr, plan.mc)


def coherent_adjoint(model: CoherentModel, band: torch.Tensor, gc: torch.Tensor, field_dots: bool = False):
    """W [B, nch, br, bc] (summed over planes) and, optionally, field dots [B, Z, K*nch]."""
    b, plan = model.band, adjoint_plan(model)
    B, nch = band.shape[0], band.shape[1]
    Z, K = model.planes, model.count
    nsplit = field_split(K * nch, B * Z)
    wout = torch.empty((nsplit, B, Z, nch, b.br, b.bc), dtype=torch.complex64, device=model.device)
    dots = torch.empty((B, Z, K * nch), dtype=torch.float32, device=model.device) if field_dots else None
    N.call('oi_coherent_adjoint', N.ptr(band), B, nch, b.m0r, b.br, b.m0c, b.bc, N.ptr(model.pupils),
           N.ptr(model.weights), Z, K, N.ptr(gc.contiguous()), plan.mr, plan.mc, N.ptr(plan.wm_r),
           N.ptr(plan.wm_c), nsplit, N.ptr(wout), N.ptr(dots), N.stream_handle(model.device))
    return wout.sum(dim=(0, 2)), dots


def mask_gradient_from_w(model: CoherentModel, w: torch.Tensor) -> torch.Tensor:
    """dL/dt [B, ny, nx] = 2/(ny nx) Re sum_{m in band} W(m) exp(-2 pi i m.y/N) for W [B, br, bc]."""
    b = model.band
    B = w.shape[0]
    R = max(abs(b.m0r), abs(b.m0r + b.br - 1))
    C = max(abs(b.m0c), abs(b.m0c + b.bc - 1))
    full = torch.zeros((B, 2 * R + 1, 2 * C + 1), dtype=torch.complex64, device=w.device)
    full[:, b.m0r + R: b.m0r + R + b.br, b.m0c + C: b.m0c + C + b.bc] = w
    herm = 0.5 * (full + torch.conj(torch.flip(full, dims=(1, 2))))       # H(q) = (W(q) + conj W(-q)) / 2
    half = herm[:, :, C:] * (2.0 / (model.ny * model.nx))
    half[:, :, 1:] *= 2.0
    return _half_spectrum_to_image(half, R + 1, C + 1, model.ny, model.nx)


class _CoherentImage(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mask, model):
        ctx.model = model
        ctx.save_for_backward(mask)
        with torch.no_grad():
            return CoherentModel.image(model, mask.detach().contiguous())   # [B, Z, ny, nx] for every model

    @staticmethod
    def backward(ctx, g):
        (mask,) = ctx.saved_tensors
        model = ctx.model
        with torch.no_grad():
            band = band_spectrum(mask.detach().contiguous(), N.FIELD_REAL_F32, model.plan)
            gc = coarse_gradient(model, g.to(torch.float32).contiguous())
            w, _ = coherent_adjoint(model, band, gc)
            grad = mask_gradient_from_w(model, w[:, 0])
        return grad.view_as(mask), None


def aerial_image(model: CoherentModel, mask: torch.Tensor) -> torch.Tensor:
    """Differentiable image [B, Z, ny, nx] of real float32 masks [B, ny, nx] (gradient via the adjoint kernel)."""
    if mask.dtype != torch.float32 or mask.dim() != 3:
        raise ValueError('mask must be a float32 [B, ny, nx] tensor')
    return _CoherentImage.apply(mask, model)


def source_weight_gradient(model: CoherentModel, mask: torch.Tensor, g: torch.Tensor, values: torch.Tensor,
                           index_image: float) -> torch.Tensor:
    """dL/dv [B, S] for the source weights v (the Value of Calc_SourceSimple, length S) of an Abbe model
    built from them: dI/dv_j = (n I_j - I) / sum(v), I_j = sum_e |E_{j,e}|^2 (CalculateAerialImage.py:89-92)."""
    if model.kind != 'abbe':
        raise ValueError('source_weight_gradient needs an Abbe model (abbe_model)')
    with torch.no_grad():
        band = band_spectrum(mask.contiguous(), N.FIELD_REAL_F32, model.plan)
        gc = coarse_gradient(model, g.to(torch.float32).contiguous())
        _, dots = coherent_adjoint(model, band, gc, field_dots=True)    # [B, Z, P*S*E]
        S = values.numel()
        P = getattr(model, 'pol_states', 1)                              # incoherent polarisation states
        E = model.count // (S * P)
        d = dots.view(dots.shape[0], dots.shape[1], P, S, E).sum(dim=(1, 2, 4)).double()   # <g, I_j>
        v = values.to(d.device, torch.float64).reshape(1, -1)
        W = v.sum()
        gI = (d * v).sum(dim=1, keepdim=True) * index_image / W               # <g, I>
        return ((index_image * d - gI) / W).float()
