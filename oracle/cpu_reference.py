"""The reference's SOCS imaging algorithm at its own precision, for timing on host cores.  TEST/BENCH ONLY.

CalculateAerialImage_SOCS.py:3-11 and Scatter.py:10-21 restated with torch's CPU FFT on complex64, running on
all requested host threads: the centred spectrum of the [N, N, 3] scatter field, one full-grid fft2 per
(kernel, channel) -- 3K transforms per clip, as the reference does even for all-zero channels -- |.|^2 summed
and fftshifted.  Used as ``cpu_baseline`` (kind "port") and as ``bench.py --impl reference``.
"""
import numpy as np
import scipy.fft as sfft


def socs_clip(field, kernels, npx, npy, workers):
    """field [N, N, 3] complex64, kernels [N, N, K] complex64 (reference layout) -> image [N, N] float32.

    torch CPU FFTs on complex64 -- the reference's own primitives and precision -- on `workers` threads.
    """
    import torch
    torch.set_num_threads(workers)
    h = torch.as_tensor(field)
    k = torch.as_tensor(kernels)
    hk = torch.fft.fftshift(torch.fft.ifft2(torch.fft.ifftshift(h, dim=(0, 1)), dim=(0, 1)), dim=(0, 1))
    hk = hk * (npx * npy)
    sp = torch.fft.ifftshift(hk.unsqueeze(3).permute(0, 1, 3, 2), dim=(0, 1))
    e = (1.0 / (npx * npy)) * torch.fft.fft2(k.unsqueeze(3) * sp, dim=(0, 1))
    inten = torch.sum(torch.abs(e) ** 2, dim=(2, 3))
    return torch.fft.fftshift(inten, dim=(0, 1)).numpy()


def socs_kernels(sr, po, nm, xypitch, nfg, focus=0.0):
    """SOCS kernels [Ny, Nx, K] complex64 in the reference's layout, built on the host: the TCC of
    CalculateTCCMatrix.py:9-75 (complex64, as the reference) and its top-K eigenvectors embedded as
    DecomposeTCC_SOCS.py:26-35 does."""
    from . import optics64 as O
    G, w, fg = O.pupil_matrix(sr, xypitch, po, focus, nm)
    Gs = (G * np.sqrt(w / np.sum(w))[None, None, :]).astype(np.complex64)
    T = po.IndexImage * sum(g @ g.conj().T for g in Gs)
    lam, U = np.linalg.eigh(T)
    lam, U = np.maximum(lam[::-1], 0), U[:, ::-1]
    k = O.socs_count(nm, lam, U.shape[1])
    nf, ng = nfg
    out = np.zeros((ng, nf, k), dtype=np.complex64)
    tmp = np.zeros((ng, nf), dtype=np.complex64)
    r0, c0 = (ng - fg[1] + 1) // 2, (nf - fg[0] + 1) // 2
    for i in range(k):
        tmp[r0:r0 + fg[1], c0:c0 + fg[0]] = U[:, i].reshape(fg[1], fg[0])
        out[:, :, i] = sfft.fftshift(tmp)
    return out * np.sqrt(lam[:k]).astype(np.float32).reshape(1, 1, -1)
