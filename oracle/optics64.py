"""FP64 CPU oracle of the aerial-image path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import this module, and
only to check or time results.  The engine never routes through it.

It restates, in numpy float64/complex128, the reference's algorithm literally (full-grid FFTs, one per source
point / kernel / channel / field component), citing the reference file:line each step follows:

* ``source_points``   -- Source.py:47-54, 64-180, 229-297
* ``spectrum``        -- Scatter.py:10-35
* ``aberration``      -- Projection.py:13-128
* ``char_matrix``     -- CalculateCharacteristicMatrix.py:3-17
* ``abbe``            -- CalculateAerialImage.py:18-103
* ``tcc``             -- CalculateTCCMatrix.py:9-75
* ``decompose``       -- DecomposeTCC_SOCS.py:3-37 (Hermitian ``eigh`` in place of ``svd``)
* ``socs``            -- CalculateAerialImage_SOCS.py:3-11
* ``socs_resist``     -- the resist loss on that image and its gradient (the chain rule torch autograd applies
                         through CalculateAerialImage_SOCS.py:3-11)
* ``hopkins``         -- CalculateAerialImage.py:105-130
* ``socs_floquet``    -- CalculateAerialImage_SOCS.py:13-32

Precision policy.  The reference computes in float32/complex64.  Its *discrete* decisions -- which source
points exist, which pupil samples are inside the pupil -- are float32 comparisons, and this oracle repeats them
in float32 with the same operation order, so that both sides sum over the same samples.  The source grid comes
from ``torch.linspace`` (and the optional source blur from ``torch.nn.functional.conv2d``) because those are
the reference's own primitives and numpy's equivalents differ from them in the last bit.  Everything else --
pupil phases, the polarisation transfer, the transforms, the TCC, its eigendecomposition -- runs in float64 at
the reference's float32 sample positions.

Pinned against fixtures produced by running the reference itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
import os

import numpy as np

F32 = np.float32

try:   # the same pocketfft transforms as numpy.fft, on every host core
    import scipy.fft as _sfft
except ImportError:   # pragma: no cover
    _sfft = None


def _fft2(a, axes=(-2, -1)):
    """Forward 2-D DFT (numpy.fft.fft2 convention), threaded over the host cores when scipy is present."""
    if _sfft is not None:
        return _sfft.fft2(a, axes=axes, workers=os.cpu_count() or 1)
    return np.fft.fft2(a, axes=axes)


def _ifft2(a, axes=(-2, -1)):
    if _sfft is not None:
        return _sfft.ifft2(a, axes=axes, workers=os.cpu_count() or 1)
    return np.fft.ifft2(a, axes=axes)


# ----------------------------------------------------------------------------------------------- source
def _linspace_f32(n):
    import torch
    return torch.linspace(-1, 1, n).numpy()


def _source_matrix(sr):
    """Rasterised source value matrix and its coordinates, float32 (Source.py:64-143, 229-286)."""
    shape = sr.Shape.lower()
    if shape == "pixel":
        return (np.asarray(sr.SPointX, dtype=F32), np.asarray(sr.SPointY, dtype=F32),
                np.asarray(sr.SPointValue, dtype=F32).copy())
    c = _linspace_f32(sr.PntNum)
    X, Y = np.meshgrid(c, c, indexing='ij')
    V = np.zeros_like(X)
    if shape == "multipole":
        step = 2 * math.pi / sr.PoleNumber
        for i in range(sr.PoleNumber):
            xc = F32(sr.SigmaCenter * math.cos(sr.RotateAngle + i * step))
            yc = F32(sr.SigmaCenter * math.sin(sr.RotateAngle + i * step))
            V[((X - xc) ** 2 + (Y - yc) ** 2) <= F32(sr.SigmaRadius ** 2)] = 1.0 / sr.PoleNumber / (sr.SigmaRadius ** 2)
        return X, Y, V
    R = np.sqrt(X * X + Y * Y)
    ring = (R <= F32(sr.SigmaOut)) & (R >= F32(sr.SigmaIn))
    if shape == "annular":
        V[ring] = 1.0 / ((sr.SigmaOut ** 2 - sr.SigmaIn ** 2) * math.pi)
    elif shape == "quasar":
        th = np.arctan2(Y, X)
        h = F32(sr.OpenAngle / 2)
        a = np.abs(th)
        on = (a <= h) | ((a >= F32(math.pi - sr.OpenAngle / 2)) & (a <= F32(math.pi)))
        on |= (np.abs(th - F32(math.pi / 2)) <= h) | (np.abs(th + F32(math.pi / 2)) <= h)
        V[ring & on] = 0.5 / ((sr.SigmaOut ** 2 - sr.SigmaIn ** 2) * sr.OpenAngle)
    elif shape == "dipolecirc":
        th = np.arctan2(Y, X)
        on = np.abs(np.cos(th - F32(sr.RotateAngle))) >= F32(math.cos(sr.OpenAngle / 2))
        V[ring & on] = 1.0 / ((sr.SigmaOut ** 2 - sr.SigmaIn ** 2) * sr.OpenAngle)
    else:
        raise ValueError("unsupported illumination")
    return X, Y, V


def source_points(sr):
    """(X, Y, Value) of the live source points, float32 1-D (Source.py:47-54, 144-180, 288-297)."""
    X, Y, V = _source_matrix(sr)
    if V.ndim == 2:
        if sr.Source_Mask is not None:
            V = V * np.asarray(sr.Source_Mask, dtype=F32)
        if V.shape[0] == V.shape[1]:
            if sr.PSFEnable:
                import torch
                import torch.nn.functional as Fnn
                ks = round(sr.PntNum / 10) * 2 + 1
                ke = 1 / (sr.PntNum - 1) * (ks - 1)
                kx, ky = torch.meshgrid(torch.linspace(-ke, ke, ks), torch.linspace(-ke, ke, ks), indexing='ij')
                ker = 1 / math.sqrt(2 * math.pi) / sr.PSFSigma * torch.exp(-(kx.pow(2) + ky.pow(2)) / sr.PSFSigma ** 2)
                ker = ker[~torch.all(ker < 1e-6, 0)]
                kt = torch.transpose(ker, 0, 1)
                ker = kt[~torch.all(kt < 1e-6, 1)]
                ker = ker / torch.sum(ker)
                n0, n1 = V.shape
                V = Fnn.conv2d(torch.from_numpy(V).reshape(1, 1, n0, n1), ker.reshape(1, 1, *ker.shape),
                               padding='same').reshape(n0, n1).numpy()
            V = V.copy()
            V[int((V.shape[0] - 1) / 2), int((V.shape[1] - 1) / 2)] = 0
            V[(X * X + Y * Y) > 1] = 0
    X, Y, V = (np.asarray(a, dtype=F32).reshape(-1) for a in (X, Y, V))
    keep = ~(V < F32(1e-5))
    return X[keep], Y[keep], V[keep]


# --------------------------------------------------------------------------------------------- spectrum
def freq_axes(sc, po, sr):
    """Spectrum axes f (columns, X) and g (rows, Y) as the reference's float32 values (Scatter.py:17-18)."""
    ny, nx = np.asarray(sc.ScatterField).shape[:2]
    npx = sc.Period_X / (sr.Wavelength / po.NA)
    npy = sc.Period_Y / (sr.Wavelength / po.NA)
    f = F32(1 / npx) * np.arange(-(nx // 2), (nx + 1) // 2).astype(F32)
    g = F32(1 / npy) * np.arange(-(ny // 2), (ny + 1) // 2).astype(F32)
    return f, g, npx, npy


def spectrum(sc, po, sr):
    """Hk = npx*npy * fftshift(ifft2(ifftshift(h))), complex128 [Ny, Nx, C]; plus f, g (Scatter.py:10-35)."""
    h = np.asarray(sc.ScatterField).astype(np.complex128)
    f, g, npx, npy = freq_axes(sc, po, sr)
    hk = np.fft.fftshift(_ifft2(np.fft.ifftshift(h, axes=(0, 1)), axes=(0, 1)), axes=(0, 1)) * (npx * npy)
    return hk, f, g


def _cell_area(sc, po, sr):
    """Frequency cell area df*dg = 1/(npx*npy) (CalculateAerialImage.py:38, CalculateAerialImage_SOCS.py:7)."""
    _, _, npx, npy = freq_axes(sc, po, sr)
    return 1.0 / (npx * npy)


def pupil_image(hk, f, g, npx, npy):
    """Cropped spectrum with NaN outside the unit disc (Scatter.py:22-33)."""
    ny, nx = hk.shape[:2]
    pim = hk.copy()
    fm, gm = np.meshgrid(g, f, indexing='ij')
    pim[(fm * fm + gm * gm) > 1] = np.nan
    ox, oy = int(npx) + 3, int(npy) + 3
    return pim[(ny // 2) - oy:(ny // 2) + oy, (nx // 2) - ox:(nx // 2) + ox]


# ------------------------------------------------------------------------------------------ pupil terms
_ZERNIKE = (  # (m, trig, ((power, coefficient), ...)) for Fringe Z1..Z37 (Projection.py:356-434)
    (0, 0, ((0, 1),)), (1, 1, ((1, 1),)), (1, -1, ((1, 1),)), (0, 0, ((2, 2), (0, -1))),
    (2, 1, ((2, 1),)), (2, -1, ((2, 1),)), (1, 1, ((3, 3), (1, -2))), (1, -1, ((3, 3), (1, -2))),
    (0, 0, ((4, 6), (2, -6), (0, 1))), (3, 1, ((3, 1),)), (3, -1, ((3, 1),)),
    (2, 1, ((4, 4), (2, -3))), (2, -1, ((4, 4), (2, -3))),
    (1, 1, ((5, 10), (3, -12), (1, 3))), (1, -1, ((5, 10), (3, -12), (1, 3))),
    (0, 0, ((6, 20), (4, -30), (2, 12), (0, -1))), (4, 1, ((4, 1),)), (4, -1, ((4, 1),)),
    (3, 1, ((5, 5), (3, -4))), (3, -1, ((5, 5), (3, -4))),
    (2, 1, ((6, 15), (4, -20), (2, 6))), (2, -1, ((6, 15), (4, -20), (2, 6))),
    (1, 1, ((7, 35), (5, -60), (3, 30), (1, -4))), (1, -1, ((7, 35), (5, -60), (3, 30), (1, -4))),
    (0, 0, ((8, 70), (6, -140), (4, 90), (2, -20), (0, 1))), (5, 1, ((5, 1),)), (5, -1, ((5, 1),)),
    (4, 1, ((6, 6), (4, -5))), (4, -1, ((6, 6), (4, -5))),
    (3, 1, ((7, 21), (5, -30), (3, 10))), (3, -1, ((7, 21), (5, -30), (3, 10))),
    (2, 1, ((8, 56), (6, -105), (4, 60), (2, -10))), (2, -1, ((8, 56), (6, -105), (4, 60), (2, -10))),
    (1, 1, ((9, 126), (7, -280), (5, 210), (3, -60), (1, 5))),
    (1, -1, ((9, 126), (7, -280), (5, 210), (3, -60), (1, 5))),
    (0, 0, ((10, 252), (8, -630), (6, 560), (4, -210), (2, 30), (0, -1))),
    (0, 0, ((12, 924), (10, -2772), (8, 3150), (6, -1680), (4, 420), (2, -42), (0, 1))),
)


def aberration(coef, rho, theta):
    """Fringe Zernike phase in waves, float64 (Projection.py:13-128, Orientation = 0)."""
    coef = np.asarray(coef, dtype=np.float64)
    out = np.full(np.shape(rho), coef[0], dtype=np.float64)
    for i in range(1, 37):
        if coef[i] == 0:
            continue
        m, trig, poly = _ZERNIKE[i]
        rad = sum(c * rho ** p for p, c in poly)
        if trig == 1:
            rad = rad * np.cos(m * theta)
        elif trig == -1:
            rad = rad * np.sin(m * theta)
        out = out + coef[i] * rad
    return out


def char_matrix(f, g, NA, n):
    """Polarisation transfer Mxx, Myx, Mxy, Myy, Mxz, Myz (CalculateCharacteristicMatrix.py:3-17)."""
    a = (NA / n) * np.asarray(f, dtype=np.complex128)
    b = (NA / n) * np.asarray(g, dtype=np.complex128)
    gam = np.sqrt(1 - a * a - b * b)
    mxx = 1 - a * a / (1 + gam)
    myx = -a * b / (1 + gam)
    myy = 1 - b * b / (1 + gam)
    return mxx, myx, myx, myy, -a, -b


def polarization_states(sr, X, Y):
    """Jones vectors per source point, one (Px[S], Py[S]) complex128 pair per incoherent polarisation state.

    * The reference: the constant PolarizationVector (Source.py:222-226), one state.
    * PolarizationType set: the typed map whose formulas Source.py:185-217 keeps unused -- x (1, 0), y (0, 1),
      c (1, i)/sqrt 2, d (1, 1)/sqrt 2, r (cos t, sin t), t (sin t, -cos t), line (sin a, cos a) with
      (rho, t) = polar(X, Y) in float64 and points with rho below the float64 epsilon set to (0, 0); 'custom' is
      the PolarizationVector.
    * PolarizationParameters.CoherencyMatrix J set (README.md:45): J = sum_i l_i e_i e_i^H, states sqrt(l_i) e_i
      (l_i above 1e-12 of the largest), whose intensities add.
    """
    S = len(X)
    J = getattr(getattr(sr, 'PolarizationParameters', None), 'CoherencyMatrix', None)
    if J is not None:
        m = np.asarray(J, dtype=np.complex128).reshape(2, 2)
        lam, U = np.linalg.eigh(m)
        top = float(np.max(lam))
        return [(np.full(S, math.sqrt(lam[i]) * U[0, i]), np.full(S, math.sqrt(lam[i]) * U[1, i]))
                for i in range(2) if lam[i] > 1e-12 * top]
    kind = getattr(sr, 'PolarizationType', None)
    if kind is None or kind == 'custom':
        px, py = (complex(v) for v in sr.PolarizationVector)
        return [(np.full(S, px), np.full(S, py))]
    x, y = np.asarray(X, np.float64), np.asarray(Y, np.float64)
    rho, t = np.sqrt(x * x + y * y), np.arctan2(y, x)
    one, h = np.ones(S, np.complex128), math.sqrt(0.5)
    a = float(np.asarray(sr.PolarizationParameters.Angle))
    px, py = {'x_pol': (one, 0 * one), 'y_pol': (0 * one, one), 'c_pol': (h * one, 1j * h * one),
              'd_pol': (h * one, h * one), 'r_pol': (np.cos(t) + 0j, np.sin(t) + 0j),
              't_pol': (np.sin(t) + 0j, -np.cos(t) + 0j), 'line_pol': (math.sin(a) * one, math.cos(a) * one)}[kind]
    small = rho < np.finfo(np.float64).eps
    px, py = px.copy(), py.copy()
    px[small] = 0
    py[small] = 0
    return [(px, py)]


def _pupil(po, sr, rho2, focus):
    """obliquity * exp(2 pi i W) * defocus at squared radius rho2 (CalculateAerialImage.py:64-67)."""
    NA, M, n, lam = po.NA, po.Magnification, po.IndexImage, sr.Wavelength
    with np.errstate(invalid='ignore'):
        obl = np.power((1 - (NA / M) ** 2 * rho2) / (1 - NA ** 2 * rho2), 0.25)
        dz = np.exp(1j * 2 * np.pi / lam * np.sqrt(n ** 2 - (NA / M) ** 2 * rho2) * float(focus))
    return obl, dz


# ------------------------------------------------------------------------------------------------- Abbe
def abbe(sr, sc, po, nm, chunk=None, points=None):
    """Abbe aerial image [nFocus, Ny, Nx], float64 (CalculateAerialImage.py:18-103).  Source points are
    transformed `chunk` at a time (default: about 1 GB of fields per stack).

    With `points` (source-point indices) it also returns {j: A_j}, A_j [nFocus, Ny, Nx] the unweighted intensity
    of point j, dfdg^2 fftshift(sum over channels and field components |E|^2), so that the image is
    n / sum(v) * sum_j v_j A_j (CalculateAerialImage.py:86-92) -- what a source-weight derivative needs."""
    X, Y, V = source_points(sr)
    hk, f, g = spectrum(sc, po, sr)
    ny, nx, nch = hk.shape
    if chunk is None:
        chunk = max(1, min(64, (1 << 30) // (16 * ny * nx * 3 * max(1, nch))))
    W = float(np.sum(V.astype(np.float64)))
    vector = nm.ImageCalculationMode.lower() == 'vector'
    ne = 3 if vector else 1
    dfdg = _cell_area(sc, po, sr)
    # float32 pupil membership test, same operation order as CalculateAerialImage.py:43-57
    fm32, gm32 = np.meshgrid(g, f, indexing='ij')
    fg2 = fm32 * fm32 + gm32 * gm32
    fm64, gm64 = fm32.astype(np.float64), gm32.astype(np.float64)
    live = [c for c in range(nch) if np.any(hk[:, :, c] != 0)]
    focus_range = np.atleast_1d(np.asarray(po.FocusRange, dtype=np.float64))
    states = polarization_states(sr, X, Y) if vector else [None]
    out = np.zeros((len(focus_range), ny, nx))
    keep = {int(j): np.zeros((len(focus_range), ny, nx)) for j in (points if points is not None else ())}
    for iz, z in enumerate(focus_range):
        acc = np.zeros((ny, nx))
        for j0 in range(0, len(V), chunk):
            js = range(j0, min(j0 + chunk, len(V)))
            fields = []
            wts = []
            owner = []
            for j in js:
                rho2_32 = (fg2 + F32(2) * (X[j] * fm32 + Y[j] * gm32)) + (X[j] * X[j] + Y[j] * Y[j])
                valid = rho2_32 <= 1
                fc = fm64[valid] + float(X[j])
                gc = gm64[valid] + float(Y[j])
                r2 = fc * fc + gc * gc
                obl, dz = _pupil(po, sr, r2, z)
                ab = aberration(po.Aberration_Zernike, np.sqrt(r2), np.arctan2(gc, fc))
                P = obl * np.exp(1j * 2 * np.pi * ab) * dz
                comps = []
                if vector:
                    mxx, myx, mxy, myy, mxz, myz = char_matrix(fc, gc, po.NA, po.IndexImage)
                    for pxs, pys in states:   # one field set per polarisation state; intensities add
                        px, py = pxs[j], pys[j]
                        comps += [px * mxx + py * myx, px * mxy + py * myy, px * mxz + py * myz]
                else:
                    comps = [1.0]
                for c in live:
                    base = hk[:, :, c][valid] * P
                    for comp in comps:
                        fld = np.zeros((ny, nx), dtype=np.complex128)
                        fld[valid] = base * comp
                        fields.append(fld)
                        wts.append(float(V[j]))
                        owner.append(j)
            if fields:
                E2 = np.abs(_fft2(np.stack(fields), axes=(1, 2))) ** 2
                acc += np.tensordot(np.asarray(wts), E2, axes=(0, 0))
                for i, j in enumerate(owner):
                    if j in keep:
                        keep[j][iz] += dfdg ** 2 * np.fft.fftshift(E2[i])
        out[iz] = po.IndexImage / W * dfdg ** 2 * np.fft.fftshift(acc)
    return (out, keep) if points is not None else out


# ------------------------------------------------------------------------------------------------- TCC
def tcc_axes(sr, xypitch, po):
    """TCC frequency axes: f along rows (xypitch[0]) and g along columns (CalculateTCCMatrix.py:17-22)."""
    npf = F32(xypitch[0] / (sr.Wavelength / po.NA))
    npg = F32(xypitch[1] / (sr.Wavelength / po.NA))
    nf = int(np.ceil(F32(2) * npf))
    ng = int(np.ceil(F32(2) * npg))
    f = (F32(1) / npf) * np.arange(-nf, nf + 1).astype(F32)
    g = (F32(1) / npg) * np.arange(-ng, ng + 1).astype(F32)
    return f, g


def pupil_matrix(sr, xypitch, po, focus, nm):
    """Shifted pupil matrices [ncomp, FG, S] complex128 and weights (CalculateTCCMatrix.py:9-46)."""
    X, Y, V = source_points(sr)
    f, g = tcc_axes(sr, xypitch, po)
    ff, gg = np.meshgrid(f, g, indexing='ij')
    nf32 = ff.reshape(-1, 1) + X.reshape(1, -1)
    ng32 = gg.reshape(-1, 1) + Y.reshape(1, -1)
    valid = np.sqrt(nf32 * nf32 + ng32 * ng32) <= 1
    nf64 = ff.reshape(-1, 1).astype(np.float64) + X.reshape(1, -1).astype(np.float64)
    ng64 = gg.reshape(-1, 1).astype(np.float64) + Y.reshape(1, -1).astype(np.float64)
    r2 = nf64 * nf64 + ng64 * ng64
    P = np.zeros(r2.shape, dtype=np.complex128)
    obl, dz = _pupil(po, sr, r2[valid], focus)
    ab = aberration(po.Aberration_Zernike, np.sqrt(r2[valid]), np.arctan2(ng64[valid], nf64[valid]))
    P[valid] = obl * np.exp(1j * 2 * np.pi * ab) * dz
    if nm.ImageCalculationMode == 'vector':
        mxx, myx, mxy, myy, mxz, myz = char_matrix(nf64, ng64, po.NA, po.IndexImage)
        G = []
        for pxs, pys in polarization_states(sr, X, Y):   # per point (columns j); states stack as components
            px, py = pxs.reshape(1, -1), pys.reshape(1, -1)
            G += [(px * mxx + py * myx) * P, (px * mxy + py * myy) * P, (px * mxz + py * myz) * P]
        G = np.stack(G)
    else:
        G = P[None]
    return G, V.astype(np.float64), [len(g), len(f)]


def tcc(sr, xypitch, po, focus, nm):
    """TCC = n * sum_c G_c diag(w) G_c^H / sum(w), complex128 [FG, FG] (CalculateTCCMatrix.py:9-75)."""
    G, w, fg = pupil_matrix(sr, xypitch, po, focus, nm)
    T = np.zeros((G.shape[1], G.shape[1]), dtype=np.complex128)
    for Gc in G:
        T += (Gc * w[None, :]) @ Gc.conj().T
    return po.IndexImage * T / np.sum(w), fg


def socs_count(nm, evals, size):
    """Number of SOCS kernels kept (DecomposeTCC_SOCS.py:8-21).

    'threshold' is implemented as intended -- the smallest k whose leading eigenvalues reach the requested
    fraction of the trace -- because the reference's version raises on a multi-element comparison.
    """
    kind = nm.Hopkins_SettingType.lower()
    if kind == 'order':
        return min(nm.Hopkins_Order, size - 1)
    if kind == 'threshold':
        c = np.cumsum(evals)
        k = int(np.searchsorted(c, nm.Hopkins_Threshold * c[-1], side='right'))
        return min(k, size - 1)
    raise ValueError('Error: Hopkins_SettingType should be order or threshold!')


def decompose(T, fg, nfg, nm):
    """SOCS kernels sqrt(lambda_k) u_k embedded centred and fftshifted, complex128 [Ny, Nx, K].

    DecomposeTCC_SOCS.py:3-37 with a Hermitian eigendecomposition (eigenvalues descending, clamped at 0)
    instead of the SVD; for a Hermitian PSD matrix the two agree up to the phase of each vector.
    """
    nf, ng = nfg
    lam, U = np.linalg.eigh(T)
    lam, U = lam[::-1], U[:, ::-1]
    lam = np.maximum(lam, 0)
    k = socs_count(nm, lam, U.shape[1])
    out = np.zeros((ng, nf, k), dtype=np.complex128)
    tmp = np.zeros((ng, nf), dtype=np.complex128)
    r0, c0 = (ng - fg[1] + 1) // 2, (nf - fg[0] + 1) // 2
    for i in range(k):
        tmp[r0:r0 + fg[1], c0:c0 + fg[0]] = U[:, i].reshape(fg[1], fg[0])
        out[:, :, i] = np.fft.fftshift(tmp)
    return out * np.sqrt(lam[:k]).reshape(1, 1, -1)


def socs(sc, kernels, sr, po):
    """SOCS aerial image [Ny, Nx] float64 (CalculateAerialImage_SOCS.py:3-11)."""
    hk, f, g = spectrum(sc, po, sr)
    ny, nx, nch = hk.shape
    dfdg = _cell_area(sc, po, sr)
    sp = np.fft.ifftshift(hk, axes=(0, 1))
    acc = np.zeros((ny, nx))
    for c in range(nch):
        if not np.any(sp[:, :, c] != 0):
            continue
        for k in range(kernels.shape[2]):
            E = dfdg * _fft2(kernels[:, :, k] * sp[:, :, c])
            acc += np.abs(E) ** 2
    return np.fft.fftshift(acc)


def socs_resist(logits, target, kernels, a, thr):
    """SOCS image of the mask sigmoid(logits) (CalculateAerialImage_SOCS.py:3-11, one live channel), the resist
    loss L = sum (sigmoid(a (I - thr)) - target)^2 and its exact gradient dL/dlogits, all float64.

    The gradient is the chain rule through the reference's own operations -- what torch autograd computes
    through them -- restated: with u = ifftshift(t), E_k = fft2(K_k .* ifft2(u)) (the npx npy and df dg factors
    of Scatter.py:20 and CalculateAerialImage_SOCS.py:7 cancel), I = fftshift(sum_k |E_k|^2) and
    gA = ifftshift(dL/dI), the adjoint of fft2 being N^2 ifft2 gives
        dL/du = 2 sum_k Re fft2(conj(K_k) .* ifft2(gA .* E_k)),   dL/dt = fftshift(dL/du),
    and dL/dlogits = dL/dt * t (1 - t).  Returns (I, L, grad)."""
    l = np.asarray(logits, dtype=np.float64)
    t = 1.0 / (1.0 + np.exp(-l))
    d = _ifft2(np.fft.ifftshift(t))
    K = np.asarray(kernels)
    E = [_fft2(K[:, :, k] * d) for k in range(K.shape[2])]
    acc = np.zeros(t.shape)
    for e in E:
        acc += e.real ** 2 + e.imag ** 2
    I = np.fft.fftshift(acc)
    s = 1.0 / (1.0 + np.exp(-a * (I - thr)))
    r = s - np.asarray(target, dtype=np.float64)
    loss = float(np.sum(r * r))
    gA = np.fft.ifftshift(2.0 * r * a * s * (1.0 - s))
    du = np.zeros(t.shape)
    for k, e in enumerate(E):
        du += 2.0 * _fft2(np.conj(K[:, :, k]) * _ifft2(gA * e)).real
    return I, loss, np.fft.fftshift(du) * t * (1.0 - t)


def socs_pixel_fields(kernels):
    """F_k = fft2(K_k) / N^2: changing the mask t at pixel p by delta changes E_k by delta * roll(F_k, q), with
    q = ifftshift's image of p (so E_k(x) + delta F_k(x - q)) -- the exact single-pixel update of the SOCS
    fields, for finite differences without recomputing every transform."""
    K = np.asarray(kernels)
    n = K.shape[0] * K.shape[1]
    return [_fft2(K[:, :, k]) / n for k in range(K.shape[2])]


def hopkins(sr, sc, po, nm):
    """Hopkins image [nFocus, Ny, Nx]: TCC -> SOCS kernels -> image per plane (CalculateAerialImage.py:105-130)."""
    ny, nx = np.asarray(sc.ScatterField).shape[:2]
    zs = np.atleast_1d(np.asarray(po.FocusRange, dtype=np.float64))
    out = np.zeros((len(zs), ny, nx))
    for i, z in enumerate(zs):
        T, fg = tcc(sr, [sc.Period_Y, sc.Period_X], po, z, nm)
        K = decompose(T, fg, [nx, ny], nm)
        out[i] = socs(sc, K, sr, po)
    return out


def socs_floquet(floquet, kernels, nm):
    """Direct-DFT SOCS image from Floquet modes [Gx, Gy] (CalculateAerialImage_SOCS.py:13-32)."""
    gx, gy = nm.ScatterGrid_X, nm.ScatterGrid_Y
    xa = ((np.arange(gx) + 0.5) / gx).reshape(-1, 1, 1)
    ya = ((np.arange(gy) + 0.5) / gy).reshape(1, -1, 1)
    ox = np.arange(-nm.ScatterOrder_X, nm.ScatterOrder_X + 1)
    oy = np.arange(-nm.ScatterOrder_Y, nm.ScatterOrder_Y + 1)
    oxg, oyg = np.meshgrid(ox, oy, indexing='ij')
    ph = np.exp(2j * np.pi * (oxg.reshape(-1) * xa + oyg.reshape(-1) * ya))[..., None, None]
    fm = np.asarray(floquet, dtype=np.complex128).reshape(1, 1, -1, 3, 1)
    kt = np.fft.ifftshift(np.transpose(np.asarray(kernels), (1, 0, 2)), axes=(0, 1))
    kt = kt.reshape(1, 1, -1, 1, kernels.shape[2])
    S = np.sum(ph * fm * kt, axis=2)
    return np.sum(np.abs(S) ** 2, axis=(2, 3))
