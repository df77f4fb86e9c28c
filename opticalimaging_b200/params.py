"""Parameter objects of the aerial-image path, kept call-compatible with the reference.

The reference describes an imaging run with four mutable attribute bags -- ``Source``, ``Projection``,
``Numerics`` and ``Scatter`` -- and returns ``ImageData``.  User code builds them attribute by attribute,
so the engine keeps the same class names, attribute names and defaults:

* ``Numerics``   -- Numerics.py:1-15
* ``Source``     -- Source.py:15-54 (defaults), 64-180 (shape rasterisers), 183-226 (polarisation)
* ``Projection`` -- Projection.py:4-10 (defaults), 13-128 (Fringe Zernike), 130-161 (rotation)
* ``Scatter``    -- Scatter.py:3-8 (defaults), 10-35 (spectrum)
* ``ImageData``  -- CalculateAerialImage.py:7-11

Source synthesis stays on the host in float32 torch, in the same operation order as the reference, because
the set of source points is decided by float32 comparisons (``Radius <= SigmaOut`` and friends) and must come
out bit-identical for the images to agree.  It runs once per request and costs microseconds.

Divergences, all deliberate:

* ``Calc_SourceSimple`` returns a fresh ``SourceData`` instance.  The reference stores the result on the
  *class* ``SourceData`` (Source.py:293-295) and returns the class, which is not re-entrant.
* ``Scatter.CalculateSpectrum`` runs on the GPU through the native band-spectrum kernel.
"""
from __future__ import annotations

import math
import sys

import torch
import torch.nn.functional as F

__all__ = [
    "Numerics", "Source", "SourceData", "PolarizationParameters", "Projection", "Scatter", "ImageData",
    "CalculateAnnularSourceMatrix", "CalculateQuasarSourceMatrix", "CalculateDipoleSourceMatrix",
    "CalculateMultiCircSourceMatrix", "ConvertSourceMatrix2SourceData", "cartesian_to_polar",
]


def cartesian_to_polar(x, y):
    """(rho, theta) of Cartesian pupil coordinates (CalculateAerialImage.py:13-16)."""
    return torch.sqrt(x ** 2 + y ** 2), torch.atan2(y, x)


class Numerics:
    """Numerical settings (Numerics.py:1-15).  Class attributes, as in the reference."""
    ImageCalculationMode: str = 'scalar'        # 'scalar' | 'vector'
    ImageCalculationMethod: str = 'hopkins'     # 'abbe' | 'hopkins' | 'optimized'
    Hopkins_SettingType: str = 'order'          # 'order' | 'threshold'
    Hopkins_Order: int = 100
    Hopkins_Threshold: float = 0.95
    ScatterGrid_X: int = 100
    ScatterGrid_Y: int = 100
    ScatterOrder_X: int = 15
    ScatterOrder_Y: int = 15

    def __init__(self):
        pass


class ImageData:
    """Aerial image container (CalculateAerialImage.py:7-11): Intensity [nFocus, Ny, Nx] and axes."""
    Intensity: torch.Tensor = None
    ImageX: torch.Tensor = None
    ImageY: torch.Tensor = None
    ImageZ: torch.Tensor = None


class SourceData:
    """Source samples: X, Y, Value (Source.py:299-303)."""

    def __init__(self, x, y):
        self.X = torch.zeros((x, y))
        self.Y = torch.zeros((x, y))
        self.Value = torch.zeros((x, y))


class PolarizationParameters:
    """Polarisation parameters (Source.py:305-308), plus the CoherencyMatrix the reference documents (README.md:45)
    but does not implement: a 2 x 2 Hermitian positive semi-definite matrix J = <E E^H> of the illumination's
    (Ex, Ey).  None (the default) keeps the Jones-vector polarisation."""

    def __init__(self):
        self.Degree = 1
        self.Angle = torch.tensor(0)
        self.CoherencyMatrix = None


POLARIZATION_TYPES = ('x_pol', 'y_pol', 'c_pol', 'd_pol', 'r_pol', 't_pol', 'line_pol', 'custom')


def polarization_map(kind, theta, rho, vector=(1.0, 0.0), angle=0.0):
    """Jones vector (Px, Py) per source point, complex128, for a polarisation type (README.md:41; the formulas of
    Source.py:185-217, which the reference keeps as an unused string): x_pol (1, 0), y_pol (0, 1), c_pol
    (1, i)/sqrt 2, d_pol (1, 1)/sqrt 2, r_pol (cos theta, sin theta), t_pol (sin theta, -cos theta), line_pol
    (sin Angle, cos Angle); 'custom' is the constant PolarizationVector.  Points with rho below the float64
    epsilon get (0, 0), as there."""
    theta = torch.as_tensor(theta, dtype=torch.float64)
    rho = torch.as_tensor(rho, dtype=torch.float64)
    one = torch.ones_like(theta, dtype=torch.complex128)
    h = math.sqrt(0.5)
    if kind == 'x_pol':
        px, py = one, 0 * one
    elif kind == 'y_pol':
        px, py = 0 * one, one
    elif kind == 'c_pol':
        px, py = h * one, 1j * h * one
    elif kind == 'd_pol':
        px, py = h * one, h * one
    elif kind == 'r_pol':
        px, py = torch.cos(theta).to(torch.complex128), torch.sin(theta).to(torch.complex128)
    elif kind == 't_pol':
        px, py = torch.sin(theta).to(torch.complex128), -torch.cos(theta).to(torch.complex128)
    elif kind == 'line_pol':
        a = float(angle)
        px, py = math.sin(a) * one, math.cos(a) * one
    elif kind == 'custom':
        px, py = complex(vector[0]) * one, complex(vector[1]) * one
    else:
        raise ValueError("unsupported polarization type")
    if kind != 'custom':
        small = rho < sys.float_info.epsilon
        px, py = px.clone(), py.clone()
        px[small] = 0
        py[small] = 0
    return px, py


def coherency_states(J):
    """The coherency matrix as <= 2 Jones vectors whose intensities add: J = sum_i lambda_i e_i e_i^H, state i =
    sqrt(lambda_i) e_i (eigenvalues below 1e-12 of the largest dropped).  A rank-1 J = j j^H gives j back (up to a
    phase, which no intensity sees); J = I / 2 (unpolarised) gives two orthogonal states of weight 1/2."""
    m = torch.as_tensor(J, dtype=torch.complex128).reshape(2, 2)
    if not torch.allclose(m, m.conj().T, rtol=1e-9, atol=1e-12):
        raise ValueError('CoherencyMatrix must be Hermitian')
    lam, U = torch.linalg.eigh(m)
    if float(lam.min()) < -1e-9 * max(1.0, float(lam.max())):
        raise ValueError('CoherencyMatrix must be positive semi-definite')
    top = float(lam.max())
    return [(math.sqrt(float(lam[i])) * U[:, i]) for i in range(2) if float(lam[i]) > 1e-12 * top]


def _grid(coord):
    s = SourceData(len(coord), len(coord))
    s.X, s.Y = torch.meshgrid(coord, coord, indexing='ij')
    return s


def CalculateAnnularSourceMatrix(SigmaOut, SigmaIn, Source_Coordinate_X, Source_Coordinate_Y):
    """Annulus SigmaIn <= r <= SigmaOut, uniform weight 1/(pi (so^2 - si^2)) (Source.py:229-238)."""
    s = _grid(Source_Coordinate_X)
    r = torch.sqrt(s.X.pow(2) + s.Y.pow(2))
    s.Value[(r <= SigmaOut) & (r >= SigmaIn)] = 1.0 / ((SigmaOut ** 2 - SigmaIn ** 2) * math.pi)
    return s


def CalculateQuasarSourceMatrix(SigmaOut, SigmaIn, openAngle, Source_Coordinate_X, Source_Coordinate_Y):
    """Four poles on the axes, each openAngle wide (Source.py:240-256)."""
    s = _grid(Source_Coordinate_X)
    r = torch.sqrt(s.X.pow(2) + s.Y.pow(2))
    th = torch.atan2(s.Y, s.X)
    half = openAngle / 2
    on_x = (torch.abs(th) <= half) | ((torch.abs(th) >= (math.pi - half)) & (torch.abs(th) <= math.pi))
    on_y = (torch.abs(th - math.pi / 2) <= half) | (torch.abs(th + math.pi / 2) <= half)
    s.Value[(r <= SigmaOut) & (r >= SigmaIn) & (on_x | on_y)] = 0.5 / ((SigmaOut ** 2 - SigmaIn ** 2) * openAngle)
    return s


def CalculateDipoleSourceMatrix(SigmaOut, SigmaIn, openAngle, rotateAngle, Source_Coordinate_X,
                                Source_Coordinate_Y):
    """Two poles along rotateAngle (Source.py:258-270)."""
    s = _grid(Source_Coordinate_X)
    r = torch.sqrt(s.X.pow(2) + s.Y.pow(2))
    th = torch.atan2(s.Y, s.X)
    in_pole = torch.abs(torch.cos(th - rotateAngle)) >= math.cos(openAngle / 2)
    s.Value[(r <= SigmaOut) & (r >= SigmaIn) & in_pole] = 1.0 / ((SigmaOut ** 2 - SigmaIn ** 2) * openAngle)
    return s


def CalculateMultiCircSourceMatrix(SigmaCenter, SigmaRadius, PoleNumber, RotateAngle, Source_Coordinate_X,
                                   Source_Coordinate_Y):
    """PoleNumber discs of radius SigmaRadius on a circle of radius SigmaCenter (Source.py:273-286)."""
    s = _grid(Source_Coordinate_X)
    step = 2 * math.pi / PoleNumber
    for i in range(PoleNumber):
        xc = SigmaCenter * math.cos(RotateAngle + i * step)
        yc = SigmaCenter * math.sin(RotateAngle + i * step)
        s.Value[((s.X - xc).pow(2) + (s.Y - yc).pow(2)) <= SigmaRadius ** 2] = 1.0 / PoleNumber / (SigmaRadius ** 2)
    return s


def ConvertSourceMatrix2SourceData(s):
    """Zero samples outside the unit disc and flatten to [P*P, 1] columns (Source.py:288-297).

    Returns a new ``SourceData`` (the reference writes class attributes instead).
    """
    n = s.X.shape[0]
    s.Value[(s.X ** 2 + s.Y ** 2) > 1] = 0
    out = SourceData(0, 0)
    out.X = torch.reshape(s.X, (n * n, 1))
    out.Y = torch.reshape(s.Y, (n * n, 1))
    out.Value = torch.reshape(s.Value, (n * n, 1))
    return out


def _conv2_same(matr, ker):
    mx, my = matr.size()
    kx, ky = ker.size()
    out = F.conv2d(matr.reshape((1, 1, mx, my)), ker.reshape((1, 1, kx, ky)), padding='same')
    return out.reshape((mx, my))


class Source:
    """Illumination source (Source.py:15-226).

    Shapes: 'annular', 'quasar', 'dipolecirc', 'multipole', 'pixel'.  The polarisation is the constant Jones
    vector ``PolarizationVector`` (Source.py:222-226), as in the reference, unless one of two engine extensions is
    set: ``PolarizationType`` (None by default) selects a typed polarisation map per source point
    (``polarization_map``: the types README.md lists, whose formulas the reference keeps unused in
    Source.py:185-217), and ``PolarizationParameters.CoherencyMatrix`` (README.md:45) describes partially
    polarised light, imaged as the sum of its eigen-polarisations' intensities (``polarization_states``).
    """

    def __init__(self):
        self.PntNum = 81
        self.Wavelength = 365
        self.Shape = "annular"
        self.SigmaOut = 0.7
        self.SigmaIn = 0.1
        self.SigmaCenter = 0.5
        self.SigmaRadius = 0.1
        self.OpenAngle = math.pi / 6
        self.RotateAngle = 0
        self.PoleNumber = 2
        self.Source_Mask = None
        self.SPointX = torch.zeros(self.PntNum)
        self.SPointY = torch.zeros(self.PntNum)
        self.SPointValue = torch.zeros(self.PntNum)
        self.PSFEnable = False
        self.PSFSigma = 0.02
        self.PolarizationParameters = PolarizationParameters()
        self.source_data = SourceData(self.PntNum, self.PntNum)
        self.PolarizationVector = [1.0, 0.0]
        self.PolarizationType = None

    def Calc_SourceSimple(self):
        """Source samples with weight >= 1e-5, as 1-D float32 X, Y, Value (Source.py:47-54)."""
        d = self.Calc_SourceAll()
        keep = ~(d.Value < 1e-5)
        out = SourceData(0, 0)
        out.X, out.Y, out.Value = d.X[keep], d.Y[keep], d.Value[keep]
        self.source_data = out
        return out

    def Calc_SourceValid(self):
        """All samples with the weight zeroed outside the unit disc (Source.py:56-62)."""
        d = self.Calc_SourceAll()
        self.source_data.Value = torch.where((d.X.pow(2) + d.Y.pow(2)) > 1, 0, d.Value)
        return self.source_data

    def _check_rotate(self):
        if (self.RotateAngle > math.pi / 2) | (self.RotateAngle < -1 * math.pi / 2):
            raise ValueError('error: roate angle must be in the range of [-pi/2,pi/2] ')

    def Calc_SourceAll(self):
        """Rasterise the source on a PntNum x PntNum grid over [-1, 1]^2 (Source.py:64-180)."""
        coord = torch.linspace(-1, 1, self.PntNum)
        shape = self.Shape.lower()
        if shape == "pixel":
            n2 = self.PntNum ** 2
            if self.SPointX.numel() != n2:
                raise ValueError('Source Matrix Size X and difined PntNum are not matched ')
            if self.SPointY.numel() != n2:
                raise ValueError('Source Matrix Size Y and difined PntNum are not matched ')
            if self.SPointValue.numel() != n2:
                raise ValueError('Source Matrix Size Value and difined PntNum are not matched ')
            d = SourceData(0, 0)
            d.X, d.Y, d.Value = self.SPointX, self.SPointY, self.SPointValue
        elif shape == "annular":
            d = CalculateAnnularSourceMatrix(self.SigmaOut, self.SigmaIn, coord, coord)
        elif shape == "quasar":
            self._check_rotate()
            if (self.OpenAngle <= 0) | (self.OpenAngle >= math.pi / 2):
                raise ValueError('error: open angle must be in the range of [0,pi/2] ')
            d = CalculateQuasarSourceMatrix(self.SigmaOut, self.SigmaIn, self.OpenAngle, coord, coord)
        elif shape == "dipolecirc":
            self._check_rotate()
            if (self.OpenAngle < 0) | (self.OpenAngle > math.pi / 2):
                raise ValueError('error: open angle must be in the range of [0,pi/2] ')
            d = CalculateDipoleSourceMatrix(self.SigmaOut, self.SigmaIn, self.OpenAngle, self.RotateAngle,
                                            coord, coord)
        elif shape == "multipole":
            self._check_rotate()
            d = CalculateMultiCircSourceMatrix(self.SigmaCenter, self.SigmaRadius, self.PoleNumber,
                                               self.RotateAngle, coord, coord)
        else:
            raise ValueError("unsupported illumination")

        size_x, size_y = d.Value.size()
        if self.Source_Mask is not None:
            d.Value = torch.mul(d.Value, self.Source_Mask)
        if size_x == size_y:
            if self.PSFEnable:
                ksize = round(self.PntNum / 10) * 2 + 1
                kedge = 1 / (self.PntNum - 1) * (ksize - 1)
                kx, ky = torch.meshgrid(torch.linspace(-kedge, kedge, ksize),
                                        torch.linspace(-kedge, kedge, ksize), indexing='ij')
                ker = 1 / math.sqrt(2 * math.pi) / self.PSFSigma * torch.exp(
                    -(kx.pow(2) + ky.pow(2)) / self.PSFSigma ** 2)
                ker = ker[~torch.all(ker < 1e-6, 0)]
                ker_t = torch.transpose(ker, 0, 1)
                ker = ker_t[~torch.all(ker_t < 1e-6, 1)]
                ker = ker / torch.sum(ker)
                d.Value = _conv2_same(d.Value, ker)
            d.Value[int((size_x - 1) / 2), int((size_y - 1) / 2)] = 0
            d = ConvertSourceMatrix2SourceData(d)
        self.source_data = d
        return d

    def Calc_PolarizationMap(self, theta, rho):
        """Jones vector per source point, complex64: the constant PolarizationVector (Source.py:222-226), or the
        typed map of PolarizationType when one is set (``polarization_map``)."""
        if self.PolarizationType is None:
            px = (self.PolarizationVector[0] * torch.ones(theta.size())).to(torch.complex64)
            py = (self.PolarizationVector[1] * torch.ones(theta.size())).to(torch.complex64)
            return px, py
        px, py = polarization_map(self.PolarizationType, theta, rho, self.PolarizationVector,
                                  self.PolarizationParameters.Angle)
        return px.to(torch.complex64), py.to(torch.complex64)

    def polarization_states(self, X, Y):
        """The incoherent polarisation states the image sums over, each a per-point Jones array [S, 2]
        complex128, or None for 'the constant PolarizationVector' (one state, the reference's behaviour).  With a
        CoherencyMatrix: one constant state per eigen-polarisation (``coherency_states``); with a PolarizationType:
        one state from the typed map at the points' (theta, rho)."""
        J = self.PolarizationParameters.CoherencyMatrix
        n = torch.as_tensor(X).numel()
        if J is not None:
            return [torch.stack((st[0] * torch.ones(n, dtype=torch.complex128),
                                 st[1] * torch.ones(n, dtype=torch.complex128)), 1) for st in coherency_states(J)]
        if self.PolarizationType is None:
            return None
        rho, theta = cartesian_to_polar(torch.as_tensor(X).reshape(-1).double(), torch.as_tensor(Y).reshape(-1).double())
        px, py = polarization_map(self.PolarizationType, theta, rho, self.PolarizationVector,
                                  self.PolarizationParameters.Angle)
        return [torch.stack((px, py), 1)]


# Fringe Zernike Z1..Z37 as (m, trig, radial) -- Projection.py:356-434.  Each radial part is a
# polynomial in rho with the listed (power, coefficient) pairs; trig is 0 (none), 1 (cos m theta), -1 (sin).
FRINGE_ZERNIKE = (
    (0, 0, ((0, 1),)),
    (1, 1, ((1, 1),)), (1, -1, ((1, 1),)),
    (0, 0, ((2, 2), (0, -1))),
    (2, 1, ((2, 1),)), (2, -1, ((2, 1),)),
    (1, 1, ((3, 3), (1, -2))), (1, -1, ((3, 3), (1, -2))),
    (0, 0, ((4, 6), (2, -6), (0, 1))),
    (3, 1, ((3, 1),)), (3, -1, ((3, 1),)),
    (2, 1, ((4, 4), (2, -3))), (2, -1, ((4, 4), (2, -3))),
    (1, 1, ((5, 10), (3, -12), (1, 3))), (1, -1, ((5, 10), (3, -12), (1, 3))),
    (0, 0, ((6, 20), (4, -30), (2, 12), (0, -1))),
    (4, 1, ((4, 1),)), (4, -1, ((4, 1),)),
    (3, 1, ((5, 5), (3, -4))), (3, -1, ((5, 5), (3, -4))),
    (2, 1, ((6, 15), (4, -20), (2, 6))), (2, -1, ((6, 15), (4, -20), (2, 6))),
    (1, 1, ((7, 35), (5, -60), (3, 30), (1, -4))), (1, -1, ((7, 35), (5, -60), (3, 30), (1, -4))),
    (0, 0, ((8, 70), (6, -140), (4, 90), (2, -20), (0, 1))),
    (5, 1, ((5, 1),)), (5, -1, ((5, 1),)),
    (4, 1, ((6, 6), (4, -5))), (4, -1, ((6, 6), (4, -5))),
    (3, 1, ((7, 21), (5, -30), (3, 10))), (3, -1, ((7, 21), (5, -30), (3, 10))),
    (2, 1, ((8, 56), (6, -105), (4, 60), (2, -10))), (2, -1, ((8, 56), (6, -105), (4, 60), (2, -10))),
    (1, 1, ((9, 126), (7, -280), (5, 210), (3, -60), (1, 5))),
    (1, -1, ((9, 126), (7, -280), (5, 210), (3, -60), (1, 5))),
    (0, 0, ((10, 252), (8, -630), (6, 560), (4, -210), (2, 30), (0, -1))),
    (0, 0, ((12, 924), (10, -2772), (8, 3150), (6, -1680), (4, 420), (2, -42), (0, 1))),
)


class Projection:
    """Projection optics (Projection.py:4-161)."""

    def __init__(self):
        self.Aberration_Zernike = torch.zeros(37)
        self.Magnification = 100
        self.NA = 0.9
        self.IndexImage = 1.0
        self.FocusRange = torch.tensor([0])

    def CalculateAberrationFast(self, rho, theta, Orientation):
        """Fringe Zernike aberration in waves at (rho, theta) (Projection.py:13-128)."""
        if abs(Orientation) > sys.float_info.epsilon:
            coef = Projection.RotateAngle(self.Aberration_Zernike, Orientation)
        else:
            coef = self.Aberration_Zernike
        out = coef[0]
        for i in range(1, 37):
            m, trig, poly = FRINGE_ZERNIKE[i]
            radial = None
            for p, c in poly:
                term = c * (rho.pow(p) if p > 1 else (rho if p == 1 else torch.ones_like(rho)))
                radial = term if radial is None else radial + term
            if trig == 1:
                radial = torch.mul(radial, torch.cos(m * theta) if m > 1 else torch.cos(theta))
            elif trig == -1:
                radial = torch.mul(radial, torch.sin(m * theta) if m > 1 else torch.sin(theta))
            out = out + coef[i] * radial
        return out

    @staticmethod
    def RotateAngle(c0, theta):
        """Rotate Fringe Zernike coefficients by theta (Projection.py:130-161)."""
        m = torch.tensor([FRINGE_ZERNIKE[i][0] for i in range(37)])
        t = [FRINGE_ZERNIKE[i][1] for i in range(37)]
        # partner index: the sin twin of a cos term and vice versa; rotationally symmetric terms map to themselves
        partner = list(range(37))
        for i in range(37):
            if t[i] == 1:
                partner[i], partner[i + 1] = i + 1, i
        c1 = torch.zeros(37)
        for i in range(37):
            c1[i] = c1[i] + c0[i] * torch.cos(m[i] * theta)
            c1[partner[i]] = c1[partner[i]] - t[i] * c0[i] * torch.sin(m[i] * theta)
        return c1


class Scatter:
    """Mask near field and period (Scatter.py:3-35)."""

    def __init__(self):
        self.Period_X = 1000
        self.Period_Y = 1000
        self.ScatterField = []
        self.FloquetMode = []

    def CalculateSpectrum(self, po, sr):
        """Centred, pitch-scaled spectrum Hk [Ny, Nx, 3], the f/g axes and the cropped pupil diagnostic.

        Same contract as Scatter.py:10-35.  Hk is computed on the GPU by the native band-spectrum kernel.
        """
        from .imaging import calculate_spectrum
        return calculate_spectrum(self, po, sr)
