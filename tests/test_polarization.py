"""Polarisation beyond the constant Jones vector: the typed maps of Calc_PolarizationMap (Source.py:183-221, whose
formulas the reference keeps unused) and the CoherencyMatrix of PolarizationParameters (README.md:45, not in the
reference's code).  CPU: identities of the FP64 oracle and of the host-side states.  GPU: the engine against the
oracle at 1e-5 of peak, and a rank-1 coherency matrix against the Jones-vector path."""
import math

import numpy as np
import pytest
import torch

from oracle import optics64 as O
from opticalimaging_b200.params import coherency_states, polarization_map
from tests.fixtures import build, load, rel_err


def _case(kind=None, J=None, pol=(1.0, 0.0)):
    meta, a = load('vec_small')
    sr, sc, po, nm = build(meta, a)
    sr.PolarizationVector = list(pol)
    sr.PolarizationType = kind
    sr.PolarizationParameters.CoherencyMatrix = J
    return sr, sc, po, nm


def test_typed_maps_match_the_documented_formulas():
    th = torch.tensor([0.0, 0.5, -2.0, 3.0], dtype=torch.float64)
    rho = torch.tensor([0.0, 0.3, 0.9, 1.0], dtype=torch.float64)
    px, py = polarization_map('r_pol', th, rho)
    assert px[0] == 0 and py[0] == 0                      # on-axis point: (0, 0)
    np.testing.assert_allclose(px[1:].real.numpy(), np.cos(th[1:].numpy()))
    np.testing.assert_allclose(py[1:].real.numpy(), np.sin(th[1:].numpy()))
    px, py = polarization_map('t_pol', th, rho)
    np.testing.assert_allclose(py[1:].real.numpy(), -np.cos(th[1:].numpy()))
    px, py = polarization_map('c_pol', th, rho)
    assert torch.allclose(py[1:], 1j * px[1:]) and abs(abs(px[1]) - math.sqrt(0.5)) < 1e-15
    with pytest.raises(ValueError, match='unsupported polarization type'):
        polarization_map('e_pol', th, rho)


def test_coherency_states():
    j = torch.tensor([0.6, 0.8j], dtype=torch.complex128)
    st = coherency_states(torch.outer(j, j.conj()))
    assert len(st) == 1 and abs(abs(torch.vdot(st[0], j)) - 1.0) < 1e-12    # j up to a phase
    st = coherency_states(0.5 * torch.eye(2))
    assert len(st) == 2 and all(abs(float(torch.vdot(s, s).real) - 0.5) < 1e-12 for s in st)
    with pytest.raises(ValueError, match='Hermitian'):
        coherency_states(torch.tensor([[1.0, 1.0], [0.0, 1.0]]))
    with pytest.raises(ValueError, match='semi-definite'):
        coherency_states(torch.tensor([[1.0, 0.0], [0.0, -0.5]]))


def test_oracle_coherency_identities():
    """Rank 1 equals the Jones vector it is made of; unpolarised light (J = I/2) is the mean of x and y
    polarised images (for both imaging paths' pupil matrices, through the Abbe image and the TCC)."""
    j = np.array([0.6, 0.8j])
    ref = O.abbe(*_case(pol=tuple(j)))
    got = O.abbe(*_case(J=np.outer(j, j.conj())))
    assert rel_err(got, ref) < 1e-12
    un = O.abbe(*_case(J=0.5 * np.eye(2)))
    mean = 0.5 * (O.abbe(*_case(pol=(1.0, 0.0))) + O.abbe(*_case(pol=(0.0, 1.0))))
    assert rel_err(un, mean) < 1e-12
    sr, sc, po, nm = _case(J=0.5 * np.eye(2))
    T, _ = O.tcc(sr, [sc.Period_Y, sc.Period_X], po, 0.0, nm)
    Tx, _ = O.tcc(*(lambda c: (c[0], [c[1].Period_Y, c[1].Period_X], c[2], 0.0, c[3]))(_case(pol=(1.0, 0.0))))
    Ty, _ = O.tcc(*(lambda c: (c[0], [c[1].Period_Y, c[1].Period_X], c[2], 0.0, c[3]))(_case(pol=(0.0, 1.0))))
    assert rel_err(T, 0.5 * (Tx + Ty)) < 1e-12
    # a typed constant map equals the constant vector
    assert rel_err(O.abbe(*_case(kind='y_pol')), O.abbe(*_case(pol=(0.0, 1.0)))) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize('kind,J', [('r_pol', None), ('t_pol', None), (None, 'unpolarised'), (None, 'elliptic')])
def test_engine_polarisation_vs_oracle(kind, J, report):
    from opticalimaging_b200 import imaging
    Jm = {None: None, 'unpolarised': 0.5 * np.eye(2),
          'elliptic': np.array([[0.7, 0.2 + 0.1j], [0.2 - 0.1j, 0.3]])}[J]
    sr, sc, po, nm = _case(kind=kind, J=Jm)
    img, _ = imaging.CalculateAbbeImage(sr, sc, po, nm)
    ref = O.abbe(*_case(kind=kind, J=Jm))
    nm.Hopkins_Order = 10 ** 6      # untruncated: no eigenvalue cut that a degenerate pair could straddle
    h, _ = imaging.CalculateHopkinsImage(sr, sc, po, nm)
    href = O.hopkins(sr, sc, po, nm)
    report(f'polarisation_{kind or J}', abbe_vs_fp64=rel_err(img.Intensity.numpy(), ref),
           hopkins_vs_fp64=rel_err(h.Intensity.numpy(), href))
    assert rel_err(img.Intensity.numpy(), ref) < 1e-5
    assert rel_err(h.Intensity.numpy(), href) < 1e-5


@pytest.mark.gpu
def test_engine_rank1_coherency_equals_jones_path():
    from opticalimaging_b200 import imaging
    j = np.array([0.6, 0.8j])
    a, _ = imaging.CalculateAbbeImage(*_case(pol=tuple(j)))
    b, _ = imaging.CalculateAbbeImage(*_case(J=np.outer(j, j.conj())))
    assert rel_err(b.Intensity.numpy(), a.Intensity.numpy()) < 1e-6
