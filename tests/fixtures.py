"""Loading of the golden fixtures and the seeded parameter sets used across the tests."""
import json
import os

import numpy as np
import torch

from opticalimaging_b200.params import Numerics, Projection, Scatter, Source

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
LAM, NA, N_IMG = 193.0, 1.35, 1.44


def load(name):
    z = np.load(os.path.join(GOLDEN, f'ref_{name}.npz'))
    meta = json.loads(str(z['meta']))
    return meta, {k: z[k] for k in z.files if k != 'meta'}


def make_source(p):
    sr = Source()
    for k, v in p.items():
        if k == 'PolarizationVector':
            v = [complex(x) if isinstance(x, str) else x for x in v]
            v = [x.real if isinstance(x, complex) and x.imag == 0 else x for x in v]
        setattr(sr, k, v)
    return sr


def build(meta, arrays):
    """(Source, Scatter, Projection, Numerics) for an imaging fixture."""
    sr = make_source(meta['src'])
    po = Projection()
    po.NA, po.IndexImage, po.Magnification = meta['NA'], meta['IndexImage'], meta['Magnification']
    po.FocusRange = torch.tensor(meta['focus'])
    po.Aberration_Zernike = torch.from_numpy(arrays['zernike'])
    nm = Numerics()
    nm.ImageCalculationMode = 'vector' if meta['vector'] else 'scalar'
    if 'hopkins_order' in meta:
        nm.Hopkins_SettingType, nm.Hopkins_Order = 'order', meta['hopkins_order']
    sc = Scatter()
    sc.Period_X, sc.Period_Y = meta['Period_X'], meta['Period_Y']
    sc.ScatterField = torch.from_numpy(arrays['field'])
    return sr, sc, po, nm


def rel_err(a, b):
    """max |a - b| / max |b|: error relative to the peak of the reference image."""
    a, b = np.asarray(a), np.asarray(b)
    dt = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a, b = a.astype(dt), b.astype(dt)
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def cfg4_kernels(meta, arrays, dtype=np.complex128):
    """The reference's SOCS-16 kernels of the configuration-4 fixture on the full [n, n, 16] grid (the fixture keeps
    only their band rows and columns)."""
    n = meta['n']
    k = arrays['kernels_band']
    out = np.zeros((n, n, k.shape[2]), dtype=dtype)
    out[np.ix_(arrays['kernel_rows'], arrays['kernel_cols'])] = k
    return out
