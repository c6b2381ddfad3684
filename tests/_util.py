"""Shared helpers for the parity tests."""

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + '.npz')))


def rel(a, b):
    """Normwise relative difference ||a - b|| / ||b||."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def interior(a, g):
    return a[g:a.shape[0] - g, g:a.shape[1] - g]


def moment_errors(m_test, m_ref):
    """Moments compared normwise, momenta scaled by the density norm (their
    own norm can be ~0 for symmetric distributions)."""
    scale = np.linalg.norm(m_ref['density'].ravel())
    out = {}
    for k in m_ref:
        denom = max(np.linalg.norm(m_ref[k].ravel()), scale)
        out[k] = float(np.linalg.norm((np.asarray(m_test[k]) - m_ref[k]).ravel()) / denom)
    return out
