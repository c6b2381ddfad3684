"""Shared helpers for the parity tests."""

import os

import numpy as np

import cases as C

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


MOMENTS = ('density', 'mom_v1_bulk', 'mom_v2_bulk', 'mom_v3_bulk', 'energy')


def _qsum_errors(spec, got, ref):
    """Per-column normwise errors of C.qcell_sums arrays; the velocity-weighted
    columns are scaled by at least the column-0 norm times |p|max (resp. its
    square), because their own norms can vanish for symmetric data."""
    vmax = max(abs(spec['p1_start'][0]), abs(spec['p1_end'][0]))
    n0 = np.linalg.norm(ref[..., 0])
    scale = [n0, n0 * vmax, n0 * vmax, n0 * vmax, n0 * vmax ** 2, 0.0]
    out = []
    for c in range(6):
        d = max(np.linalg.norm(ref[..., c]), scale[c], 1e-300)
        out.append(float(np.linalg.norm(got[..., c] - ref[..., c]) / d))
    return out


def check_compact(spec, G, f_final, moments, dfdt0=None, tol_f=1e-12, tol_dfdt=1e-12,
                  tol_mom=1e-12):
    """Interior df/dt and f_final against a compact fixture: in full at the
    stored q-cells, as per-q-cell velocity sums everywhere; moments in full."""
    sel = np.array(C.COMPACT_SEL)
    for key, arr, tol in (('dfdt0', dfdt0, tol_dfdt), ('f_final', f_final, tol_f)):
        if arr is None:
            continue
        e = rel(arr[sel[:, 0], sel[:, 1]], G[key + '_sel'])
        assert e < tol, (key, 'sel', e)
        errs = _qsum_errors(spec, C.qcell_sums(spec, arr), G[key + '_qsum'])
        assert max(errs) < tol, (key, 'qsum', errs)
    errs = moment_errors(moments, {k: G['mom_' + k] for k in MOMENTS})
    assert max(errs.values()) < tol_mom, errs
