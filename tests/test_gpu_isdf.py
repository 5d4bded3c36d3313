"""The separable-RI factors' device half (mbptcode_b200.isdf) against the
reference's own fit (tests/golden/isdf.npz, made by
tests/golden/make_golden.py --only isdf): the explicit estimator, the
streaming estimator from the collocations alone, the metric root with a
dropped null direction, and the route's factors (X_mo, D). FP64; the
balanced Gram matrix is conditioned at ~1e4 here, so M is held to 1e-9
relative from explicit D (5e-9 from the collocations, whose Gram matrix
sums in another order), the root to 1e-12."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from mbptcode_b200 import isdf                                      # noqa: E402


def rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_isdf_fit_matches_reference(golden):
    g = golden('isdf')
    nk = g['ao'].shape[0]
    pairs = (g['ao'][:, :, None] * (g['ao'][:, g['second']] * g['w'][None, :])[:, None, :]
             ).reshape(nk, -1)
    D = np.hstack([pairs, g['aux']])
    F = np.hstack([g['F_pairs'], np.eye(g['aux'].shape[1])])
    M1 = isdf.fit_M_stable(D, F)
    assert isinstance(M1, np.ndarray) and rel(M1, g['M']) < 1e-9
    M2 = isdf.fit_M_products(torch.as_tensor(g['ao'], device='cuda'), g['second'], g['w'],
                             g['aux'], torch.as_tensor(g['FD'], device='cuda'))
    assert isinstance(M2, torch.Tensor) and rel(M2, g['M']) < 5e-9
    root = isdf.aux_metric_sqrt(V=g['V'])
    assert rel(root, g['root']) < 1e-12
    X_mo, Dfac, X_ao = isdf.separable_factors_from_fit(g['ao'], g['mo_coeff'], g['M'], g['V'])
    assert rel(X_mo, g['X_mo']) < 1e-13 and rel(Dfac, g['D_factor']) < 1e-11
    with pytest.raises(NotImplementedError):
        isdf.aux_metric_sqrt(V=None)
