"""The separable-RI (ISDF) factors on the device, from supplied inputs.

The step before the route: MBPTcode's ``Base/factorization/separable_ri.py``
fits M (naux x nk) so that the pair densities on the nk interpolation points
reproduce their Coulomb fit, then forms the route's factor D = M^T V^(1/2)
(``GW/space_time.py:82-245`` `separable_factors`). The integrals and the
mean field need pyscf and stay with the caller; what is done here is the
dense algebra that follows them:

* `fit_M_stable(D, F)`: the balanced, Tikhonov-regularised least-squares
  estimator of M from explicit pair columns D (nk x n_rho) and fitting
  coefficients F (naux x n_rho) (``separable_ri.py:1616-1653``);
* `fit_M_products(ao, second, w, aux_on_grid, FD)`: the same estimator in the
  streaming form, from the AO collocation alone (the Gram matrix of the
  product pairs is (A A^T) o (B B^T) + aux aux^T, B the second-factor columns
  scaled by their angular weights) and F D^T accumulated by the caller's
  three-centre pass (``separable_ri.py:664-900`` `fit_M_streaming`);
* `aux_metric_sqrt(V=V)`: V^(1/2) on the metric's kept spectrum
  (``separable_ri.py:1802-1929``);
* `separable_factors_from_fit(X_ao, mo_coeff, M, V)`: (X_mo, D, X_ao).

FP64 throughout (the balanced Gram matrix is conditioned at ~1e8). Arrays
come back as they were given (NumPy in, NumPy out; device tensors stay on
the device).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import require_device
from .space_time import back, to_device

# MBPTcode src/Base/numerics/constants.py
ISDF_FIT_REGULARIZATION = 4e-7      # :1755
AUX_METRIC_ROOT_FLOOR = 1e-12       # :36


def _regularization(numerics):
    isdf = getattr(numerics, 'isdf', None)
    reg = getattr(isdf, 'regularization', None)
    return ISDF_FIT_REGULARIZATION if reg is None else float(reg)


def _balanced_solve(S, FD, regularization):
    """M = [FD (d S d + reg I)^-1] o d with d the inverse square roots of
    diag S (1 where it is zero): the estimator's solve, by a Cholesky
    factorisation of the balanced Gram matrix."""
    scale = torch.sqrt(torch.clamp(torch.diagonal(S), min=0.0))
    scale = torch.where(scale > 0, scale, torch.ones_like(scale))
    d = 1.0 / scale
    G = S * d[:, None] * d[None, :]
    G.diagonal().add_(regularization)
    L = torch.linalg.cholesky(G)
    rhs = (FD * d[None, :]).T.contiguous()
    return torch.cholesky_solve(rhs, L).T * d[None, :]


def fit_M_stable(D, F, numerics=None):
    """M (naux, nk) of the balanced, regularised estimator from explicit D
    (nk, n_rho) and F (naux, n_rho) (``separable_ri.py:1640-1653``)."""
    dev = require_device()
    Dd, Fd = to_device(D, dev), to_device(F, dev)
    return back(_balanced_solve(Dd @ Dd.T, Fd @ Dd.T, _regularization(numerics)), D)


def fit_M_products(ao, second, w, aux_on_grid, FD, numerics=None):
    """M (naux, nk) of the same estimator from the collocations alone: the
    Gram matrix of the product pairs (mu, j) -> ao[:, mu] ao[:, second[j]] w[j]
    and of the auxiliary functions, (A A^T) o (B B^T) + aux aux^T, and F D^T
    as accumulated by the three-centre pass (naux, nk), the auxiliary block's
    identity included (``separable_ri.py:664-900``)."""
    dev = require_device()
    A = to_device(ao, dev)
    sec = torch.as_tensor(np.asarray(second, dtype=np.int64), device=dev)
    B = A[:, sec] * to_device(np.asarray(w, float), dev)[None, :]
    X = to_device(aux_on_grid, dev)
    S = (A @ A.T) * (B @ B.T) + X @ X.T
    return back(_balanced_solve(S, to_device(FD, dev), _regularization(numerics)), FD)


def aux_metric_sqrt(auxmol=None, environment=None, V=None):
    """V^(1/2) of a symmetric auxiliary metric on its kept spectrum: the
    eigen-directions below AUX_METRIC_ROOT_FLOOR of the largest eigenvalue
    are its numerical null space and are dropped (``separable_ri.py:1802-1929``).
    A dressed metric (an environment's kernel) needs pyscf's integrals and is
    refused; V must be given."""
    if environment is not None:
        raise NotImplementedError('a dressed metric needs the environment kernel\'s '
                                  'integrals (pyscf); pass the bare V')
    if V is None:
        raise NotImplementedError('building V needs pyscf\'s two-centre integrals; pass V')
    dev = require_device()
    Vd = to_device(V, dev)
    w, v = torch.linalg.eigh(0.5 * (Vd + Vd.T))
    keep = w > AUX_METRIC_ROOT_FLOOR * w.max()
    vk = v[:, keep]
    return back((vk * torch.sqrt(w[keep])[None, :]) @ vk.T, V)


def separable_factors_from_fit(X_ao, mo_coeff, M, V):
    """(X_mo, D, X_ao): the route's factors from the fit, X_mo = X_ao C and
    D = M^T V^(1/2) (``GW/space_time.py:82-245``, with the collocation and the
    fit supplied)."""
    dev = require_device()
    Xa = to_device(X_ao, dev)
    root = to_device(aux_metric_sqrt(V=to_device(V, dev)), dev)
    Xm = Xa @ to_device(mo_coeff, dev)
    Dd = to_device(M, dev).T @ root
    return back(Xm, X_ao), back(Dd, X_ao), X_ao
