"""Seeded synthetic ISDF systems of the benchmark configurations.

Phi (M x n) has QR-orthonormalised Gaussian columns, scaled by 1/sqrt(M)
('literal') or left unit-norm ('calibrated', a strongly coupled variant:
the literal scaling makes chi0 ~ 1/M^2 and the system nearly non-interacting).
Occupied energies are uniform in [-1.5, -0.3] Ha, virtual ones log-uniform in
[0.05, 5] Ha, both sorted. V = L L^T + 1e-3 I with Gaussian L whose column k
is scaled by k^-1.2 (a decaying spectrum), and D = chol(V), so that the
Coulomb factor Z = D D^T of the ISDF route is V itself.
"""
from __future__ import annotations

import numpy as np

EPS_OCC = (-1.5, -0.3)
EPS_VIRT = (0.05, 5.0)
V_SHIFT = 1e-3
V_DECAY = -1.2


def synthetic_system(n_orb, nocc, M, seed=0, variant='literal'):
    """(X, D, eps) as FP64 numpy arrays."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((M, n_orb)))
    X = Q / np.sqrt(M) if variant == 'literal' else Q.copy()
    eps = np.concatenate([
        np.sort(rng.uniform(*EPS_OCC, nocc)),
        np.sort(np.exp(rng.uniform(np.log(EPS_VIRT[0]), np.log(EPS_VIRT[1]),
                                   n_orb - nocc)))])
    L = rng.standard_normal((M, M)) * np.arange(1, M + 1, dtype=float) ** V_DECAY
    V = L @ L.T + V_SHIFT * np.eye(M)
    D = np.linalg.cholesky(V)
    return np.ascontiguousarray(X), np.ascontiguousarray(D), eps


def synthetic_system_torch(n_orb, nocc, M, seed=0, variant='literal',
                           device='cuda'):
    """The same generator on the device (torch's RNG, so other numbers than
    the numpy one for the same seed): used where M is large."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    f64 = torch.float64
    Q, _ = torch.linalg.qr(torch.randn(M, n_orb, generator=g, device=device,
                                       dtype=f64))
    X = Q / np.sqrt(M) if variant == 'literal' else Q
    eo = torch.rand(nocc, generator=g, device=device, dtype=f64)
    eo = torch.sort(EPS_OCC[0] + (EPS_OCC[1] - EPS_OCC[0]) * eo).values
    lv = torch.rand(n_orb - nocc, generator=g, device=device, dtype=f64)
    ev = torch.sort(torch.exp(np.log(EPS_VIRT[0])
                              + (np.log(EPS_VIRT[1]) - np.log(EPS_VIRT[0])) * lv)).values
    eps = torch.cat([eo, ev])
    k = torch.arange(1, M + 1, device=device, dtype=f64) ** V_DECAY
    L = torch.randn(M, M, generator=g, device=device, dtype=f64) * k
    V = L @ L.T
    V.diagonal().add_(V_SHIFT)
    del L
    D = torch.linalg.cholesky(V)
    del V
    return X.contiguous(), D.contiguous(), eps
