"""Eigenvalue-self-consistent GW (evGW) on the B200.

Mirrors ``src/SingleReference/GW/evGW.py:78-229`` for the space-time route,
restricted, every orbital updated, screening rebuilt from the iterate
('updated'): each cycle runs the whole device sweep (chi0, W, Sigma for all
orbitals) on the iterate's spectrum, anchors the QP equation on the mean
field eps0 (``GW/space_time.py:706-712``), and tests convergence on
HOMO/LUMO (tol 1e-5 Ha, at most 30 cycles), accelerated by Pulay's DIIS from
the second cycle (subspace 8) -- the schedule of ``evGW.py:181, 209-210``.

`warm`: 'previous' warm-starts each cycle's QP Newton solve at the previous
cycle's roots, a `QPShiftModel` at its predicted roots, None runs the plain
graphical scan; the scan stays the fallback either way.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from .grids import space_time_axes
from .gw import gw_sweep
from .space_time import _eps_host

EVGW_MAX_CYCLE, EVGW_TOL = 30, 1e-5
EVGW_DIIS_SIZE, EVGW_DIIS_START = 8, 2


class EvGWNotConverged(RuntimeWarning):
    """The evGW loop ended without a fixed point."""


class DIIS:
    """Pulay's direct inversion in the iterative subspace (Chem. Phys. Lett.
    73, 393 (1980)): the combination of the stored iterates whose combined
    residual is smallest under sum c = 1. The first `start` updates pass the
    iterate through; at most `size` pairs are kept."""

    def __init__(self, size=EVGW_DIIS_SIZE, start=EVGW_DIIS_START):
        self.size, self.start, self.seen = size, start, 0
        self.vecs, self.errs = [], []

    def update(self, vec, err):
        self.seen += 1
        if self.seen <= self.start:
            return np.asarray(vec, float)
        self.vecs.append(np.array(vec, float))
        self.errs.append(np.array(err, float))
        if len(self.vecs) > self.size:
            self.vecs.pop(0)
            self.errs.pop(0)
        n = len(self.vecs)
        B = np.zeros((n + 1, n + 1))
        for i in range(n):
            for j in range(n):
                B[i, j] = self.errs[i] @ self.errs[j]
        B[n, :n] = B[:n, n] = -1.0
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        c = np.linalg.solve(B, rhs)[:n]
        return sum(ci * v for ci, v in zip(c, self.vecs))


def evgw_eigenvalues(X, D, eps0, nocc, ntau='auto', tol=EVGW_TOL, max_cycle=EVGW_MAX_CYCLE,
                     diis_size=EVGW_DIIS_SIZE, diis_start=EVGW_DIIS_START, precision=None,
                     warm=None, eps_init=None, verbose=False, verify=False):
    """(eps, info): the evGW spectrum (Hartree, host array) of the system
    (X, D, eps0). info: cycles, converged, history (max |d eps| over HOMO and
    LUMO per cycle), sigma_evaluations per cycle, warm_accepted per cycle.

    warm: 'previous' (the last cycle's roots) or a model with predict_roots
    (the learned warm start; the states' exchange diagonal, independent of
    the orbital energies, is computed once). verify: with a warm start, also
    solve every cycle's equations plainly (the graphical scan, on the same
    Sigma) and record in info['verify_max_diff'] the largest root difference
    per cycle; those plain solves are not counted in sigma_evaluations."""
    eps0 = _eps_host(eps0)
    n = len(eps0)
    dev = torch.device('cuda', torch.cuda.current_device())
    X = X if isinstance(X, torch.Tensor) else torch.as_tensor(X, device=dev)
    D = D if isinstance(D, torch.Tensor) else torch.as_tensor(D, device=dev)
    tested = [nocc - 1, nocc]
    eps = eps0.copy() if eps_init is None else np.asarray(eps_init, float).copy()
    acc = DIIS(diis_size, diis_start) if diis_size else None
    history, evals, accepted, verified = [], [], [], []
    converged = False
    prev = None
    sx = None
    for cycle in range(int(max_cycle)):
        axes = space_time_axes(eps, nocc, ntau=ntau, anchor=eps0)
        if warm == 'previous':
            w = prev
        elif warm is not None and hasattr(warm, 'predict_roots'):
            if sx is None:
                from .qp_mlp import exchange_diagonal
                sx = exchange_diagonal(X, D, eps0, nocc, np.arange(n), axes.mu,
                                       precision=precision)

            def w(partial, model=warm, ax=axes):
                return model.predict_roots(X, D, eps0, nocc, ax, sweep=partial, sx=sx)
        else:
            w = None
        res = gw_sweep(X, D, eps, nocc, states=np.arange(n), axes=axes, precision=precision,
                       eps_anchor=eps0, warm=w)
        eps_new = res['roots'].cpu().numpy()
        flags = res['flags'].cpu().numpy()
        if verify and w is not None:
            from .gw import qp_solve
            r_plain = qp_solve(res['sigma'], axes.pade_freq, eps0, res['states'], nocc,
                               axes.mu)[0].cpu().numpy()
            ok = np.isfinite(r_plain) & np.isfinite(eps_new)
            verified.append(float(np.abs(r_plain - eps_new)[ok].max()) if ok.any() else 0.0)
        evals.append(int(res['evals'].sum().item()))
        accepted.append(int(((flags & 16) != 0).sum()))
        prev = res['roots']
        residual = eps_new - eps
        delta = float(np.abs(residual[tested]).max())
        history.append(delta)
        if verbose:
            print(f'  evGW cycle {cycle + 1:2d}  max|d eps| {delta * 27.211386:9.6f} eV')
        if delta < tol:
            eps = eps_new
            converged = True
            break
        eps = acc.update(eps_new, residual) if acc is not None else eps_new
    if not converged:
        warnings.warn(f'evGW not converged after {len(history)} cycles, max |d eps| = '
                      f'{history[-1]:.3e} Ha against tol = {tol:.3e}', EvGWNotConverged,
                      stacklevel=2)
    return eps, {'cycles': len(history), 'converged': converged, 'history': history,
                 'sigma_evaluations': evals, 'warm_accepted': accepted,
                 'verify_max_diff': verified,
                 'eps_mean_field': eps0, 'shift': eps - eps0}
