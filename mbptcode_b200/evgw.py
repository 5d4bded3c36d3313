"""Eigenvalue-self-consistent GW (evGW) on the B200.

`evgw_eigenvalues(mf, mol=None, mode='space-time', ...)` is the drop-in for
``src/SingleReference/GW/evGW.py:78-229`` with pre-built factors: the same
arguments, numerics section, convergence test, frozen orbitals, DIIS or
damped mixing, record and warning. Each cycle runs the whole device sweep
(chi0, W, Sigma for all orbitals) on the iterate's spectrum, with the QP
equation anchored on the mean field eps0 (``GW/space_time.py:706-712``);
an unrestricted reference is driven channel by channel through the
space-time driver, one W from both spins of the iterate.

`evgw_device(X, D, eps0, nocc, ...)` is the same loop for a restricted
system given as device tensors, with the learned warm start of the QP
solve: 'previous' warm-starts each cycle's Newton solve at the last roots, a
`QPShiftModel` at its predicted roots, None runs the plain graphical scan;
the scan stays the fallback either way.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from .grids import space_time_axes
from .gw import gw_sweep
from .space_time import _eps_host

# MBPTcode src/Base/numerics/constants.py (EvGWNumerics defaults)
EVGW_MAX_CYCLE, EVGW_TOL = 30, 1e-5
EVGW_DIIS_SIZE, EVGW_DIIS_START = 8, 2
EVGW_DAMPING = 0.0
HARTREE_TO_EV = 27.211386245988
SCREENINGS = ('updated', 'fixed')


class EvGWNotConverged(RuntimeWarning):
    """The evGW loop ended without a fixed point: the last iterate comes
    back with info['converged'] False."""


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


def _settings(numerics):
    """(tol, max_cycle, diis_size, diis_start, damping) of the numerics'
    evgw section, the defaults where none is given."""
    ev = getattr(numerics, 'evgw', None)
    if ev is None:
        return EVGW_TOL, EVGW_MAX_CYCLE, EVGW_DIIS_SIZE, EVGW_DIIS_START, EVGW_DAMPING
    return (float(ev.tol), int(ev.max_cycle), int(ev.diis_size), int(ev.diis_start),
            float(getattr(ev, 'damping', EVGW_DAMPING)))


def _fixed_point(step, eps0, tested, untested, frozen, eps_init, tol, max_cycle, diis_size,
                 diis_start, damping, report=None):
    """The loop of ``evGW.py:176-212``: eps -> step(eps) until the tested
    entries move by less than tol; frozen entries are held at eps0; DIIS on
    the whole flattened spectrum against the whole residual, or damped
    mixing when diis_size is 0. Returns (eps, history, untested history,
    converged)."""
    eps = eps0.copy() if eps_init is None else np.asarray(eps_init, float).copy()
    if eps.shape != eps0.shape:
        raise ValueError(f'eps_init has shape {eps.shape}, the spectrum {eps0.shape}')
    flat0 = eps0.ravel()
    if frozen.size:
        np.put(eps, frozen, flat0[frozen])
    accel = DIIS(diis_size, diis_start) if diis_size else None
    history, rest_history = [], []
    converged = False
    for cycle in range(max_cycle):
        new = np.array(step(eps), float).reshape(eps0.shape)
        if frozen.size:
            np.put(new, frozen, flat0[frozen])
        residual = (new - eps).ravel()
        delta = float(np.abs(residual[tested]).max())
        rest = float(np.abs(residual[untested]).max()) if untested.size else 0.0
        history.append(delta)
        rest_history.append(rest)
        if report is not None:
            report(cycle, new, delta, rest)
        if delta < tol:
            eps = new
            converged = True
            break
        if accel is not None:
            eps = accel.update(new.ravel(), residual).reshape(eps0.shape)
        else:
            eps = (1.0 - damping) * new + damping * eps
    return eps, history, rest_history, converged


def evgw_eigenvalues(mf, mol=None, mode='space-time', screening='updated', converge_on=None,
                     eps_init=None, update=None, verbose=False, **route_kw):
    """(eps_qp, info): the eigenvalue-self-consistent GW spectrum in Hartree
    (``GW/evGW.py:78-229``), every orbital updated unless `update` holds
    some at the mean field, convergence on `converge_on` (flat (channel,
    orbital) indices; HOMO and LUMO of each channel by default).

    mode: 'space-time' (the device route). screening: 'updated' (evGW);
    'fixed' (evGW0) runs on the reference's Casida route and is refused.
    route_kw goes to the space-time driver (`gw.solve_qp_energy_space_time`):
    factors=(X_mo, D[, X_ao, coords]) are required (building them needs
    pyscf), numerics (its evgw section: tol, max_cycle, diis_size,
    diis_start, damping; its quadrature: ntau_st, npade, w0_gl),
    xc_diagonal, precision. mf: an object with mo_energy ((nmo,) or
    (2, nmo)), mo_occ and, for an unrestricted one, mo_coeff and nelec."""
    if mode != 'space-time':
        raise NotImplementedError(f"mode={mode!r}: the device route is mode='space-time'")
    if screening not in SCREENINGS:
        raise ValueError(f'screening={screening!r}: choose one of {SCREENINGS}')
    if screening == 'fixed':
        raise NotImplementedError(
            "screening='fixed' (evGW0) runs on the Casida route; mode='space-time' builds "
            "chi0 from the spectrum it is handed, so its W would follow the iterate")
    from .gw import solve_qp_energy_space_time
    tol, max_cycle, diis_size, diis_start, damping = _settings(route_kw.get('numerics'))
    eps0 = np.asarray(getattr(mf, 'mo_energy', mf), float)
    unrestricted = eps0.ndim == 2
    channels = ('alpha', 'beta') if unrestricted else ('alpha',)
    nmo = eps0.shape[-1]
    if unrestricted:
        noccs = tuple(int(x) for x in mf.nelec)
    else:
        mol = getattr(mf, 'mol', None) if mol is None else mol
        nel = getattr(mol, 'nelectron', None)
        noccs = ((int(nel) // 2,) if nel is not None
                 else (int((np.asarray(mf.mo_occ) > 0).sum()),))
    if converge_on is None:
        converge_on = [s * nmo + p for s, n in enumerate(noccs) for p in (n - 1, n)]
    flat = np.arange(len(channels) * nmo)
    tested = np.intersect1d(np.atleast_1d(converge_on).astype(int), flat)
    if tested.size == 0:
        raise ValueError('converge_on and states do not overlap, so nothing would decide '
                         'convergence')
    untested = np.setdiff1d(flat, tested)
    moving = flat if update is None else np.intersect1d(np.atleast_1d(update).astype(int), flat)
    if moving.size == 0:
        raise ValueError('update selects no orbital, so the spectrum could never move and the '
                         'loop would be a fixed point of nothing')
    frozen = np.setdiff1d(flat, moving)
    states = np.arange(nmo)
    kw = {k: v for k, v in route_kw.items()}

    def view(eps):
        class _View:
            pass
        v = _View()
        v.__dict__.update(getattr(mf, '__dict__', {}))
        v.mo_energy = np.asarray(eps, float)
        return v

    def step(eps):
        nocc = noccs if unrestricted else noccs[0]
        return np.array([solve_qp_energy_space_time(view(eps), mol, nocc, states,
                                                    eps_anchor=eps0, spin_channel=ch, **kw)
                         for ch in channels]).reshape(eps0.shape)

    report = None
    if verbose:
        def report(cycle, new, delta, rest):
            top = np.atleast_2d(new)[0]
            gap = (top[noccs[0]] - top[noccs[0] - 1]) * HARTREE_TO_EV
            print(f'  evGW cycle {cycle + 1:2d}  max|d eps| {delta * HARTREE_TO_EV:9.6f} eV   '
                  f'gap {gap:8.4f} eV   (untested {rest * HARTREE_TO_EV:8.5f} eV)')
    eps, history, rest, converged = _fixed_point(step, eps0, tested, untested, frozen, eps_init,
                                                 tol, max_cycle, diis_size, diis_start,
                                                 damping, report)
    info = {'cycles': len(history), 'converged': converged, 'frozen': frozen,
            'history': history, 'states': states, 'mode': mode, 'screening': screening,
            'converge_on': tested, 'residual_untested': rest[-1],
            'eps_mean_field': eps0, 'shift': eps - eps0}
    if not converged:
        warnings.warn(f'evGW not converged after {len(history)} of max_cycle = {max_cycle} '
                      f'cycles, max |delta eps| = {history[-1]:.3e} Ha against tol = '
                      f'{tol:.3e} Ha. The spectrum returned is the last iterate, not a fixed '
                      f'point; raise max_cycle or damping.', EvGWNotConverged, stacklevel=2)
    return eps, info


def evgw_device(X, D, eps0, nocc, ntau='auto', tol=EVGW_TOL, max_cycle=EVGW_MAX_CYCLE,
                diis_size=EVGW_DIIS_SIZE, diis_start=EVGW_DIIS_START, precision=None,
                warm=None, eps_init=None, verbose=False, verify=False):
    """(eps, info): the evGW spectrum (Hartree, host array) of the restricted
    system (X, D, eps0), every orbital updated, HOMO/LUMO tested. info:
    cycles, converged, history (max |d eps| over HOMO and LUMO per cycle),
    sigma_evaluations per cycle, warm_accepted per cycle.

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
    tested = np.array([nocc - 1, nocc])
    evals, accepted, verified = [], [], []
    state = {'prev': None, 'sx': None}

    def step(eps):
        axes = space_time_axes(eps, nocc, ntau=ntau, anchor=eps0)
        if warm == 'previous':
            w = state['prev']
        elif warm is not None and hasattr(warm, 'predict_roots'):
            if state['sx'] is None:
                from .qp_mlp import exchange_diagonal
                state['sx'] = exchange_diagonal(X, D, eps0, nocc, np.arange(n), axes.mu,
                                                precision=precision)

            def w(partial, model=warm, ax=axes):
                return model.predict_roots(X, D, eps0, nocc, ax, sweep=partial, sx=state['sx'])
        else:
            w = None
        res = gw_sweep(X, D, eps, nocc, states=np.arange(n), axes=axes, precision=precision,
                       eps_anchor=eps0, warm=w)
        new = res['roots'].cpu().numpy()
        flags = res['flags'].cpu().numpy()
        if verify and w is not None:
            from .gw import qp_solve
            r_plain = qp_solve(res['sigma'], axes.pade_freq, eps0, res['states'], nocc,
                               axes.mu)[0].cpu().numpy()
            ok = np.isfinite(r_plain) & np.isfinite(new)
            verified.append(float(np.abs(r_plain - new)[ok].max()) if ok.any() else 0.0)
        evals.append(int(res['evals'].sum().item()))
        accepted.append(int(((flags & 16) != 0).sum()))
        state['prev'] = res['roots']
        return new

    report = None
    if verbose:
        def report(cycle, new, delta, rest):
            print(f'  evGW cycle {cycle + 1:2d}  max|d eps| {delta * HARTREE_TO_EV:9.6f} eV')
    eps, history, _, converged = _fixed_point(
        step, eps0, tested, np.setdiff1d(np.arange(n), tested), np.array([], int), eps_init,
        tol, max_cycle, diis_size, diis_start, EVGW_DAMPING, report)
    if not converged:
        warnings.warn(f'evGW not converged after {len(history)} cycles, max |d eps| = '
                      f'{history[-1]:.3e} Ha against tol = {tol:.3e}', EvGWNotConverged,
                      stacklevel=2)
    return eps, {'cycles': len(history), 'converged': converged, 'history': history,
                 'sigma_evaluations': evals, 'warm_accepted': accepted,
                 'verify_max_diff': verified,
                 'eps_mean_field': eps0, 'shift': eps - eps0}
