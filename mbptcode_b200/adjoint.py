"""dRPA correlation energy and its adjoint on the B200.

Mirrors ``src/gradients/rpa/space_time_adjoint.py:473-563``
(`rpa_energy_and_adjoint`, gas phase, one GPU): one forward sweep keeps
proj(tau); per frequency chi0_bar = (w/2pi) [I - (1 - chi0)^-T] from the
Dyson inverse (:528-539); proj_bar = cosft_wt^T chi0_bar (:440-454); and the
reverse sweep (:136-218) recomputes G_occ(tau), G_virt(tau) per tau point --
nothing of G is stored across tau -- to accumulate eps_bar, X_bar, D_bar.

`RPAEnergy` wraps it as a torch.autograd.Function of (eps, X, D); the
Coulomb factor's own dependence on V (D = chol(V)) is left to torch's
Cholesky backward, so `rpa_energy(eps, X, V=V)` differentiates in V too.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import WORKSPACE, check, host_array, lib, ptr, require_device, stream_ptr
from .space_time import (_Err, _eps_host, _mode, chi0_sweep, dyson_batch,
                         particle_hole_window, to_device, transform)


def chi0_backward(proj_bar, X, D, eps, nocc, tau_points, mu, precision='fp64', stream=None):
    """(eps_bar, X_bar, D_bar) device tensors for an adjoint proj_bar
    (ntau, naux, naux): ``space_time_adjoint.py:136-218``."""
    dev = proj_bar.device
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    ed = to_device(eps_h, dev)
    M, norb = Xd.shape
    naux = Dd.shape[1]
    tau_h, tp = host_array(tau_points)
    mode = _mode(precision)
    eps_bar = torch.empty(norb, dtype=torch.float64, device=dev)
    X_bar = torch.empty((M, norb), dtype=torch.float64, device=dev)
    D_bar = torch.empty((M, naux), dtype=torch.float64, device=dev)
    ws = WORKSPACE.get(lib().mbpt_chi0_backward_workspace_bytes(M, norb, nocc, naux, mode), dev)
    err = _Err(dev)
    pb = proj_bar.contiguous()  # held until the call has launched its kernels
    check(lib().mbpt_chi0_backward(ptr(pb), ptr(Xd), M, norb, nocc, ptr(ed),
                                   float(mu), ptr(Dd), naux, tp, len(tau_h), mode,
                                   ptr(eps_bar), ptr(X_bar), ptr(D_bar), ptr(ws), ws.numel(),
                                   ptr(err.t), stream_ptr(stream)), 'mbpt_chi0_backward')
    err.check('mbpt_chi0_backward')
    return eps_bar, X_bar, D_bar


def energy_and_adjoint_device(X, D, eps, nocc, grid, mu=None, want_grad=True,
                              precision='fp64', stream=None):
    """(E_c 0-d tensor, eps_bar, X_bar, D_bar) on the device."""
    dev = require_device()
    eps_h = _eps_host(eps)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    chi0, proj = chi0_sweep(X, D, eps_h, nocc, grid.tau_points, grid.cosft_wt, mu=mu,
                            precision=precision, want_proj=want_grad, stream=stream)
    logdet, trace, info, _ = dyson_batch(chi0, want_w=want_grad, stream=stream)
    ow = torch.as_tensor(np.asarray(grid.omega_weights, float), device=dev)
    e_c = torch.empty((), dtype=torch.float64, device=dev)
    check(lib().mbpt_energy_sum(ptr(logdet), ptr(trace), ptr(ow), len(ow), ptr(e_c),
                                stream_ptr(stream)), 'mbpt_energy_sum')
    if not want_grad:
        return e_c, None, None, None
    if np.any(info):
        raise FloatingPointError('1 - chi0 is not positive definite at frequencies '
                                 f'{np.nonzero(info)[0].tolist()}: no dRPA gradient')
    # chi0 now holds W - I; chi0_bar = -(w/2pi) (W - I)^T in place
    check(lib().mbpt_energy_adjoint_seed(ptr(chi0), chi0.shape[-1], chi0.shape[0], ptr(ow),
                                         stream_ptr(stream)), 'mbpt_energy_adjoint_seed')
    proj_bar = transform(chi0, np.ascontiguousarray(np.asarray(grid.cosft_wt).T), stream)
    del chi0, proj
    eps_bar, X_bar, D_bar = chi0_backward(proj_bar, X, D, eps_h, nocc, grid.tau_points, mu,
                                          precision='fp64', stream=stream)
    return e_c, eps_bar, X_bar, D_bar


def rpa_energy_and_adjoint(X, D, eps, nocc, grid, mu=None, want_grad=True, tile_gb=None,
                           screening=None, counter_term=None, comm=None, precision='fp64'):
    """``space_time_adjoint.py:473-563``: (e_c, eps_bar, X_bar, D_bar,
    fold_bar) with fold_bar None (no solvent fold on the device route);
    want_grad=False returns E_c alone. Arrays come back as the inputs are
    held (NumPy or device tensors)."""
    if screening is not None or counter_term is not None:
        raise NotImplementedError('the solvent-folded energy is not on the device route')
    e_c, eb, xb, db = energy_and_adjoint_device(X, D, eps, nocc, grid, mu, want_grad,
                                                precision)
    if not want_grad:
        return float(e_c.item())
    if isinstance(X, torch.Tensor):
        return e_c, eb, xb, db, None
    return float(e_c.item()), eb.cpu().numpy(), xb.cpu().numpy(), db.cpu().numpy(), None


class RPAEnergy(torch.autograd.Function):
    """E_c^dRPA(eps, X, D) with the hand-written reverse sweep as backward.
    The grid is frozen (a discrete choice, as in the reference's chain)."""

    @staticmethod
    def forward(ctx, eps, X, D, nocc, grid, mu, precision):
        e_c, eb, xb, db = energy_and_adjoint_device(X.detach(), D.detach(), eps.detach(),
                                                    nocc, grid, mu, True, precision)
        ctx.save_for_backward(eb, xb, db)
        return e_c

    @staticmethod
    def backward(ctx, g):
        eb, xb, db = ctx.saved_tensors
        return g * eb, g * xb, g * db, None, None, None, None


def rpa_energy(eps, X, D=None, nocc=None, grid=None, V=None, mu=None, precision='fp64'):
    """Differentiable E_c of device tensors: give D (M x naux), or V (M x M,
    SPD) with D = chol(V) taken by torch so that V gets a gradient too."""
    if D is None:
        if V is None:
            raise ValueError('give D or V')
        D = torch.linalg.cholesky(V)
    if mu is None:
        mu = particle_hole_window(eps.detach().cpu().numpy(), nocc)[2]
    return RPAEnergy.apply(eps, X, D, nocc, grid, mu, precision)
