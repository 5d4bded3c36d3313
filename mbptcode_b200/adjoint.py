"""dRPA correlation energy, the self-energy diagonal, and their adjoints on
the B200.

Mirrors ``src/gradients/rpa/space_time_adjoint.py:473-563``
(`rpa_energy_and_adjoint`, gas phase, one GPU): one forward sweep keeps
proj(tau); per frequency chi0_bar = (w/2pi) [I - (1 - chi0)^-T] from the
Dyson inverse (:528-539); proj_bar = cosft_wt^T chi0_bar (:440-454); and the
reverse sweep (:136-218) recomputes G_occ(tau), G_virt(tau) per tau point --
nothing of G is stored across tau -- to accumulate eps_bar, X_bar, D_bar.

`RPAEnergy` wraps it as a torch.autograd.Function of (eps, X, D); the
Coulomb factor's own dependence on V (D = chol(V)) is left to torch's
Cholesky backward, so `rpa_energy(eps, X, V=V)` differentiates in V too.

The self-energy diagonal Sigma^c_pp(i omega) and its reverse
(``space_time_adjoint.py:652-691, 795-875``, the QP-gradient building
blocks): `selfenergy_diag` keeps proj(tau) and W(tau) as its cache;
`selfenergy_diag_backward` runs the self-energy sweep backwards
(mbpt_sigma_backward), then the Dyson step (mbpt_dyson_backward, W rebuilt
from proj(tau)) and the chi0 sweep (mbpt_chi0_backward). `SelfEnergyDiag`
wraps them as a torch.autograd.Function of (eps, X, D).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import WORKSPACE, check, host_array, lib, ptr, require_device, stream_ptr
from .space_time import (_Err, _eps_host, _mode, chi0_sweep, dyson_batch,
                         particle_hole_window, to_device, transform)

#: precision of the adjoints' sweeps (forward and reverse) where the call
#: names none: FP64-accurate, with the products and the Cholesky updates
#: emulated on the int8 tensor cores (8 seven-bit digits per operand), on
#: grids whose tau <-> omega weights stay below INT8_WEIGHT_LIMIT; native FP64
#: ('fp64') on the others. The emulation's error, ~5e-15 of the operands'
#: scale per product, changes erratically from one tau point to the next, so
#: weights that cancel at 1e8 (the 16-point grids of small gaps) lift it
#: past FP64 rounding (E_c 8e-10 relative at 2.4e8, against 1e-11).
ADJOINT_PRECISION = 'fp64_int8'
INT8_WEIGHT_LIMIT = 1e6


def _adjoint_precision(precision, *weights):
    if precision is not None:
        return precision
    w = max((float(np.abs(np.asarray(x, float)).max()) for x in weights), default=0.0)
    return ADJOINT_PRECISION if w <= INT8_WEIGHT_LIMIT else 'fp64'


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


def polarizability_backward(proj_bar, X, D, eps, nocc, grid, mu=None, tile_gb=None,
                            tau_indices=None):
    """(eps_bar, X_bar, D_bar) for an adjoint proj_bar (ntau, naux, naux) on
    proj(tau) (``space_time_adjoint.py:136-164``), the reverse chi0 sweep on
    the device; arrays come back as proj_bar is held."""
    if tau_indices is not None:
        raise NotImplementedError('tau splits over ranks are outside the one-GPU route')
    dev = require_device()
    eps_h = _eps_host(eps)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    out = chi0_backward(to_device(proj_bar, dev), X, D, eps_h, nocc, grid.tau_points, mu,
                        precision=_adjoint_precision(None, grid.cosft_wt))
    return tuple(t if isinstance(proj_bar, torch.Tensor) else t.cpu().numpy() for t in out)


def energy_and_adjoint_device(X, D, eps, nocc, grid, mu=None, want_grad=True,
                              precision=None, stream=None):
    """(E_c 0-d tensor, eps_bar, X_bar, D_bar) on the device."""
    precision = _adjoint_precision(precision, grid.cosft_wt)
    dev = require_device()
    eps_h = _eps_host(eps)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    chi0, proj = chi0_sweep(X, D, eps_h, nocc, grid.tau_points, grid.cosft_wt, mu=mu,
                            precision=precision, want_proj=want_grad, stream=stream)
    logdet, trace, info, _ = dyson_batch(chi0, want_w=want_grad, stream=stream,
                                         precision=precision)
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
                                          precision=precision, stream=stream)
    return e_c, eps_bar, X_bar, D_bar


def rpa_energy_and_adjoint(X, D, eps, nocc, grid, mu=None, want_grad=True, tile_gb=None,
                           screening=None, counter_term=None, comm=None, precision=None):
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


def rpa_energy(eps, X, D=None, nocc=None, grid=None, V=None, mu=None, precision=None):
    """Differentiable E_c of device tensors: give D (M x naux), or V (M x M,
    SPD) with D = chol(V) taken by torch so that V gets a gradient too."""
    if D is None:
        if V is None:
            raise ValueError('give D or V')
        D = torch.linalg.cholesky(V)
    if mu is None:
        mu = particle_hole_window(eps.detach().cpu().numpy(), nocc)[2]
    return RPAEnergy.apply(eps, X, D, nocc, grid, mu, precision)


# ---------------------------------------------------------------- self-energy

def _one_rank(comm, who):
    if comm is not None and comm.Get_size() > 1:
        raise NotImplementedError(f'{who}: rank splits are outside the one-GPU route')


def _back(t, like):
    return t if isinstance(like, torch.Tensor) else t.cpu().numpy()


def selfenergy_diag(X, D, eps, nocc, grid, states, transforms, mu, tile_gb=None, comm=None,
                    precision=None):
    """Sigma^c_pp(i omega_out) of `states` on the grid's own tau points, and
    the cache its reverse needs (``GW/imaginary_time.py:731-768``): chi0 and
    proj(tau) in one sweep, W - I by the Dyson step, Wt(tau) = Ctw (W - I),
    the branch sums and the tau -> omega transform with (C, S). Returns
    (sigma (nstates, nfreq_out) complex, (proj_tau, Wt_tau, None)); the
    cache's tensors stay on the device."""
    from .gw import sigma_branch_sums, sigma_frequency, w_tau_from_frequencies
    _one_rank(comm, 'selfenergy_diag')
    precision = _adjoint_precision(precision, grid.cosft_wt, *transforms)
    dev = require_device()
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    Ctw, C, S = transforms
    chi0, proj = chi0_sweep(Xd, Dd, eps_h, nocc, grid.tau_points, grid.cosft_wt, mu=mu,
                            precision=precision, want_proj=True)
    dyson_batch(chi0, want_w=True, precision=precision)
    Wt = w_tau_from_frequencies(chi0, Ctw)
    del chi0
    branch = sigma_branch_sums(Xd, Dd, Wt, eps_h, nocc, grid.tau_points,
                               np.atleast_1d(states), mu, precision)
    sigma = sigma_frequency(branch, C, S)
    return _back(sigma, X), (proj, Wt, None)


def screened_interaction_tau_backward(Wt_bar, proj_tau, grid, Ctw, tile_gb=None, comm=None,
                                      precision=None):
    """proj_bar (ntau, naux, naux) for an adjoint Wt_bar on
    Wt(tau) = sum_w Ctw[tau, w] (W_w - I) (``space_time_adjoint.py:652-691``):
    chi0 rebuilt from proj(tau), W by the Dyson step, chi0_bar = W W_bar W per
    frequency, and the two transforms turned round. FP64-accurate."""
    _one_rank(comm, 'screened_interaction_tau_backward')
    precision = _adjoint_precision(precision, grid.cosft_wt, Ctw)
    dev = require_device()
    Wb, P = to_device(Wt_bar, dev), to_device(proj_tau, dev)
    cw = np.asarray(grid.cosft_wt, float)
    chi0 = transform(P, cw)
    dyson_batch(chi0, want_w=True, precision=precision)
    wbar = transform(Wb, np.ascontiguousarray(np.asarray(Ctw, float).T))
    naux, nfreq = chi0.shape[-1], chi0.shape[0]
    ws = WORKSPACE.get(lib().mbpt_dyson_backward_workspace_bytes(naux), dev)
    check(lib().mbpt_dyson_backward(ptr(chi0), ptr(wbar), naux, nfreq, _mode(precision),
                                    ptr(ws), ws.numel(), stream_ptr()), 'mbpt_dyson_backward')
    proj_bar = transform(wbar, np.ascontiguousarray(cw.T))
    return _back(proj_bar, Wt_bar)


def sigma_backward(branch_bar, X, D, eps, nocc, tau_points, states, mu, Wt,
                   precision=ADJOINT_PRECISION):
    """(eps_bar, X_bar, D_bar, Wt_bar) device tensors of the self-energy sweep
    alone for branch adjoints (2, ntau, nstates) on (Sigma^<, Sigma^>);
    precision 'fp64' or 'fp64_int8'."""
    dev = require_device()
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    ed = to_device(eps_h, dev)
    M, norb = Xd.shape
    naux = Dd.shape[1]
    tau_h, tp = host_array(tau_points)
    st_h = np.asarray(states, dtype=np.int64)
    if st_h.size == 0 or st_h.min() < 0 or st_h.max() >= norb:
        raise ValueError(f'states must be orbital indices in [0, {norb}), got {st_h}')
    st = torch.as_tensor(st_h, device=dev)
    S = st.numel()
    bb = to_device(branch_bar, dev)
    sl, sg = bb[0].contiguous(), bb[1].contiguous()
    Wc = to_device(Wt, dev)
    if Wc.shape != (len(tau_h), naux, naux) or sl.shape != (len(tau_h), S):
        raise ValueError(f'Wt {tuple(Wc.shape)} and branch adjoints {tuple(bb.shape)} do not '
                         f'match {len(tau_h)} tau points, {S} states, naux {naux}')
    eps_bar = torch.empty(norb, dtype=torch.float64, device=dev)
    X_bar = torch.empty((M, norb), dtype=torch.float64, device=dev)
    D_bar = torch.empty((M, naux), dtype=torch.float64, device=dev)
    Wt_bar = torch.empty_like(Wc)
    ws = WORKSPACE.get(lib().mbpt_sigma_backward_workspace_bytes(M, norb, nocc, naux, S), dev)
    err = _Err(dev)
    check(lib().mbpt_sigma_backward(ptr(Xd), M, norb, nocc, ptr(ed), float(mu), ptr(Dd), naux,
                                    tp, len(tau_h), ptr(Wc), ptr(st), S, ptr(sl), ptr(sg),
                                    _mode(precision), ptr(eps_bar), ptr(X_bar), ptr(D_bar),
                                    ptr(Wt_bar),
                                    ptr(ws), ws.numel(), ptr(err.t), stream_ptr()),
          'mbpt_sigma_backward')
    err.check('mbpt_sigma_backward')
    return eps_bar, X_bar, D_bar, Wt_bar


def _branch_bar(a_re, a_im, C, S):
    """Adjoints on (Sigma^<, Sigma^>)(tau) of Sigma = -1/2 [(S> + S<)^T C^T
    + i (S> - S<)^T S^T] (``space_time_adjoint.py:830-833``)."""
    a_re = a_re.detach().cpu().numpy() if isinstance(a_re, torch.Tensor) else np.asarray(a_re)
    a_im = a_im.detach().cpu().numpy() if isinstance(a_im, torch.Tensor) else np.asarray(a_im)
    ac = np.atleast_2d(a_re) @ np.asarray(C, float)
    bs = np.atleast_2d(a_im) @ np.asarray(S, float)
    return np.stack([-0.5 * (ac - bs).T, -0.5 * (ac + bs).T])


def selfenergy_diag_backward(a_re, a_im, X, D, eps, nocc, grid, states, transforms, mu,
                             cache, tile_gb=None, comm=None):
    """(eps_bar, X_bar, D_bar) for the real functional
    sum a_re Re Sigma + a_im Im Sigma of `selfenergy_diag`'s output
    (``space_time_adjoint.py:795-875``): the self-energy sweep backwards, then
    W_bar through the Dyson step and the chi0 sweep backwards. `cache` is
    `selfenergy_diag`'s (proj_tau, Wt_tau, ...). FP64; arrays come back as X
    is held."""
    _one_rank(comm, 'selfenergy_diag_backward')
    Ctw, C, S = transforms
    proj, Wt = cache[0], cache[1]
    precision = _adjoint_precision(None, grid.cosft_wt, *transforms)
    eps_h = _eps_host(eps)
    bb = _branch_bar(a_re, a_im, C, S)
    e1, x1, d1, Wt_bar = sigma_backward(bb, X, D, eps_h, nocc, grid.tau_points,
                                        np.atleast_1d(states), mu, Wt, precision)
    proj_bar = screened_interaction_tau_backward(Wt_bar, to_device(proj, Wt_bar.device), grid,
                                                 Ctw, precision=precision)
    e2, x2, d2 = chi0_backward(proj_bar, X, D, eps_h, nocc, grid.tau_points, mu,
                               precision=precision)
    out = (e1 + e2, x1 + x2, d1 + d2)
    return tuple(_back(t, X) for t in out)


class SelfEnergyDiag(torch.autograd.Function):
    """Sigma^c_pp(i omega_out) (complex, nstates x nfreq_out) of (eps, X, D)
    with `selfenergy_diag_backward` as backward; the grid, transforms and mu
    are frozen. torch hands a real loss's gradient on a complex output as
    dL/dRe + i dL/dIm, which are the adjoints a_re, a_im."""

    @staticmethod
    def forward(ctx, eps, X, D, nocc, grid, states, transforms, mu):
        sigma, cache = selfenergy_diag(X.detach(), D.detach(), eps.detach(), nocc, grid,
                                       states, transforms, mu)
        ctx.args = (nocc, grid, states, transforms, mu, cache)
        ctx.save_for_backward(eps, X, D)
        return sigma

    @staticmethod
    def backward(ctx, g):
        eps, X, D = ctx.saved_tensors
        nocc, grid, states, transforms, mu, cache = ctx.args
        eb, xb, db = selfenergy_diag_backward(g.real, g.imag, X.detach(), D.detach(),
                                              eps.detach(), nocc, grid, states, transforms,
                                              mu, cache)
        return eb, xb, db, None, None, None, None, None


def selfenergy_diag_t(eps, X, D, nocc, grid, states, transforms=None, mu=None, omega_out=None):
    """Differentiable Sigma^c_pp(i omega_out) of device tensors (eps, X, D).
    transforms default to `grids.sigma_transforms` on the grid's own axes
    (omega_out: the grid's frequencies unless given)."""
    eps_h = eps.detach().cpu().numpy()
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    if transforms is None:
        from .grids import sigma_transforms
        out = grid.omega_points if omega_out is None else omega_out
        transforms = sigma_transforms(eps_h, nocc, grid.tau_points, grid.omega_points, out,
                                      mu=mu)
    return SelfEnergyDiag.apply(eps, X, D, nocc, grid, np.atleast_1d(states), transforms, mu)
