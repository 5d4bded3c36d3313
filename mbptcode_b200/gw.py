"""Space-time G0W0 on the B200: W(tau), the correlation self-energy diagonal,
the Pade continuation and the quasiparticle roots.

Mirrors MBPTcode's route (``src/SingleReference/GW/space_time.py:631-863``,
restricted, serial, in core) and its helpers
``GW/imaginary_time.py:181-195, 403-587`` and ``GW/qp_solve.py:529-703``;
all arithmetic runs in libmbpt_b200.
"""
from __future__ import annotations

import contextlib
import time
import warnings

import numpy as np
import torch

from ._lib import BUFFERS, WORKSPACE, check, host_array, lib, ptr, require_device, stream_ptr
from .grids import space_time_axes, space_time_axes_unrestricted
from .space_time import (_Err, _eps_host, _mode, check_mixed_weights, chi0_sweep,
                         dyson_batch, to_device, transform)

QP_FLAG_QUASIPARTICLE, QP_FLAG_NO_ROOT, QP_FLAG_Z_OUTSIDE, QP_FLAG_PADE_FAILED, \
    QP_FLAG_WARM, QP_FLAG_OVERFLOW = 1, 2, 4, 8, 16, 32


class QPNoRoot(RuntimeWarning):
    """A quasiparticle equation without a root in its widest scan window."""


class QPWeightOutside(RuntimeWarning):
    """A quasiparticle root kept with Z outside (0, 1]."""


def w_tau_from_frequencies(W_minus_I, Ctw, stream=None, out=None):
    """Wt(tau) = sum_w Ctw[tau, w] (W(i w) - I): ``imaginary_time.py:181-195``
    (here from W - I as the Dyson step leaves it), FP64 on the device."""
    return transform(W_minus_I, Ctw, stream, out=out)


def _transform_screened(Ctw, W_omega):
    """sum_w Ctw[., w] (W(i w) - I) from W itself (``imaginary_time.py:181-195``):
    NumPy in, NumPy out, as the reference."""
    from .space_time import back
    dev = require_device()
    Wm = to_device(W_omega, dev).clone()
    Wm.diagonal(dim1=-2, dim2=-1).sub_(1.0)
    return back(transform(Wm, np.asarray(Ctw, float)), W_omega)


def self_energy_matrix_imaginary_time(X_ao, D, W_omega, mo_coeff, eps, nocc, tau_points,
                                      omega_in, omega_out, mu=None, ranges=None,
                                      tau_indices=None, Wt_tau=None, block_memory_gb=None,
                                      coords=None, screen_r_cut=None, precision='fp64'):
    """Full Sigma^c_{mu nu}(i omega_out) in the AO basis, (nfreq_out, nao, nao)
    complex (``imaginary_time.py:403-533``): W(tau) from W(i omega_in) (or
    Wt_tau as given), per time point the two branches X_ao^T (G o Zt) X_ao
    with G from the MO collocation X_ao mo_coeff (mbpt_sigma_ao), then
    Sigma = -1/2 [C (S^> + S^<) + i S (S^> - S^<)]. precision: 'fp64' (the
    reference's arithmetic), 'fp64_int8' or 'mixed' (the self-energy sweep's
    split BF16 products, ~1e-5 relative). tau_indices: that subset's
    contribution. block_memory_gb and coords are accepted for signature
    compatibility; distance screening (screen_r_cut) is refused. NumPy in,
    NumPy out."""
    from .grids import COSINE_TW, COSINE_WT, SINE_TW, sigma_fit_ranges, transform_weights
    from .space_time import back
    if screen_r_cut:
        raise NotImplementedError('distance screening is outside the device route')
    dev = require_device()
    eps_h = _eps_host(eps)
    if mu is None:
        mu = float(0.5 * (eps_h[:nocc].max() + eps_h[nocc:].min()))
    rW, rS = ranges or sigma_fit_ranges(eps_h, nocc, mu=mu)
    tau = np.asarray(tau_points, float)
    which = np.arange(len(tau)) if tau_indices is None else np.atleast_1d(tau_indices)
    if Wt_tau is None:
        Ctw, _ = transform_weights(COSINE_WT, tau, omega_in, *rW, warn=False)
        Wm = to_device(W_omega, dev).clone()
        Wm.diagonal(dim1=-2, dim2=-1).sub_(1.0)
        Wt = transform(Wm, Ctw[which])
        del Wm
    else:
        Wt = to_device(Wt_tau, dev)[torch.as_tensor(which, device=dev)].contiguous()
    C, _ = transform_weights(COSINE_TW, tau, omega_out, *rS, warn=False)
    S, _ = transform_weights(SINE_TW, tau, omega_out, *rS, warn=False)
    Xa, Dd, Cm = to_device(X_ao, dev), to_device(D, dev), to_device(mo_coeff, dev)
    ed = to_device(eps_h, dev)
    M, nao = Xa.shape
    norb, naux, nt = Cm.shape[1], Dd.shape[1], len(which)
    tau_h, tp = host_array(tau[which])
    br = torch.empty((2, nt, nao, nao), dtype=torch.float64, device=dev)
    mode = _mode(precision)
    ws = WORKSPACE.get(lib().mbpt_sigma_ao_workspace_bytes(M, nao, norb, nocc, naux, mode), dev)
    err = _Err(dev)
    check(lib().mbpt_sigma_ao(ptr(Xa), M, nao, ptr(Cm), norb, nocc, ptr(ed), float(mu),
                              ptr(Dd), naux, ptr(Wt), tp, nt, mode, ptr(br), ptr(ws),
                              ws.numel(), ptr(err.t), stream_ptr()), 'mbpt_sigma_ao')
    err.check('mbpt_sigma_ao')
    re = transform((br[1] + br[0]).contiguous(), np.ascontiguousarray(C[:, which]))
    im = transform((br[1] - br[0]).contiguous(), np.ascontiguousarray(S[:, which]))
    return back(torch.complex(-0.5 * re, -0.5 * im), X_ao)


def sigma_ao_to_mo_diagonal(sigma_ao, mo_coeff, states=None):
    """MO-diagonal Sigma_pp, (nfreq, nstates), without the full MO matrix
    (``imaginary_time.py:581-587``)."""
    if isinstance(sigma_ao, torch.Tensor):
        Cm = to_device(mo_coeff, sigma_ao.device).to(sigma_ao.dtype)
        Cm = Cm if states is None else Cm[:, torch.as_tensor(np.atleast_1d(states),
                                                            device=sigma_ao.device)]
        return torch.einsum('mp,wmn,np->wp', Cm, sigma_ao, Cm)
    Cm = np.asarray(mo_coeff) if states is None else np.asarray(mo_coeff)[:, states]
    return np.einsum('mp,wmn,np->wp', Cm, sigma_ao, Cm, optimize=True)


def screened_interaction_tau(proj_tau, grid, Ctw, tile_gb=None, comm=None):
    """Wt(tau) = sum_w Ctw[t, w] ([I - chi0_w]^-1 - I) from proj(tau)
    (``imaginary_time.py:590-629``): chi0 on the grid's frequencies by the
    tau -> omega transform, the Dyson step, the omega -> tau transform; FP64
    on the device, arrays back as proj_tau is held."""
    from .space_time import back
    if comm is not None and comm.Get_size() > 1:
        raise NotImplementedError('rank splits are outside the one-GPU route')
    dev = require_device()
    chi0 = transform(to_device(proj_tau, dev), np.asarray(grid.cosft_wt, float))
    dyson_batch(chi0, want_w=True, precision='fp64')
    return back(transform(chi0, np.asarray(Ctw, float)), proj_tau)


def sigma_branch_sums(X, D, Wt, eps, nocc, tau_points, states, mu, precision=None,
                      stream=None, err=None):
    """(2, ntau, nstates) device tensor: Sigma^<_pp(tau) and Sigma^>_pp(tau) of
    the states, the diagonal form of ``imaginary_time.py:39-92``. Wt None
    stands for W = I at every tau (the bare Coulomb factor)."""
    dev = require_device()
    Wt = None if Wt is None else to_device(Wt, dev)
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    ed = to_device(eps_h, dev)
    M, norb = Xd.shape
    naux = Dd.shape[1]
    st = torch.as_tensor(np.asarray(states, dtype=np.int64), device=dev)
    S = st.numel()
    tau_h, tp = host_array(tau_points)
    ntau = len(tau_h)
    if Wt is not None and Wt.shape != (ntau, naux, naux):
        raise ValueError(f'Wt is {tuple(Wt.shape)}, need ({ntau}, {naux}, {naux})')
    mode = _mode(precision)
    branch = torch.empty((2, ntau, S), dtype=torch.float64, device=dev)
    ws = WORKSPACE.get(lib().mbpt_sigma_workspace_bytes(M, norb, nocc, naux, ntau, S, mode), dev)
    own = err is None
    err = _Err(dev) if own else err
    Wc = None if Wt is None else Wt.contiguous()  # held until the kernels are launched
    check(lib().mbpt_sigma_branch_sums(ptr(Xd), M, norb, nocc, ptr(ed), float(mu), ptr(Dd),
                                       naux, ptr(Wc), tp,
                                       ntau, ptr(st), S, mode,
                                       ptr(branch), ptr(ws), ws.numel(), ptr(err.t),
                                       stream_ptr(stream)), 'mbpt_sigma_branch_sums')
    if own:
        err.check('mbpt_sigma_branch_sums')
    return branch


def sigma_frequency(branch, C, S, stream=None):
    """Sigma_c(i w_p) = -1/2 [C (S> + S<) + i S (S> - S<)] as a complex
    (nstates, npade) device tensor: ``imaginary_time.py:525-532``."""
    dev = branch.device
    ntau, nstates = branch.shape[1], branch.shape[2]
    Cd = torch.as_tensor(np.ascontiguousarray(C, dtype=np.float64), device=dev)
    Sd = torch.as_tensor(np.ascontiguousarray(S, dtype=np.float64), device=dev)
    npade = Cd.shape[0]
    out = torch.empty((nstates, npade, 2), dtype=torch.float64, device=dev)
    bc = branch.contiguous()  # held until the call has launched its kernel
    check(lib().mbpt_sigma_frequency(ptr(bc), ntau, nstates, ptr(Cd), ptr(Sd),
                                     npade, ptr(out), stream_ptr(stream)),
          'mbpt_sigma_frequency')
    return torch.view_as_complex(out)


def qp_solve(sigma, pade_freq, eps_anchor, states, nocc, mu, xc=None, greedy=True,
             warm=None, stream=None):
    """Roots, Z, flags and Sigma-evaluation counts of the QP equations of all
    states at once (device tensors): ``qp_solve.py:575-695`` per-state loop
    with ``:529-558`` and ``Solvers/qp_equation.py:1353-1393``. `warm`
    (nstates) predicted roots warm-start a Newton solve, the scan remaining
    the fallback."""
    dev = sigma.device
    sig = torch.view_as_real(sigma.contiguous()).contiguous()
    S, npade = sigma.shape
    pf_h, pp = host_array(pade_freq)
    ea = to_device(eps_anchor, dev)
    st = torch.as_tensor(np.asarray(states, dtype=np.int64), device=dev)
    xcd = None if xc is None else to_device(np.broadcast_to(np.asarray(xc, float), (S,))
                                            if not isinstance(xc, torch.Tensor) else xc, dev)
    wd = None if warm is None else to_device(warm, dev)
    roots = torch.empty(S, dtype=torch.float64, device=dev)
    z = torch.empty(S, dtype=torch.float64, device=dev)
    flags = torch.empty(S, dtype=torch.int32, device=dev)
    evals = torch.empty(S, dtype=torch.int32, device=dev)
    ws = WORKSPACE.get(1 << 16, dev)
    check(lib().mbpt_qp_solve(ptr(sig), pp, npade, ptr(ea), ptr(xcd), ptr(st), S, int(nocc),
                              float(mu), int(bool(greedy)), ptr(wd), ptr(roots), ptr(z),
                              ptr(flags), ptr(evals), ptr(ws), ws.numel(), stream_ptr(stream)),
          'mbpt_qp_solve')
    return roots, z, flags, evals


def imaginary_axis_sample_points(freq_points, nocc, p, mu):
    """(z_fit, query): the Pade sample points z = mu -/+ i omega_p of state p,
    below mu for an occupied state, and the signed frequencies themselves
    (``qp_solve.py:698-703``, whose callers unpack both)."""
    sign = -1.0 if p < nocc else 1.0
    query = sign * np.asarray(freq_points, float)
    return mu + 1j * query, query


def solve_qp_from_imaginary_axis(eps, p_state, xc_correction, z_fit, sigma_iw, greedy=True,
                                 max_order=None, with_z=False):
    """One state's Pade continuation and QP root of largest Z on the device
    (``qp_solve.py:529-558``): the sample points are mu -/+ i omega_p
    (`imaginary_axis_sample_points`; the lower branch carries the conjugate
    values), which the QP kernel takes as (omega_p, mu, branch)."""
    if max_order is not None:
        raise NotImplementedError('a cap on the Pade order is outside the device route')
    z = np.asarray(z_fit, complex)
    mu = float(z.real[0])
    lower = bool(z.imag[0] < 0)
    if not (np.allclose(z.real, mu, rtol=0, atol=0)
            and np.all(np.sign(z.imag) == np.sign(z.imag[0]))):
        raise NotImplementedError('the device QP solve takes sample points mu -/+ i omega')
    freq = np.abs(z.imag)
    sig = np.asarray(sigma_iw, complex)
    sig = np.conj(sig) if lower else sig   # the kernel conjugates an occupied state itself
    eps = np.asarray(eps, float)
    p = int(p_state)
    dev = require_device()
    sigma = torch.as_tensor(sig[None, :], dtype=torch.complex128, device=dev)
    roots, zz, flags, _ = qp_solve(sigma, freq, eps, [p], p + 1 if lower else p, mu,
                                   xc=[float(xc_correction)], greedy=greedy)
    _report_flags(flags.cpu().numpy(), [p])
    root = float(roots[0])
    return (root, float(zz[0])) if with_z else root


def _state_list(states, limit=12):
    shown = ', '.join(str(int(s)) for s in states[:limit])
    return shown + (f', ... ({len(states) - limit} more)' if len(states) > limit else '')


def _report_flags(flags_h, states):
    """One warning per kind for a whole solve: the count and the orbitals
    (the first dozen named), as the reference's named flags report a
    condition once per call rather than once per state."""
    states = np.atleast_1d(states)
    flags_h = np.asarray(flags_h)
    none = states[(flags_h & QP_FLAG_NO_ROOT) != 0]
    outside = states[((flags_h & QP_FLAG_NO_ROOT) == 0) & ((flags_h & QP_FLAG_Z_OUTSIDE) != 0)]
    if len(none):
        warnings.warn(f'{len(none)} of {len(states)} orbitals have no root of the '
                      f'quasiparticle equation in the widest scan window: '
                      f'{_state_list(none)}', QPNoRoot, stacklevel=3)
    if len(outside):
        warnings.warn(f'{len(outside)} of {len(states)} orbitals keep a root with Z outside '
                      f'(0, 1]: {_state_list(outside)}', QPWeightOutside, stacklevel=3)


class SweepResult(dict):
    """Outputs of one chi0 -> W -> Sigma -> QP sweep (device tensors and
    host arrays), with `timings` in seconds per stage (CUDA events)."""


def screened_tau_blocked(X, D, eps, nocc, axes, freq_block, precision=None, stream=None,
                         err=None, out=None):
    """W(tau) = sum_w Ctw[tau, w] (W(i w) - I) with chi0 held for `freq_block`
    frequencies at a time (``GW/imaginary_time.py:230-348``,
    `screened_interaction_tau_blocked`): per block the chi0 sweep onto the
    block's frequencies (the tau sweep recomputed, a factor nfreq/freq_block
    in its time), the Dyson step, and the block's share added onto W(tau).
    Returns (Wt, logdet, trace, info) over all frequencies."""
    dev = require_device()
    grid = axes.grid
    nfreq, nb = grid.nfreq, int(freq_block)
    if nb < 1:
        raise ValueError(f'freq_block must be positive, got {freq_block}')
    naux = D.shape[1]
    cw, Ctw = np.asarray(grid.cosft_wt, float), np.asarray(axes.Ctw, float)
    Wt = out if out is not None else torch.empty((len(Ctw), naux, naux), dtype=torch.float64,
                                                 device=dev)
    logdet = torch.empty(nfreq, dtype=torch.float64, device=dev)
    trace = torch.empty(nfreq, dtype=torch.float64, device=dev)
    info = np.zeros(nfreq, dtype=np.int32)
    blk = BUFFERS.take('sweep_chi0', (min(nb, nfreq), naux, naux), dev)
    ctx = torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext()
    with ctx:
        Wt.zero_()
    for f0 in range(0, nfreq, nb):
        f1 = min(f0 + nb, nfreq)
        c = blk[:f1 - f0]
        chi0_sweep(X, D, eps, nocc, grid.tau_points, cw[f0:f1], mu=axes.mu,
                   precision=precision, stream=stream, out=c, err=err)
        ld, tr, inf, _ = dyson_batch(c, want_w=True, stream=stream, precision=precision,
                                     err=err)
        with ctx:
            logdet[f0:f1].copy_(ld)
            trace[f0:f1].copy_(tr)
        info[f0:f1] = inf
        transform(c, np.ascontiguousarray(Ctw[:, f0:f1]), stream, out=Wt, accumulate=True)
    return Wt, logdet, trace, info


def gw_sweep(X, D, eps, nocc, states=None, ntau='auto', axes=None, precision=None,
             eps_anchor=None, xc_diagonal=None, greedy=True, warm=None, keep=False,
             stream=None, timings=None, freq_block=None, _deferred=True):
    """The whole space-time G0W0 sweep on device-resident (or host) inputs.

    Returns a SweepResult with 'roots', 'z', 'flags', 'evals' (device),
    'sigma' (nstates, npade) complex, 'axes', and with `keep` also 'Wt' and
    'W_minus_I'. eps_anchor: the spectrum the equation is anchored on (evGW);
    None is eps. timings: a dict receiving per-stage device times.
    freq_block: hold chi0 for that many frequencies at a time
    (`screened_tau_blocked`; 't_chi0' then times the whole blocked build of
    W(tau) and 't_dyson' is zero); W - I is then not kept.

    The Dyson step issues every frequency's inverse without reading its info
    word (no host wait inside the sweep); the words are read with the sweep's
    error word at its end, and a sweep that met a frequency where 1 - chi0 is
    not positive definite is repeated with the Dyson step's LU fallback.
    """
    dev = require_device()
    # host inputs cross to the device once, here (both halves of the sweep read them)
    X, D = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    n = len(eps_h)
    states = np.arange(n) if states is None else np.atleast_1d(np.asarray(states, int))
    if axes is None:
        axes = space_time_axes(eps_h, nocc, ntau=ntau,
                               anchor=None if eps_anchor is None else _eps_host(eps_anchor))
    mu = axes.mu
    check_mixed_weights(precision, axes.grid.cosft_wt, axes.Ctw, axes.C, axes.S)
    # one device error word for the sweep, read once at its end with the
    # Dyson step's info words: no host sync between the stages
    err = _Err(dev)
    ev = None
    if timings is not None:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ev[0].record()
    naux = D.shape[1]
    if freq_block is not None and int(freq_block) < axes.grid.nfreq:
        Wt, logdet, trace, info = screened_tau_blocked(
            X, D, eps_h, nocc, axes, freq_block, precision, stream, err,
            out=None if keep else BUFFERS.take('sweep_wt', (len(axes.Ctw), naux, naux), dev))
        if ev:
            ev[1].record()
            ev[2].record()
        e_c = torch.empty((), dtype=torch.float64, device=dev)
        ow = torch.as_tensor(np.asarray(axes.grid.omega_weights, float), device=dev)
        check(lib().mbpt_energy_sum(ptr(logdet), ptr(trace), ptr(ow), len(ow), ptr(e_c),
                                    stream_ptr(stream)), 'mbpt_energy_sum')
        return _sweep_tail(X, D, eps_h, nocc, states, axes, precision, eps_anchor, xc_diagonal,
                           greedy, warm, keep, stream, timings, err, ev, Wt, None, info, e_c)
    # the two 10 GB-class intermediates come from the per-device buffer cache
    # unless the caller keeps them
    chi0, _ = chi0_sweep(X, D, eps_h, nocc, axes.grid.tau_points, axes.grid.cosft_wt, mu=mu,
                         precision=precision, stream=stream,
                         out=None if keep else BUFFERS.take(
                             'sweep_chi0', (axes.grid.nfreq, naux, naux), dev), err=err)
    if ev:
        ev[1].record()
    logdet, trace, info, _ = dyson_batch(chi0, want_w=True, stream=stream,
                                         precision=precision, err=err, deferred=_deferred)
    # E_c from the same factorisations: the frequency axis is a minimax quadrature
    e_c = torch.empty((), dtype=torch.float64, device=dev)
    ow = torch.as_tensor(np.asarray(axes.grid.omega_weights, float), device=dev)
    check(lib().mbpt_energy_sum(ptr(logdet), ptr(trace), ptr(ow), len(ow), ptr(e_c),
                                stream_ptr(stream)), 'mbpt_energy_sum')
    if ev:
        ev[2].record()
    Wt = w_tau_from_frequencies(
        chi0, axes.Ctw, stream,
        out=None if keep else BUFFERS.take('sweep_wt', (len(axes.Ctw), naux, naux), dev))
    W_minus_I = chi0 if keep else None
    del chi0
    res = _sweep_tail(X, D, eps_h, nocc, states, axes, precision, eps_anchor, xc_diagonal,
                      greedy, warm, keep, stream, timings, err, ev, Wt, W_minus_I, info, e_c)
    if _deferred and res['dyson_info'].any():
        # a frequency whose 1 - chi0 is not positive definite: its W was not
        # valid, so everything after the Dyson step is redone with its LU
        return gw_sweep(X, D, eps_h, nocc, states=states, axes=axes, precision=precision,
                        eps_anchor=eps_anchor, xc_diagonal=xc_diagonal, greedy=greedy,
                        warm=warm, keep=keep, stream=stream, timings=timings,
                        _deferred=False)
    return res


def _sweep_tail(X, D, eps_h, nocc, states, axes, precision, eps_anchor, xc_diagonal, greedy,
                warm, keep, stream, timings, err, ev, Wt, W_minus_I, info, e_c):
    """The self-energy half of `gw_sweep` from W(tau): branch sums, Sigma(i w),
    the (warm-started) QP solve, and the result."""
    mu = axes.mu
    branch = sigma_branch_sums(X, D, Wt, eps_h, nocc, axes.tau_sigma, states, mu, precision,
                               stream, err=err)
    sigma = sigma_frequency(branch, axes.C, axes.S, stream)
    if ev:
        ev[3].record()
    anchor = eps_h if eps_anchor is None else _eps_host(eps_anchor)
    if warm is not None and hasattr(warm, 'predict_roots'):
        # the learned warm start: features from this sweep's Sigma and the
        # states' exchange diagonal, in the sweep's precision
        from .qp_mlp import exchange_diagonal
        sx = exchange_diagonal(X, D, eps_h, nocc, states, mu, precision=precision, err=err)
        warm = warm.predict_roots(X, D, eps_h, nocc, axes, eps_anchor=anchor, sx=sx,
                                  sweep=SweepResult(sigma=sigma, axes=axes, states=states))
    elif callable(warm):
        # a predictor that reads this sweep's Sigma
        warm = warm(SweepResult(sigma=sigma, axes=axes, states=states))
    roots, z, flags, evals = qp_solve(sigma, axes.pade_freq, anchor, states, nocc, mu,
                                      xc=xc_diagonal, greedy=greedy, warm=warm, stream=stream)
    if ev:
        ev[4].record()
        ev[4].synchronize()
        for k, name in enumerate(('t_chi0', 't_dyson', 't_sigma', 't_qp')):
            timings[name] = ev[k].elapsed_time(ev[k + 1]) / 1e3
        timings['dyson_frequencies'] = axes.grid.nfreq
        timings['ntau'] = axes.ntau
    err.check('gw_sweep')
    if isinstance(info, torch.Tensor):
        info = info.cpu().numpy()
    res = SweepResult(roots=roots, z=z, flags=flags, evals=evals, sigma=sigma, axes=axes,
                      states=states, branch=branch, dyson_info=info, e_c=e_c)
    if keep:
        res['Wt'] = Wt
        res['W_minus_I'] = W_minus_I
    return res


def gw_space_time(X, D, eps, nocc, states=None, ntau='auto', precision=None,
                  eps_anchor=None, xc_diagonal=None, greedy=True, with_z=False,
                  failures=None, timings=None, warm=None):
    """QP energies (Hartree, host array) of `states`, the equation
    w = eps_p + xc_p + Re Sigma_c(w) solved for the root of largest Z, on the
    synthetic or caller-built ISDF factors X (M x norb, MO collocation) and
    D (M x naux)."""
    t0 = time.perf_counter()
    res = gw_sweep(X, D, eps, nocc, states=states, ntau=ntau, precision=precision,
                   eps_anchor=eps_anchor, xc_diagonal=xc_diagonal, greedy=greedy,
                   timings=timings, warm=warm)
    roots = res['roots'].cpu().numpy()
    z = res['z'].cpu().numpy()
    flags = res['flags'].cpu().numpy()
    _report_flags(flags, res['states'])
    if failures is not None:
        for s, f in zip(res['states'], flags):
            if f & QP_FLAG_PADE_FAILED:
                failures[int(s)] = 'FloatingPointError: greedy Pade ordering failed'
    if timings is not None:
        timings['t_total_host'] = time.perf_counter() - t0
    return (roots, z) if with_z else roots


def gw_sweep_unrestricted(X_mos, D, spectra, noccs, states=None, ntau='auto', axes=None,
                          precision=None, eps_anchors=None, xc_diagonals=None, greedy=True,
                          channels=(0, 1), stream=None):
    """The space-time G0W0 sweep of an unrestricted reference
    (``GW/space_time.py:866-1009``, serial, in core): one W from
    chi0_alpha + chi0_beta (each half the restricted chi0 of that spin's
    collocation X_mos[s], spectrum and occupation, at its own mid-gap), then
    for each channel in `channels` the restricted self-energy sweep on that
    channel's orbitals (Sigma_s = -G_s W has no spin factor) and its QP roots,
    Sigma sampled through the channel's own mid-gap.

    states: per channel, None (all) or the orbitals; eps_anchors and
    xc_diagonals: per channel or None. Returns {'channels': {s: SweepResult},
    'axes', 'e_c' (the spin-summed RPA energy from the same factorisations),
    'dyson_info'}.
    """
    dev = require_device()
    X_mos = [to_device(X, dev) for X in X_mos]
    D = to_device(D, dev)
    spectra = [_eps_host(e) for e in spectra]
    noccs = [int(n) for n in noccs]
    if len(X_mos) != 2 or len(spectra) != 2 or len(noccs) != 2:
        raise ValueError('an unrestricted sweep takes two spin channels')
    if axes is None:
        axes = space_time_axes_unrestricted(
            spectra, noccs, ntau=ntau,
            anchors=None if eps_anchors is None else [_eps_host(a) for a in eps_anchors])
    check_mixed_weights(precision, axes.grid.cosft_wt, axes.Ctw, axes.C, axes.S)
    err = _Err(dev)
    naux = D.shape[1]
    shape = (axes.grid.nfreq, naux, naux)
    chi0, _ = chi0_sweep(X_mos[0], D, spectra[0], noccs[0], axes.grid.tau_points,
                         axes.grid.cosft_wt, mu=axes.mu[0], precision=precision,
                         stream=stream, out=BUFFERS.take('sweep_chi0', shape, dev), err=err)
    beta, _ = chi0_sweep(X_mos[1], D, spectra[1], noccs[1], axes.grid.tau_points,
                         axes.grid.cosft_wt, mu=axes.mu[1], precision=precision,
                         stream=stream, err=err)
    # spin_summed: half of each spin's restricted chi0
    with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
        chi0.add_(beta).mul_(0.5)
    del beta
    logdet, trace, info, _ = dyson_batch(chi0, want_w=True, stream=stream,
                                         precision=precision, err=err)
    e_c = torch.empty((), dtype=torch.float64, device=dev)
    ow = torch.as_tensor(np.asarray(axes.grid.omega_weights, float), device=dev)
    check(lib().mbpt_energy_sum(ptr(logdet), ptr(trace), ptr(ow), len(ow), ptr(e_c),
                                stream_ptr(stream)), 'mbpt_energy_sum')
    Wt = w_tau_from_frequencies(
        chi0, axes.Ctw, stream,
        out=BUFFERS.take('sweep_wt', (len(axes.Ctw), naux, naux), dev))
    del chi0
    out = {}
    for s in channels:
        eps_s, n_s, mu_s = spectra[s], noccs[s], axes.mu[s]
        st = states[s] if states is not None else None
        st = np.arange(len(eps_s)) if st is None else np.atleast_1d(np.asarray(st, int))
        branch = sigma_branch_sums(X_mos[s], D, Wt, eps_s, n_s, axes.tau_sigma, st, mu_s,
                                   precision, stream, err=err)
        sigma = sigma_frequency(branch, axes.C, axes.S, stream)
        anchor = eps_s if eps_anchors is None else _eps_host(eps_anchors[s])
        xc = None if xc_diagonals is None else xc_diagonals[s]
        roots, z, flags, evals = qp_solve(sigma, axes.pade_freq, anchor, st, n_s, mu_s,
                                          xc=xc, greedy=greedy, stream=stream)
        out[s] = SweepResult(roots=roots, z=z, flags=flags, evals=evals, sigma=sigma,
                             states=st, branch=branch)
    err.check('gw_sweep_unrestricted')
    return {'channels': out, 'axes': axes, 'e_c': e_c, 'dyson_info': info}


def _factors(factors):
    if factors is None:
        raise NotImplementedError(
            'building the ISDF factors needs pyscf (integrals and the fit); pass '
            'factors=(X_mo, D) or (X_mo, D, X_ao, coords)')
    if isinstance(factors, dict):
        return factors['X_mo'], factors['D']
    return factors[0], factors[1]


def solve_qp_energy_space_time(mf, mol, nocc, p_state, numerics=None, auxbasis=None,
                               radii=None, factors=None, greedy=True, dm_correction=None,
                               timings=None, distribute=None, comm=None, freq_block=None,
                               scratch_dir=None, extras=None, screen_r_cut=None,
                               sigma_x='mf', eps_anchor=None, sigma_x_matrix=None,
                               spin_channel='alpha', xc_diagonal=None, with_z=False,
                               failures=None, counts=None, grid_accuracy=None,
                               precision=None):
    """Drop-in for ``GW/space_time.py:631-863`` on a gas-phase reference with
    pre-built factors. Restricted: the mean field gives eps (mo_energy).
    Unrestricted (mo_energy of shape (2, nmo), nocc = (nalpha, nbeta)): channel
    `spin_channel`, from the factors' AO collocation (X_mo, D, X_ao[, coords])
    and mf.mo_coeff per spin (``GW/space_time.py:866-1009``);
    the static term <Sigma_x - v_xc> is `xc_diagonal` (0 on an HF reference,
    ``qp_solve.py:311``). numerics.quadrature: ntau_st ('auto' or a size),
    npade and w0_gl. Returns Hartree, a float for a scalar p_state."""
    for name, val in (('distribute', distribute), ('screen_r_cut', screen_r_cut),
                      ('sigma_x_matrix', sigma_x_matrix), ('extras', extras),
                      ('dm_correction (the static term is xc_diagonal here)', dm_correction)):
        if val:
            raise NotImplementedError(f'{name} is outside the one-GPU device route')
    if scratch_dir:
        raise NotImplementedError(
            'scratch_dir caches proj(tau) on disk between frequency blocks; the device '
            'recomputes the tau sweep per block instead (freq_block alone)')
    X, D = _factors(factors)
    eps = np.asarray(getattr(mf, 'mo_energy', mf), float)
    ntau, pade = 'auto', None
    if numerics is not None:
        q = numerics.quadrature
        ntau = q.ntau_st
        from .grids import pade_nodes
        pade = pade_nodes(q.npade, q.w0_gl)
    states = np.atleast_1d(p_state)
    if eps.ndim == 2:
        if freq_block:
            raise NotImplementedError(
                'freq_block on an unrestricted reference: the blocked path is built for one '
                'spin; run it unblocked')
        roots, z, evals = _unrestricted_channel(mf, nocc, states, factors, D, eps, ntau, pade,
                                                spin_channel, eps_anchor, xc_diagonal,
                                                greedy, precision, timings)
        if counts is not None:
            counts['sigma_evaluations'] = evals
        scalar = np.ndim(p_state) == 0
        if with_z:
            return (roots[0], z[0]) if scalar else (roots, z)
        return roots[0] if scalar else roots
    axes = space_time_axes(eps, nocc, ntau=ntau, pade_freq=pade,
                           anchor=None if eps_anchor is None else np.asarray(eps_anchor))
    res = gw_sweep(X, D, eps, nocc, states=states, axes=axes, precision=precision,
                   eps_anchor=eps_anchor, xc_diagonal=xc_diagonal, greedy=greedy,
                   timings=timings, freq_block=freq_block)
    if timings is not None:
        timings['ntau_auto'] = axes.ntau
        timings['tau_fit_error'] = axes.tau_fit_error
    roots = res['roots'].cpu().numpy()
    z = res['z'].cpu().numpy()
    _report_flags(res['flags'].cpu().numpy(), states)
    if counts is not None:
        counts['sigma_evaluations'] = res['evals'].cpu().numpy()
    scalar = np.ndim(p_state) == 0
    if with_z:
        return (roots[0], z[0]) if scalar else (roots, z)
    return roots[0] if scalar else roots


def _unrestricted_channel(mf, nocc, states, factors, D, eps, ntau, pade, spin_channel,
                          eps_anchor, xc_diagonal, greedy, precision, timings):
    """One channel of an unrestricted reference (``GW/space_time.py:866-1009``):
    each spin's collocation X_ao C_s off the one factorization, one W from both
    spins, the channel's Sigma and roots. Returns host (roots, z, evals)."""
    if spin_channel not in ('alpha', 'beta'):
        raise ValueError(f"spin_channel must be 'alpha' or 'beta', got {spin_channel!r}")
    spin = 0 if spin_channel == 'alpha' else 1
    X_ao = factors.get('X_ao') if isinstance(factors, dict) else (
        tuple(factors) + (None,) * 4)[2]
    if X_ao is None:
        raise ValueError(
            'an unrestricted reference needs the AO collocation of the factors, '
            '(X_mo, D, X_ao[, coords]): each spin projects it on its own orbitals')
    dev = require_device()
    Xa = to_device(X_ao, dev)
    X_mos = [Xa @ to_device(c, dev) for c in mf.mo_coeff]
    noccs = tuple(int(n) for n in nocc)
    anchors = None
    if eps_anchor is not None:
        anchors = np.asarray(eps_anchor, float)
        if anchors.shape != (2, eps.shape[1]):
            raise ValueError(f'an unrestricted eps_anchor is one spectrum per spin, shape '
                             f'(2, {eps.shape[1]}); got {anchors.shape}')
    axes = space_time_axes_unrestricted(list(eps), noccs, ntau=ntau, pade_freq=pade,
                                        anchors=anchors)
    per = [None, None]
    per[spin] = states
    xcs = None
    if xc_diagonal is not None:
        xcs = [None, None]
        xcs[spin] = xc_diagonal
    res = gw_sweep_unrestricted(X_mos, D, list(eps), noccs, states=per, axes=axes,
                                precision=precision,
                                eps_anchors=None if anchors is None else list(anchors),
                                xc_diagonals=xcs, greedy=greedy, channels=(spin,))
    if timings is not None:
        timings['ntau_auto'] = axes.ntau
        timings['tau_fit_error'] = axes.tau_fit_error
    ch = res['channels'][spin]
    _report_flags(ch['flags'].cpu().numpy(), states)
    return ch['roots'].cpu().numpy(), ch['z'].cpu().numpy(), ch['evals'].cpu().numpy()


def solve_qp_diagonal_space_time(mf, mol, nocc, states=None, **kw):
    """``GW/space_time.py:1091-1105``: (qp energies, states)."""
    n = np.asarray(getattr(mf, 'mo_energy', mf)).shape[-1]
    states = np.arange(n) if states is None else np.atleast_1d(states)
    return solve_qp_energy_space_time(mf, mol, nocc, states, **kw), states


HARTREE_TO_EV = 27.211386245988  # MBPTcode constants.py:11 (CODATA 2018)
# self_consistency values entering the evGW loop and the screening each keeps
# (``GW/qp_energy.py:64-65``)
EVGW_SCREENING = {'evgw': 'updated', 'ev': 'updated', 'evgw0': 'fixed', 'ev0': 'fixed'}


class _MeanFieldView:
    """The fields of a mean field the space-time drivers read, for a caller
    that hands a bare spectrum with nocc (or an object lacking some)."""

    def __init__(self, mf, eps, nocc):
        self.__dict__.update(getattr(mf, '__dict__', {}))
        self.mo_energy = np.asarray(eps, float)
        if isinstance(nocc, tuple):
            self.nelec = nocc
        elif not hasattr(self, 'mo_occ'):
            self.mo_occ = np.where(np.arange(self.mo_energy.size) < nocc, 2.0, 0.0)


def _mean_field_view(mf, eps, nocc):
    return _MeanFieldView(mf, eps, nocc)


def _resolve_states(state, nocc):
    """'homo', an index or a list of them -> orbital indices
    (``qp_energy.py:608-616``)."""
    if state == 'homo':
        return [nocc - 1]
    if isinstance(state, list):
        return state
    if isinstance(state, (int, np.integer)):
        return [int(state)]
    raise ValueError(f'Invalid state parameter: {state}')


def calc_qp_energy(mf, selfenergy='GW', polarizability='RPA', df=True, eta=None, state='homo',
                   spin_channel='alpha', printSpectralFunction=False, dm_correction=None,
                   tda=False, nroots=8, mode='casida', self_consistency='G0W0',
                   eps_anchor=None, n_workers=None, continuation=None, return_z=False,
                   solver='auto', equilibrium=False, out=None, **route_kwargs):
    """Quasiparticle energies in eV (``GW/qp_energy.py:294-616``), mode
    'space-time' on pre-built factors (route_kwargs['factors'] = (X_mo, D) or
    (X_mo, D, X_ao)): G0W0 with continuation 'pade' (the default; no Z, as
    the reference), 'cd' or 'laplace' (the contour with explicit or cubic
    residues, Z from its slope), or self_consistency 'evGW'. mf: an object
    with mo_energy and mo_occ (or route_kwargs['nocc']). The reference's
    refusals are kept: GW@RPA on density fitting only, no eta, no tda; the
    Casida and imaginary-frequency modes are other routes and refused; 'sop'
    solves the contour's pole model."""
    if mode != 'space-time':
        raise NotImplementedError(f"mode={mode!r}: the device route is mode='space-time'")
    if isinstance(selfenergy, list) or str(selfenergy).upper() != 'GW':
        raise ValueError(f"mode='space-time' implements GW only, got selfenergy={selfenergy!r}")
    if str(polarizability).upper() != 'RPA':
        raise ValueError(f"mode='space-time' implements RPA screening only, got "
                         f"polarizability={polarizability!r}")
    if not df:
        raise ValueError("mode='space-time' requires density fitting (df=True).")
    if tda:
        raise ValueError("tda has no meaning for mode='space-time'")
    if eta is not None:
        raise ValueError("eta broadens nothing on mode='space-time'")
    continuation = 'pade' if continuation is None else continuation
    if continuation not in ('pade', 'laplace', 'cd', 'sop'):
        raise NotImplementedError(f'continuation={continuation!r} is outside the device route')
    eps = np.asarray(getattr(mf, 'mo_energy', mf), float)
    nocc = route_kwargs.pop('nocc', None)
    if nocc is None:
        occ = np.asarray(getattr(mf, 'mo_occ'))
        nocc = (tuple(int((o > 0).sum()) for o in occ) if occ.ndim == 2
                else int((occ > 0).sum()))
    nocc_ch = nocc[0 if spin_channel == 'alpha' else 1] if isinstance(nocc, tuple) else nocc
    states = _resolve_states(state, nocc_ch)
    consistency = str(self_consistency).lower()
    if consistency in EVGW_SCREENING:
        if eps_anchor is not None:
            raise TypeError(f'self_consistency={self_consistency!r} sets its own anchor every '
                            f'cycle, so eps_anchor would be overwritten by the loop rather '
                            f'than read')
        if continuation != 'pade':
            raise ValueError(f"self_consistency={self_consistency!r} drives continuation="
                             f"'pade' only, not {continuation!r}")
        from .evgw import evgw_eigenvalues
        e, _ = evgw_eigenvalues(_mean_field_view(mf, eps, nocc), None, mode='space-time',
                                screening=EVGW_SCREENING[consistency], **route_kwargs)
        e_ch = e if e.ndim == 1 else e[0 if spin_channel == 'alpha' else 1]
        res = [float(e_ch[p]) * HARTREE_TO_EV for p in states]
        z = None
    elif consistency != 'g0w0':
        raise NotImplementedError(f'self_consistency={self_consistency!r} is outside the device '
                                  'route')
    elif continuation in ('laplace', 'cd', 'sop'):
        from .contour import solve_qp_energy_contour
        ev, zs, _ = solve_qp_energy_contour(mf if eps.ndim == 2 else eps, None, nocc,
                                            np.asarray(states), continuation=continuation,
                                            eps_anchor=eps_anchor, spin_channel=spin_channel,
                                            **route_kwargs)
        res, z = list(ev), list(zs)
    else:
        if return_z:
            raise ValueError("continuation='pade' returns no Z: differentiating a Thiele "
                             "recursion divides by vanishing inverse differences")
        e = solve_qp_energy_space_time(mf, None, nocc, np.asarray(states),
                                       dm_correction=dm_correction, eps_anchor=eps_anchor,
                                       spin_channel=spin_channel, **route_kwargs)
        res, z = [float(x) * HARTREE_TO_EV for x in np.atleast_1d(e)], None
    if return_z and z is None:
        raise ValueError('this route returns no Z')
    if not isinstance(state, list):
        return (res[0], z[0]) if return_z else res[0]
    return (res, z) if return_z else res
