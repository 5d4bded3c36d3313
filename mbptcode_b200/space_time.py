"""Space-time polarizability, Dyson step and dRPA energy on the B200.

Mirrors the kernel seams of MBPTcode's
``src/SingleReference/LinearResponse/space_time.py`` with the same names,
argument meaning and error behaviour; the arithmetic runs in libmbpt_b200
(include/mbpt_b200.h). Inputs may be NumPy arrays (results come back as
NumPy, as the reference returns them) or torch tensors (results stay on the
device).

``precision``: 'fp64' (default; every product in FP64, the reference's
arithmetic) or 'mixed' (the N^3 products as split-BF16 tensor-core products
with FP32 accumulation; transforms, Cholesky and sums stay FP64).
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from . import _lib
from ._lib import MODES, WORKSPACE, check, host_array, lib, ptr, require_device, stream_ptr

_DEFAULT_PRECISION = ['fp64']


def set_default_precision(precision):
    """Precision used where a call does not name one ('fp64' or 'mixed')."""
    if precision not in MODES:
        raise ValueError(f'precision {precision!r}: choose one of {sorted(MODES)}')
    _DEFAULT_PRECISION[0] = precision


def _mode(precision):
    p = _DEFAULT_PRECISION[0] if precision is None else precision
    if p not in MODES:
        raise ValueError(f'precision {p!r}: choose one of {sorted(MODES)}')
    return MODES[p]


#: largest transform weight the mixed path accepts: its products carry ~1e-5
#: relative error, which a tau <-> omega sum cancelling by max|w| would lift
#: past the accuracy bars (the unregularised 16/18-point grids reach 1e8-1e9)
MIXED_WEIGHT_LIMIT = 1e3


def check_mixed_weights(precision, *weights):
    if _mode(precision) != MODES['mixed']:
        return
    worst = max(float(np.abs(np.asarray(w)).max()) for w in weights)
    if not worst <= MIXED_WEIGHT_LIMIT:
        raise ValueError(
            f'mixed precision refused: the tau <-> omega transform weights reach '
            f'{worst:.3g} (limit {MIXED_WEIGHT_LIMIT:g}), so split-BF16 product errors '
            f'would not survive the transform; use precision="fp64" or a grid of 20 '
            f'or more points (regularised fit)')


def to_device(a, device, dtype=torch.float64):
    """`a` on `device` as a contiguous `dtype` tensor. A pinned host tensor is
    copied asynchronously (stream-ordered before the kernels that read it),
    so that the host work that follows overlaps the transfer."""
    if isinstance(a, torch.Tensor):
        pinned = a.device.type == 'cpu' and a.is_pinned() and a.dtype == dtype
        return a.to(device=device, dtype=dtype, non_blocking=pinned).contiguous()
    a = np.ascontiguousarray(a)
    if not a.flags.writeable:   # a broadcast view: torch wants memory it may own
        a = a.copy()
    return torch.as_tensor(a, dtype=dtype, device=device)


def back(t, like):
    """Return t as `like` is held: NumPy for NumPy input, the tensor otherwise."""
    if isinstance(like, torch.Tensor):
        return t
    return t.cpu().numpy()


class _Err:
    """The device error word of one call."""

    def __init__(self, device):
        self.t = torch.zeros(1, dtype=torch.int32, device=device)

    def check(self, where):
        v = int(self.t.item())
        if v:
            raise _lib.MBPTError(v, where + ' (device)')


def particle_hole_window(eps, nocc):
    """(gap, span, mu): ``src/Base/orbital_spaces.py:12-20``."""
    eps = np.asarray(eps, float)
    homo, lumo = eps[:nocc].max(), eps[nocc:].min()
    return lumo - homo, eps[nocc:].max() - eps[:nocc].min(), 0.5 * (homo + lumo)


def _eps_host(eps):
    return eps.detach().cpu().numpy() if isinstance(eps, torch.Tensor) else np.asarray(eps, float)


def _taus(tau_points, tau_indices):
    tau = np.asarray(tau_points, float)
    which = np.arange(len(tau)) if tau_indices is None else np.atleast_1d(tau_indices)
    return tau, which


def chi0_sweep(X, D, eps, nocc, tau_points, cosft_wt, mu=None, precision=None,
               want_proj=False, stream=None, out=None, err=None):
    """(chi0 (nfreq, naux, naux), proj (ntau, naux, naux) or None) as device
    tensors: the whole N^3 sweep in one library call. `out`: a contiguous
    FP64 device array of chi0's shape to write into. `err`: a device error
    word the caller checks later (no host sync here); None checks now."""
    dev = require_device()
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    ed = to_device(eps_h, dev)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    M, norb = Xd.shape
    naux = Dd.shape[1]
    if Dd.shape[0] != M or len(eps_h) != norb or not 0 < nocc < norb:
        raise ValueError(f'shapes: X {tuple(Xd.shape)}, D {tuple(Dd.shape)}, '
                         f'eps {len(eps_h)}, nocc {nocc}')
    tau_h, tp = host_array(tau_points)
    cw_h, cp = host_array(cosft_wt)
    ntau, nfreq = len(tau_h), cw_h.shape[0]
    if cw_h.shape != (nfreq, ntau):
        raise ValueError(f'cosft_wt is {cw_h.shape}, need (nfreq, {ntau})')
    mode = _mode(precision)
    check_mixed_weights(precision, cw_h)
    if out is not None:
        if tuple(out.shape) != (nfreq, naux, naux) or out.dtype != torch.float64 \
                or not out.is_contiguous() or out.device != dev:
            raise ValueError(f'out must be a contiguous FP64 ({nfreq}, {naux}, {naux}) array '
                             f'on {dev}')
        chi0 = out
    else:
        chi0 = torch.empty((nfreq, naux, naux), dtype=torch.float64, device=dev)
    proj = (torch.empty((ntau, naux, naux), dtype=torch.float64, device=dev)
            if want_proj else None)
    nbytes = lib().mbpt_chi0_workspace_bytes(M, norb, nocc, naux, ntau, mode)
    ws = WORKSPACE.get(nbytes, dev)
    own = err is None
    err = _Err(dev) if own else err
    check(lib().mbpt_chi0_sweep(ptr(Xd), M, norb, nocc, ptr(ed), float(mu), ptr(Dd), naux,
                                tp, ntau, cp, nfreq, mode, ptr(chi0), ptr(proj), ptr(ws),
                                ws.numel(), ptr(err.t), stream_ptr(stream)),
          'mbpt_chi0_sweep')
    if own:
        err.check('mbpt_chi0_sweep')
    return chi0, proj


def chi0_imaginary_frequency(X, D, eps, nocc, grid, mu=None, tau_indices=None,
                             tile_memory_gb=None, precision=None):
    """chi0(i omega) in the auxiliary basis, (nfreq, naux, naux):
    ``space_time.py:607-651``. tile_memory_gb is accepted for signature
    compatibility; the device sweep is not row-tiled."""
    tau, which = _taus(grid.tau_points, tau_indices)
    chi0, _ = chi0_sweep(X, D, eps, nocc, tau[which], np.asarray(grid.cosft_wt)[:, which],
                         mu=mu, precision=precision)
    return back(chi0, X)


def polarizability_projected_sweep(X, D, eps, nocc, tau_points, mu=None, tau_indices=None,
                                   tile_memory_gb=None, precision=None):
    """proj(tau) on every time point, (ntau, naux, naux), zero outside
    tau_indices: ``space_time.py:533-560``."""
    tau, which = _taus(tau_points, tau_indices)
    _, proj = chi0_sweep(X, D, eps, nocc, tau[which], np.zeros((1, len(which))), mu=mu,
                         precision=precision, want_proj=True)
    if len(which) != len(tau):
        full = torch.zeros((len(tau),) + tuple(proj.shape[1:]), dtype=proj.dtype,
                           device=proj.device)
        full[torch.as_tensor(which, device=proj.device)] = proj
        proj = full
    return back(proj, X)


def polarizability_projected_tau(X_o, X_v, e_o, e_v, D, tau, tile_memory_gb=None, out=None,
                                 work=None, tiles=None, precision=None):
    """proj(tau) at one time point from already-split branches and shifted
    energies: ``space_time.py:478-530``. ``tiles`` (a subset of grid-row
    tiles) is not supported: the device sweep covers every row."""
    if tiles is not None:
        raise NotImplementedError('a partial row-tile sum is not offered by the device sweep')
    X = np.concatenate([np.asarray(X_o), np.asarray(X_v)], axis=1) \
        if not isinstance(X_o, torch.Tensor) else torch.cat([X_o, X_v], dim=1)
    e = np.concatenate([np.asarray(e_o, float), np.asarray(e_v, float)])
    proj = polarizability_projected_sweep(X, D, e, len(e_o), [float(tau)], mu=0.0,
                                          precision=precision)[0]
    if out is not None:
        out[...] = proj
        return out
    return proj


def split_branches(X, eps, nocc, mu=None, branches=None):
    """``space_time.py:448-475``: (X_o, X_v, e_o, e_v, mu, occ, virt)."""
    eps = np.asarray(eps, float)
    occ, virt = np.arange(nocc), np.arange(nocc, len(eps))
    if mu is None:
        mu = particle_hole_window(eps, nocc)[2]
    if branches is not None:
        X_o, X_v = branches
    else:
        X_o, X_v = np.ascontiguousarray(X[:, occ]), np.ascontiguousarray(X[:, virt])
    return X_o, X_v, eps[occ] - mu, eps[virt] - mu, mu, occ, virt


class NonPositiveDielectric(RuntimeWarning):
    """det(1 - chi0) is not positive at an imaginary frequency."""


def dyson_batch(chi0, want_w=True, stream=None, precision='fp64', err=None, deferred=False):
    """In place over a device tensor (nfreq, naux, naux): chi0 -> W - I (or
    the Cholesky factors). Returns (logdet, trace, info, sign) with logdet and
    trace on the device and info/sign as host int arrays. The factorisation
    and log-determinant are FP64 in both precisions; 'mixed' forms the
    inverse from the FP64 factor by TF32x3 tensor-core products.
    deferred: no host wait; info comes back as a device int32 tensor and sign
    as None, and a nonzero info word means that frequency's results are not
    valid (repeat without `deferred`)."""
    dev = chi0.device
    mode = _mode(precision)
    nfreq, naux = chi0.shape[0], chi0.shape[-1]
    logdet = torch.empty(nfreq, dtype=torch.float64, device=dev)
    trace = torch.empty(nfreq, dtype=torch.float64, device=dev)
    own = err is None
    err = _Err(dev) if own else err
    ws = WORKSPACE.get(lib().mbpt_dyson_workspace_bytes(naux, nfreq, mode), dev)
    if deferred:
        info_d = torch.zeros(nfreq, dtype=torch.int32, device=dev)
        check(lib().mbpt_dyson_deferred(ptr(chi0), naux, nfreq, int(bool(want_w)), mode,
                                        ptr(logdet), ptr(trace), ptr(info_d), ptr(ws),
                                        ws.numel(), ptr(err.t), stream_ptr(stream)),
              'mbpt_dyson_deferred')
        if own:
            err.check('mbpt_dyson_deferred')
        return logdet, trace, info_d, None
    info = np.zeros(nfreq, dtype=np.int32)
    sign = np.ones(nfreq, dtype=np.int32)
    import ctypes
    rc = lib().mbpt_dyson(ptr(chi0), naux, nfreq, int(bool(want_w)), mode, ptr(logdet),
                          ptr(trace), info.ctypes.data_as(ctypes.c_void_p),
                          sign.ctypes.data_as(ctypes.c_void_p), ptr(ws), ws.numel(),
                          ptr(err.t), stream_ptr(stream))
    if rc not in (_lib.OK, _lib.ERR_NOT_SPD):
        check(rc, 'mbpt_dyson')
    if own:
        err.check('mbpt_dyson')
    return logdet, trace, info, sign


def dyson_screening(chi0, transform=None, correlation=False):
    """W = [I - T^T chi0 T]^-1 at one frequency (or a stack), minus I when
    `correlation`: ``space_time.py:956-968``, by Cholesky factorisation."""
    dev = require_device()
    c = to_device(chi0, dev)
    if transform is not None:
        T = to_device(transform, dev)
        c = T.T @ c @ T
    single = c.dim() == 2
    stack = (c[None] if single else c).clone()
    dyson_batch(stack, want_w=True)
    if not correlation:
        stack.diagonal(dim1=-2, dim2=-1).add_(1.0)
    out = stack[0] if single else stack
    return back(out, chi0)


def frequency_factor(d, w, imaginary, eta=0.0, slopes=False):
    """The bubble's frequency factor for pair energies d at frequency w
    (``LinearResponse/imaginary_frequency.py:25-59``), host FP64 on nov
    numbers: -2d/(d^2 + w^2) on the imaginary axis, 1/(w - d) - 1/(w + d) on
    the real one, a/(a^2 + eta^2) - b/(b^2 + eta^2) broadened (a = w - d,
    b = w + d). slopes=True returns (f, df/dd, df/dw), df/dw None on the
    imaginary axis."""
    d = np.asarray(d, float)
    if imaginary:
        den = d ** 2 + w ** 2
        f = -2.0 * d / den
        return (f, -2.0 * (w ** 2 - d ** 2) / den ** 2, None) if slopes else f
    a, b = w - d, w + d
    if eta == 0.0:
        f = 1.0 / a - 1.0 / b
        return (f, 1.0 / a ** 2 + 1.0 / b ** 2, -1.0 / a ** 2 + 1.0 / b ** 2) if slopes else f
    da, db = a ** 2 + eta ** 2, b ** 2 + eta ** 2
    f = a / da - b / db
    if not slopes:
        return f
    return (f, -(eta ** 2 - a ** 2) / da ** 2 - (eta ** 2 - b ** 2) / db ** 2,
            (eta ** 2 - a ** 2) / da ** 2 - (eta ** 2 - b ** 2) / db ** 2)


def chi0_aux(blocks, spin_factor=1.0, scratch=None, out=None, precision='fp64'):
    """chi0 = spin_factor sum_s (C_s f_s) C_s^T in the auxiliary basis, on the
    device (``LinearResponse/space_time.py:934-953``): blocks = [(C_ov, f)],
    C_ov (naux, n_ov) and f its pairs' frequency factor (`frequency_factor`).
    One mbpt_chi0_aux call per block, accumulating into `out` (a device
    (naux, naux) FP64 tensor, allocated when None), which is returned.
    precision 'fp64' (default: a symmetric rank-k DGEMM over column chunks)
    or 'mixed' (one split BF16x3 tensor-core product per block, ~1e-5
    relative; one block only). scratch is accepted for the reference's
    signature; the chunks live in the call's workspace. NumPy factors give
    a NumPy result unless `out` is given; device factors keep it on the
    device."""
    del scratch
    dev = require_device()
    mode = _mode(precision)
    blocks = list(blocks)
    if mode == MODES['mixed'] and len(blocks) > 1:
        raise ValueError("chi0_aux: precision='mixed' takes one block (stack the pairs)")
    host = out is None and bool(blocks) and not isinstance(blocks[0][0], torch.Tensor)
    err = _Err(dev)
    for s, (C, f) in enumerate(blocks):
        Cd = to_device(C, dev)
        naux, nov = Cd.shape
        fd = to_device(np.ascontiguousarray(f, dtype=float), dev)
        if fd.numel() != nov:
            raise ValueError(f'chi0_aux: f has {fd.numel()} pairs, C_ov {nov}')
        if out is None:
            out = torch.empty((naux, naux), dtype=torch.float64, device=dev)
        ws = WORKSPACE.get(lib().mbpt_chi0_aux_workspace_bytes(naux, nov, mode), dev)
        check(lib().mbpt_chi0_aux(ptr(Cd), naux, nov, Cd.stride(0), ptr(fd),
                                  float(spin_factor), int(s > 0), mode, ptr(out), ptr(ws),
                                  ws.numel(), ptr(err.t), stream_ptr()), 'mbpt_chi0_aux')
    if mode == MODES['mixed']:
        err.check('mbpt_chi0_aux')
    return out.cpu().numpy() if host else out


def _one_rank(comm, who):
    if comm is not None and comm.Get_size() > 1:
        raise NotImplementedError(f'{who}: rank splits are outside the one-GPU route')


def static_screening_matrix(X, D, eps, nocc, grid=None, mu=None, comm=None,
                            tile_memory_gb=None, branches=None, precision=None):
    """W = [1 - chi0(i omega = 0)]^-1 in the auxiliary basis
    (``space_time.py:1003-1050``): the BSE kernel's and the reaction field's
    static screened interaction. The grid's tau points form chi0 on its one
    frequency in a single device sweep (the reference's ordered sum of the
    tau addends is the transform's FP64 sum over tau), then the Dyson step
    (FP64 Cholesky; the inverse on the tensor cores in mixed precision).
    `branches` = (X_o, X_v) already split takes the place of X's columns;
    tile_memory_gb is accepted for signature compatibility."""
    _one_rank(comm, 'static_screening_matrix')
    from .grids import static_screening_grid
    eps_h = _eps_host(eps)
    if branches is not None:
        X_o, X_v = branches
        if X_o.shape[1] != nocc:
            raise ValueError(f'branches: X_o has {X_o.shape[1]} columns, nocc is {nocc}')
        cat = torch.cat if isinstance(X_o, torch.Tensor) else np.concatenate
        X = cat([X_o, X_v], 1)
    grid = static_screening_grid(eps_h, nocc) if grid is None else grid
    chi0, _ = chi0_sweep(X, D, eps_h, nocc, grid.tau_points, grid.cosft_wt, mu=mu,
                         precision=precision)
    return _static_w(chi0, precision, X)


def _static_w(chi0, precision, like):
    """W = [1 - chi0]^-1 of a (1, naux, naux) device chi0, in place."""
    dyson_batch(chi0, want_w=True,
                precision='mixed' if _mode(precision) == MODES['mixed'] else 'fp64')
    chi0.diagonal(dim1=-2, dim2=-1).add_(1.0)
    return back(chi0[0], like)


def spin_summed(kernel, X_mos, D, spectra, noccs, *args, **kwargs):
    """chi0_alpha + chi0_beta of an unrestricted reference from a kernel's
    restricted form (``space_time.py:774-796``): every kernel carries the
    closed-shell factor 2, so each spin contributes half the kernel on its own
    collocation, spectrum and occupation, at its own mid-gap."""
    out = None
    for X, eps, nocc in zip(X_mos, spectra, noccs):
        part = kernel(X, D, eps, nocc, *args,
                      mu=particle_hole_window(_eps_host(eps), nocc)[2], **kwargs)
        out = part if out is None else out + part
    return out * 0.5


def static_screening_matrix_unrestricted(X_mos, D, spectra, noccs, tau_target=None,
                                         precision=None):
    """`static_screening_matrix` of an unrestricted reference
    (``space_time.py:1053-1066``): one W from chi0_alpha + chi0_beta on a grid
    spanning both spins' transitions, with as many points as the harder spin
    needs. Both spins' chi0 sweeps accumulate on the device."""
    from .grids import (DEFAULT_TAU_TARGET, TimeFrequencyGrid, minimax_points_for_bse,
                        transition_range)
    target = DEFAULT_TAU_TARGET if tau_target is None else tau_target
    spectra = [_eps_host(e) for e in spectra]
    e_min, e_max = transition_range(spectra, noccs)
    ntau = max(minimax_points_for_bse(e, n, tau_target=target)[0]
               for e, n in zip(spectra, noccs))
    grid = TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, [0.0], [1.0],
                                           with_sine=False, with_inverse=False)

    def sweep(X, D, eps, nocc, mu=None):
        return chi0_sweep(X, D, eps, nocc, grid.tau_points, grid.cosft_wt, mu=mu,
                          precision=precision)[0]
    chi0 = spin_summed(sweep, X_mos, D, spectra, noccs)
    return _static_w(chi0, precision, X_mos[0])


def dielectric_log_determinant(one_minus_c, where, flags=None):
    """log|det(1 - c)| with a NonPositiveDielectric warning and the
    'nonpositive_det' flag when the determinant is not positive:
    ``space_time.py:1073-1097``. Takes the matrix 1 - c itself."""
    dev = require_device()
    m = to_device(one_minus_c, dev)
    n = m.shape[-1]
    chi = (torch.eye(n, dtype=torch.float64, device=dev) - m)[None].contiguous()
    logdet, _, info, sign = dyson_batch(chi, want_w=False)
    if info[0] != 0 and not sign[0] > 0:
        _flag_nonpositive(where, int(sign[0]), flags)
    return float(logdet[0].item())


def _flag_nonpositive(where, sign, flags):
    warnings.warn(f'det(1 - chi0) is not positive at {where} (sign {sign}): the RPA '
                  f'dielectric has been driven singular; log|det| is used.',
                  NonPositiveDielectric, stacklevel=3)
    if flags is not None:
        flags.setdefault('nonpositive_det', []).append(where)


def rpa_energy_device(X, D, eps, nocc, tau_points, cosft_wt, omega_weights, mu=None,
                      precision=None, want_proj=False, stream=None):
    """(E_c as a 0-d device tensor, info, proj or None): chi0 sweep, Cholesky
    log-determinants and the weighted frequency sum in one library call."""
    dev = require_device()
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    eps_h = _eps_host(eps)
    ed = to_device(eps_h, dev)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    M, norb = Xd.shape
    naux = Dd.shape[1]
    tau_h, tp = host_array(tau_points)
    cw_h, cp = host_array(cosft_wt)
    ow_h, op = host_array(omega_weights)
    ntau, nfreq = len(tau_h), cw_h.shape[0]
    mode = _mode(precision)
    check_mixed_weights(precision, cw_h)
    e_c = torch.empty((), dtype=torch.float64, device=dev)
    proj = (torch.empty((ntau, naux, naux), dtype=torch.float64, device=dev)
            if want_proj else None)
    info = np.zeros(nfreq, dtype=np.int32)
    nbytes = lib().mbpt_rpa_energy_workspace_bytes(M, norb, nocc, naux, ntau, nfreq, mode)
    ws = WORKSPACE.get(nbytes, dev)
    err = _Err(dev)
    import ctypes
    rc = lib().mbpt_rpa_energy(ptr(Xd), M, norb, nocc, ptr(ed), float(mu), ptr(Dd), naux, tp,
                               ntau, cp, op, nfreq, mode, ptr(e_c), ptr(proj),
                               info.ctypes.data_as(ctypes.c_void_p), ptr(ws), ws.numel(),
                               ptr(err.t), stream_ptr(stream))
    if rc not in (_lib.OK, _lib.ERR_NOT_SPD):
        check(rc, 'mbpt_rpa_energy')
    err.check('mbpt_rpa_energy')
    return e_c, info, proj


def rpa_correlation_energy_space_time(X, D, eps, nocc, grid, mu=None, tile_gb=None,
                                      screening=None, counter_term=None, comm=None,
                                      want_tape=False, flags=None, precision=None):
    """dRPA E_c = (1/2pi) sum_w w_w [log det(1 - chi0_w) + tr chi0_w]:
    ``space_time.py:1100-1183`` (gas phase, one GPU). The solvent fold
    (`screening`, `counter_term`) and the MPI split (`comm`) are outside this
    route."""
    if screening is not None or counter_term is not None:
        raise NotImplementedError('the solvent-folded energy is not on the device route')
    if comm is not None and getattr(comm, 'Get_size', lambda: 1)() > 1:
        raise NotImplementedError('the device route runs on one GPU, without MPI ranks')
    e_c, info, proj = rpa_energy_device(X, D, eps, nocc, grid.tau_points, grid.cosft_wt,
                                        grid.omega_weights, mu=mu, precision=precision,
                                        want_proj=want_tape)
    bad = [int(k) for k in np.nonzero(info)[0]]
    for k in bad:
        _flag_nonpositive(k, -1, None)
    if flags is not None and bad:
        flags.setdefault('nonpositive_det', []).extend(bad)
    value = float(e_c.item())
    if not want_tape:
        return value
    from types import SimpleNamespace
    return value, SimpleNamespace(proj_tau=back(proj, X), tau_indices=None, freq_indices=None)


def transform(values, weights, stream=None, out=None, accumulate=False):
    """sum_k weights[j, k] values[k] over (K, n, n) device tensors, FP64
    (into `out`, a contiguous (J, n, n) FP64 array, when given; added onto
    `out` with `accumulate`)."""
    dev = values.device
    K, n = values.shape[0], values.shape[-1]
    w = torch.as_tensor(np.ascontiguousarray(weights, dtype=np.float64), device=dev)
    J = w.shape[0]
    if out is None:
        if accumulate:
            raise ValueError('accumulate needs out')
        out = torch.empty((J, n, n), dtype=torch.float64, device=dev)
    elif tuple(out.shape) != (J, n, n) or out.dtype != torch.float64 or not out.is_contiguous():
        raise ValueError(f'out must be a contiguous FP64 ({J}, {n}, {n}) array')
    vc = values.contiguous()  # held until the call has launched its kernel
    fn = lib().mbpt_transform_acc if accumulate else lib().mbpt_transform
    check(fn(ptr(vc), K, n, ptr(w), J, ptr(out), stream_ptr(stream)),
          'mbpt_transform_acc' if accumulate else 'mbpt_transform')
    return out


__all__ = ['chi0_imaginary_frequency', 'polarizability_projected_sweep',
           'polarizability_projected_tau', 'split_branches', 'dyson_screening',
           'dielectric_log_determinant', 'rpa_correlation_energy_space_time',
           'NonPositiveDielectric', 'set_default_precision', 'chi0_sweep', 'dyson_batch',
           'rpa_energy_device', 'transform', 'particle_hole_window']
