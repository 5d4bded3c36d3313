"""Contour-deformation correlation self-energy on the B200.

Mirrors the kernel seams of MBPTcode's ``src/SingleReference/GW/contour_deformation.py``
and ``GW/real_screening.py`` with the same names and argument meaning:

    Sigma^c_pp(omega) = Sigma^int + Sigma^res,
    Sigma^int = -(1/pi) sum_kq c[k, q](omega) wc[k, q],
    wc[k, q]  = B_p[:, q]^T (W(i nu_k) - I) B_p[:, q],
    Sigma^res = sum_{q in residues} w_q (b_q^T W(|eps_q - omega|) b_q - b_q^T b_q),

with B_p = D^T diag(X[:, p]) X the state's three-index slice, W = [1 - chi0]^-1
on the contour's Gauss-Legendre frequencies nu_k, c the quadrature weights with
the Lorentzian's singular part integrated in closed form
(`cd_integral_weights`), and the residues' W at real frequencies below the gap
from the cosh transform of proj(tau) (`LaplaceRealScreening`).

On the device: proj(tau) on the contour's own time grid and chi0(i nu) by the
chi0 sweep and the tau -> omega transform, W - I by the Dyson step (one
batched FP64 Cholesky of every frequency), the slices and the screening
contraction (mbpt_three_index_slices, mbpt_screening_contraction: one W per
frequency serves every state) and each residue frequency's W. The quadrature
weights, the residue sets and the sums over k and q are host arithmetic on
nfreq x norb numbers. FP64 throughout.

The quasiparticle equation of this route, w = eps_p + xc + Sigma^c(w), is
solved as the reference solves it (`qp_energy_cd` on
``Solvers/qp_equation.py`` `solve_qp_equation_scan`, without a followed root):
a grid over the narrowest window about the bare level walked outward, cells
halved where the secant slope hides a pole, each bracket refined by Newton on
the closed-form slope (`sigma_cd_slope`) safeguarded by the bracket, the
weights of a positive-weight self-energy summing to one ending the walk.

Continuation 'cd' takes the residues' W from the explicit particle-hole
response instead (`ExplicitRealScreening`, ``real_screening.py:57-91``):
C_ov = B[:, occ, virt] from the occupied states' slices, chi0(freq) =
2 (C_ov f) C_ov^T by mbpt_chi0_aux (a symmetric rank-k FP64 product over
column chunks) and the Dyson step, which falls back from Cholesky to LU above
the particle-hole gap where 1 - chi0 is indefinite.
"""
from __future__ import annotations

import warnings
from collections import OrderedDict

import numpy as np
import torch

from ._lib import WORKSPACE, check, lib, ptr, require_device, stream_ptr
from .grids import TimeFrequencyGrid, gauss_legendre_grid, particle_hole_window
from .space_time import (_eps_host, chi0_aux, chi0_sweep, dyson_batch, frequency_factor,
                         to_device, transform)

# MBPTcode src/Base/numerics/constants.py
RESIDUE_ON_CONTOUR_TOL = 1e-10   # :461
CD_NFREQ = 64                    # :478
CD_NTAU = 24                     # :493
LAPLACE_SCREENING_TOL = 1e-8     # :577
QP_GRAPHICAL_N_OMEGA = 150       # :273
QP_ROOT_TOL, QP_ROOT_MAX_ITER = 1e-11, 100   # :501-502
QP_WINDOW_Z_MIN = 0.5            # :553
QP_SEARCH_WINDOW_TIERS = ((0.0, 0.5), (1.5, 1.0), (4.0, 2.0))   # :1464
QP_SCAN_SECANT_MIN, QP_SCAN_SPLIT_DEPTH = 0.5, 6                # :1613-1614
QP_WEIGHT_SUM_SLACK = 1e-3       # :1625

_MAX_J = 32  # output rows per transform call (the transform kernel's limit is 34)


class ResidueRefused(ValueError):
    """A real frequency the imaginary-time representation does not carry
    (``real_screening.py:49-54``)."""


def gap_scaled_w0(eps, nocc, scale=0.5):
    """w0 = scale (eps_LUMO - eps_HOMO) (``Base/utils/grids/grids.py:173-186``)."""
    eps = np.asarray(eps, float)
    w0 = scale * (eps[nocc] - eps[nocc - 1])
    if not w0 > 0:
        raise ValueError(f'gap_scaled_w0: the gap {eps[nocc] - eps[nocc - 1]:.6g} is not positive')
    return w0


def cd_grid_range(eps, nocc, e_min_below_gap=None, pair_energies=None):
    """(e_min, e_max) of the contour's time grid: e_min reaches below the gap,
    by default by half of it (``contour_deformation.py:439-468``).
    pair_energies: the screening's particle-hole energies when they are not
    the ones (eps, nocc) spans (both spins of an unrestricted reference): the
    range and the default shift then follow them."""
    if pair_energies is not None:
        d = np.asarray(pair_energies, float)
        gap, e_max = float(d.min()), float(d.max())
        shift = 0.5 * gap if e_min_below_gap is None else float(e_min_below_gap)
    else:
        eps = np.asarray(eps, float)
        gap, e_max, _ = particle_hole_window(eps, nocc)
        shift = (gap_scaled_w0(eps, nocc) if e_min_below_gap is None
                 else float(e_min_below_gap))
    if gap - shift <= 0:
        raise ValueError(f'e_min_below_gap {shift} exceeds the gap {gap:.4f}: the imaginary-'
                         f'time grid would be asked to represent e^{{-y tau}} at y <= 0')
    return gap - shift, e_max


def cd_frequency_grid(eps, nocc, ntau=CD_NTAU, nfreq_cd=CD_NFREQ, w0_cd=None,
                      e_min_below_gap=None, pair_energies=None):
    """(nu, nu_weights, grid, w0): Gauss-Legendre nu on w0 (half the gap by
    default; half the smallest pair energy with pair_energies) and the
    minimax time grid over `cd_grid_range` onto it, cosine tau -> omega
    weights only (``contour_deformation.py:471-503``)."""
    e_min, e_max = cd_grid_range(eps, nocc, e_min_below_gap, pair_energies)
    if w0_cd is not None:
        w0 = float(w0_cd)
    elif pair_energies is not None:
        w0 = 0.5 * float(np.min(pair_energies))
    else:
        w0 = gap_scaled_w0(eps, nocc)
    nu, nu_weights = gauss_legendre_grid(int(nfreq_cd), w0=w0)
    grid = TimeFrequencyGrid.minimax_split(int(ntau), e_min, e_max, nu, nu_weights,
                                           with_sine=False, with_inverse=False)
    return nu, nu_weights, grid, w0


def cd_integral_weights(de, nu_points, nu_weights):
    """(c, dc), (nfreq, norb): Sigma^int = -(1/pi) sum c wc for de = omega -
    eps, and its derivative in de (``contour_deformation.py:150-202``). The
    Lorentzian de/(de^2 + nu^2) times wc is integrated as wc(0) times a
    closed-form integral of de/(de^2 + nu^2) a^2/(a^2 + nu^2) plus the
    quadrature of the remainder, wc(0) extrapolated in nu^2 from the two
    smallest nodes (a = four times the median node); at |de| below
    RESIDUE_ON_CONTOUR_TOL the closed form takes sign 0, as the residue term
    takes that pole at half weight."""
    de = np.asarray(de, float)
    nu = np.asarray(nu_points, float)
    wt = np.asarray(nu_weights, float)
    den = de[None, :] ** 2 + nu[:, None] ** 2
    g = de[None, :] / den
    dg = (nu[:, None] ** 2 - de[None, :] ** 2) / den ** 2
    c = wt[:, None] * g
    dc = wt[:, None] * dg
    k1, k2 = np.argsort(nu)[:2]
    n1, n2 = nu[k1] ** 2, nu[k2] ** 2
    a = 4.0 * float(np.median(nu))
    h = wt * a * a / (a * a + nu ** 2)
    side = np.where(np.abs(de) < RESIDUE_ON_CONTOUR_TOL, 0.0, np.sign(de))
    ad = a + np.abs(de)
    err = 0.5 * np.pi * side * a / ad - h @ g
    derr = -0.5 * np.pi * a / ad ** 2 - h @ dg
    for k, coef in ((k1, n2 / (n2 - n1)), (k2, -n1 / (n2 - n1))):
        c[k] += coef * err
        dc[k] += coef * derr
    return c, dc


def residue_set(eps, nocc, omega, tol=RESIDUE_ON_CONTOUR_TOL):
    """[(q, weight)]: the poles of G the deformation sweeps over
    (``real_screening.py:157-168``): occupied levels above omega (-1),
    virtual ones below it (+1), a level on the contour at half weight."""
    eps = np.asarray(eps, float)
    out = []
    for q in range(len(eps)):
        gap = eps[q] - omega
        if abs(gap) < tol:
            out.append((q, -0.5 if q < nocc else 0.5))
        elif q < nocc and gap > 0.0:
            out.append((q, -1.0))
        elif q >= nocc and gap < 0.0:
            out.append((q, 1.0))
    return out


def real_frequency_weights(grid, omega):
    """(c, dc): chi0(omega) = sum_k c_k proj(tau_k) at a real omega below the
    gap, c_k = 2 w_k cosh(omega tau_k) on the grid's bare Laplace quadrature,
    and its omega derivative (``real_screening.py:184-209``)."""
    t = np.asarray(grid.tau_points, float)
    w = 2.0 * np.asarray(grid.tau_weights, float)
    return w * np.cosh(omega * t), w * t * np.sinh(omega * t)


def laplace_representation_error(grid, eps, nocc, freq, pair_energies=None):
    """max over y = d -+ freq of |y sum_k w_k e^{-y tau_k} - 1| on the pair
    energies d (those of (eps, nocc), or pair_energies), inf where freq
    reaches the gap (``LinearResponse/space_time.py:908-931``)."""
    if pair_energies is None:
        d = ov_energies(eps, nocc)
    else:
        d = np.asarray(pair_energies, float)
    y = np.concatenate([d - freq, d + freq])
    if y.min() <= 0.0:
        return np.inf
    q = np.exp(-np.outer(y, grid.tau_points)) @ grid.tau_weights
    return float(np.abs(q * y - 1.0).max())


def _rows_transform(proj, weights):
    """sum_k weights[j, k] proj[k] for any number of output rows (in chunks
    of the transform kernel's limit)."""
    weights = np.asarray(weights, float)
    parts = [transform(proj, np.ascontiguousarray(weights[j:j + _MAX_J]))
             for j in range(0, weights.shape[0], _MAX_J)]
    return parts[0] if len(parts) == 1 else torch.cat(parts)


def polarizability_tau(X, D, eps, nocc, grid, mu=None):
    """proj(tau) on the grid's time points, (ntau, naux, naux) on the device,
    FP64 (``gradients/rpa/space_time_adjoint.py:94-113``)."""
    _, proj = chi0_sweep(X, D, eps, nocc, grid.tau_points,
                         np.zeros((1, len(grid.tau_points))), mu=mu, precision='fp64',
                         want_proj=True)
    return proj


def screening_minus_identity(proj_tau, cosft_wt, precision='fp64'):
    """W(i nu) - I for every frequency of cosft_wt: chi0 = cosft_wt proj(tau),
    then the Dyson step (FP64 Cholesky; ``contour_deformation.py:209-226``
    factorises and solves per frequency; 'mixed' forms the inverse from the
    FP64 factor by TF32x3 tensor-core products). Returns (W - I, info)."""
    dev = require_device()
    chi0 = _rows_transform(to_device(proj_tau, dev), cosft_wt)
    _, _, info, _ = dyson_batch(chi0, want_w=True, precision=precision)
    return chi0, info


def three_index_slices(X, D, states):
    """(nstates, naux, norb) device tensor of B_p = D^T diag(X[:, p]) X
    (``LinearResponse/space_time.py:804-815``)."""
    dev = require_device()
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    M, norb = Xd.shape
    naux = Dd.shape[1]
    st = np.ascontiguousarray(np.atleast_1d(states), dtype=np.int64)
    B = torch.empty((len(st), naux, norb), dtype=torch.float64, device=dev)
    ws = WORKSPACE.get(lib().mbpt_three_index_slices_workspace_bytes(M, norb), dev)
    import ctypes
    check(lib().mbpt_three_index_slices(ptr(Xd), M, norb, ptr(Dd), naux,
                                        st.ctypes.data_as(ctypes.c_void_p), len(st), ptr(B),
                                        ptr(ws), ws.numel(), stream_ptr()),
          'mbpt_three_index_slices')
    return B


def screening_contraction_device(w_minus_i, Bps, precision='fp64'):
    """[wc_s (nfreq, norb)] for each slice: wc[k, q] = B[:, q]^T (W - I)_k
    B[:, q], one product per frequency for all slices side by side; 'mixed'
    forms the products as split-BF16 tensor-core products (FP32 out)."""
    from .space_time import _Err, _mode
    dev = w_minus_i.device
    Bs = [to_device(b, dev) for b in Bps]
    naux, norb = Bs[0].shape
    B = torch.cat(Bs, dim=1).contiguous()
    nfreq, ncols = w_minus_i.shape[0], B.shape[1]
    mode = _mode(precision)
    wc = torch.empty((nfreq, ncols), dtype=torch.float64, device=dev)
    ws = WORKSPACE.get(lib().mbpt_screening_contraction_workspace_bytes(naux, ncols, mode), dev)
    wm = w_minus_i.contiguous()
    err = _Err(dev)
    check(lib().mbpt_screening_contraction(ptr(wm), nfreq, naux, ptr(B), ncols, mode, ptr(wc),
                                           ptr(ws), ws.numel(), ptr(err.t), stream_ptr()),
          'mbpt_screening_contraction')
    err.check('mbpt_screening_contraction')
    return [wc[:, i * norb:(i + 1) * norb] for i in range(len(Bs))]


def cd_screening_contraction_multi(proj_tau, cosft_wt, Bps, tile_gb=None, freq_indices=None,
                                   precision='fp64'):
    """wc[nu, q] for a list of bra slices on one factorisation per frequency
    (``contour_deformation.py:248-270``); arrays come back as Bps[0] is held.
    precision 'mixed': the Dyson inverses and the contraction's products on
    the tensor cores (the factorisations stay FP64)."""
    if freq_indices is not None:
        raise NotImplementedError('frequency splits over ranks are outside the one-GPU route')
    wmi, info = screening_minus_identity(proj_tau, cosft_wt, precision=precision)
    if np.any(info):
        import warnings
        warnings.warn('1 - chi0(i nu) is not positive definite at frequencies '
                      f'{np.nonzero(info)[0].tolist()}; solved by LU', RuntimeWarning)
    out = screening_contraction_device(wmi, Bps, precision=precision)
    if isinstance(Bps[0], torch.Tensor):
        return out
    return [w.cpu().numpy() for w in out]


def screening_contraction(Bp, wbp):
    """wc[k, q] = sum_P Bp[P, q] (W(i nu_k) Bp - Bp)[P, q] from W Bp given per
    frequency (``contour_deformation.py:229-237``)."""
    return np.einsum('Pq,kPq->kq', np.asarray(Bp), np.asarray(wbp) - np.asarray(Bp)[None],
                     optimize=True)


class _ResidueSolves:
    """W(freq) b for the residues of one backend: 1 - chi0(freq) factorised
    once per frequency by the Dyson step's FP64 Cholesky and kept for the
    latest `cap` frequencies (the value and the slope of one scan point
    apply W at the same frequencies), each b then solved against the factor
    by two triangular solves (mbpt_chol_solve) without forming W. Where
    1 - chi0 is not positive definite (the explicit response above the
    gap) W - I comes from the LU inverse instead."""

    def __init__(self, cap):
        self.cap = cap
        self._c = OrderedDict()

    def entry(self, key, build):
        ent = self._c.get(key)
        if ent is not None:
            self._c.move_to_end(key)
            return ent
        chi0 = build()
        _, _, info, _ = dyson_batch(chi0, want_w=False, precision='fp64')
        if info[0] == 0:
            ent = ('factor', chi0[0])
        else:
            chi0 = build()
            dyson_batch(chi0, want_w=True, precision='fp64')
            ent = ('w', chi0[0])
        self._c[key] = ent
        if len(self._c) > self.cap:
            self._c.popitem(last=False)
        return ent

    @staticmethod
    def solve(ent, bd):
        kind, m = ent
        if kind == 'w':
            return bd + m @ bd
        y = bd.clone().contiguous()
        check(lib().mbpt_chol_solve(ptr(m), m.shape[0], ptr(y), 1, stream_ptr()),
              'mbpt_chol_solve')
        return y


class LaplaceRealScreening:
    """W at a real frequency below the particle-hole gap from proj(tau): one
    (ntau, naux^2) transform and one Cholesky factorisation per frequency,
    the factor kept for later calls and W b solved against it
    (``real_screening.py:94-154``).
    Refuses (ResidueRefused) a frequency the grid does not carry.
    pair_energies: the particle-hole energies proj(tau) was summed over, when
    they are not the ones (eps, nocc) spans (both spins of an unrestricted
    reference)."""

    def __init__(self, proj_tau, grid, eps, nocc, tol=LAPLACE_SCREENING_TOL,
                 pair_energies=None, cache_bytes=4e9):
        self.proj_tau = to_device(proj_tau, require_device())
        self.grid = grid
        self.eps = np.asarray(eps, float)
        self.nocc = nocc
        self.tol = tol
        self.pair_energies = (None if pair_energies is None
                              else np.asarray(pair_energies, float))
        # the latest frequencies' W - I (the value and the slope of one point
        # apply W at the same frequencies), bounded by memory
        naux = self.proj_tau.shape[-1]
        self._cap = max(2, min(2 * len(self.eps), int(cache_bytes // (8 * naux * naux))))
        self._w = OrderedDict()
        self._solves = _ResidueSolves(self._cap)
        # the representability check on the device: 2 nocc nvirt x ntau
        # exponentials per new frequency
        dev = self.proj_tau.device
        d = (ov_energies(self.eps, nocc) if self.pair_energies is None
             else self.pair_energies)
        self._d = torch.as_tensor(d, dtype=torch.float64, device=dev)
        self._tau = torch.as_tensor(np.asarray(grid.tau_points, float), device=dev)
        self._tw = torch.as_tensor(np.asarray(grid.tau_weights, float), device=dev)

    def representation_error(self, freq):
        """max over y = d -+ freq of |y sum_k w_k e^{-y tau_k} - 1|, inf where
        freq reaches the gap (``LinearResponse/space_time.py:908-931``)."""
        y = torch.cat([self._d - freq, self._d + freq])
        if float(y.min()) <= 0.0:
            return np.inf
        q = torch.exp(-y[:, None] * self._tau[None, :]) @ self._tw
        return float((q * y - 1.0).abs().max())

    def _weights(self, freq):
        err = self.representation_error(freq)
        if not err < self.tol:
            gap = (particle_hole_window(self.eps, self.nocc)[0] if self.pair_energies is None
                   else float(self.pair_energies.min()))
            raise ResidueRefused(
                f'real frequency {freq:.4f} Ha is not carried by the tau grid: bare-quadrature '
                f'error {err:.1e} against tol {self.tol:.0e}; gap - freq = {gap - freq:.4f} '
                f'Ha, the grid\'s e_min is {self.grid.meta.get("e_min", float("nan")):.4f}. '
                f'Build the grid with e_min <= gap - freq, or use the explicit backend.')
        return real_frequency_weights(self.grid, freq)

    def w_minus_identity(self, freq):
        key = float(freq)
        w = self._w.get(key)
        if w is None:
            c, _ = self._weights(key)
            chi0 = _rows_transform(self.proj_tau, c[None, :])
            dyson_batch(chi0, want_w=True, precision='fp64')
            w = self._w[key] = chi0[0]
            if len(self._w) > self._cap:
                self._w.popitem(last=False)
        else:
            self._w.move_to_end(key)
        return w

    def apply(self, freq, b):
        """W(freq) b = [1 - chi0(freq)]^-1 b, by a solve against the
        frequency's kept Cholesky factor (``real_screening.py:147-150``)."""
        key = float(freq)
        ent = self._solves.entry(
            key, lambda: _rows_transform(self.proj_tau, self._weights(key)[0][None, :]))
        y = _ResidueSolves.solve(ent, to_device(b, self.proj_tau.device))
        return y if isinstance(b, torch.Tensor) else y.cpu().numpy()

    def slope(self, freq, y):
        """y^T [dchi0/dfreq] y, dchi0/dfreq = sum_k dc_k proj(tau_k)
        (``real_screening.py:152-154``)."""
        _, dc = self._weights(freq)
        dchi0 = _rows_transform(self.proj_tau, dc[None, :])[0]
        yd = to_device(y, self.proj_tau.device)
        return float(yd @ (dchi0 @ yd))


def ov_energies(eps, nocc):
    """d[(i, a)] = eps_a - eps_i on the pair index of C_ov, i major
    (``Base/orbital_spaces.py:31-34``)."""
    eps = np.asarray(eps, float)
    return (eps[nocc:][None, :] - eps[:nocc][:, None]).ravel()


def three_index_ov(X, D, eps, nocc, tile_gb=None):
    """C_ov[P, (i, a)] = sum_k D[k, P] X[k, i] X[k, a], (naux, nocc * nvirt)
    on the device (``LinearResponse/space_time.py:833-851``): the occupied
    states' three-index slices (mbpt_three_index_slices), a block of
    occupied states at a time, their virtual columns laid side by side.
    tile_gb bounds a block's slices (default 2 GB)."""
    dev = require_device()
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    norb, naux = Xd.shape[1], Dd.shape[1]
    nvirt = norb - nocc
    C = torch.empty((naux, nocc, nvirt), dtype=torch.float64, device=dev)
    per = 8 * naux * norb
    step = max(1, min(nocc, int((tile_gb or 2.0) * 1e9 // per)))
    for i0 in range(0, nocc, step):
        i1 = min(nocc, i0 + step)
        B = three_index_slices(Xd, Dd, np.arange(i0, i1))
        C[:, i0:i1, :] = B[:, :, nocc:].permute(1, 0, 2)
    return C.reshape(naux, nocc * nvirt)


def require_three_index(C_ov, what):
    """``contour_deformation.py:109-114``."""
    if C_ov is None:
        raise ResidueRefused(
            f'{what} needs C_ov = B[:, occ, virt] as (naux, nocc*nvirt) and it was not '
            f'supplied. A frontier state sweeps no residues and needs none once the '
            f'imaginary-axis screening comes in as wbp or wc.')


class ExplicitRealScreening:
    """W at a real frequency from the particle-hole block C_ov, explicitly
    (``real_screening.py:57-91``, continuation 'cd'): chi0 = 2 (C_ov f) C_ov^T
    by mbpt_chi0_aux (a symmetric rank-k product over column chunks) and
    W - I by the Dyson step (Cholesky below the gap, LU above it, where
    1 - chi0 is indefinite), the W - I of the latest frequencies kept for
    later calls. eta broadens the particle-hole poles (off by default).
    pair_energies: the pair index of C_ov when it is not the one (eps, nocc)
    spans. O(naux^2 nocc nvirt) per frequency, the route the cubic one is
    checked against and the only one above the particle-hole gap. precision
    'fp64' (default) or 'mixed' (the response as one split BF16x3
    tensor-core product; the Dyson step stays FP64)."""

    def __init__(self, C_ov, eps, nocc, eta=0.0, pair_energies=None, cache_bytes=4e9,
                 precision='fp64'):
        self.C_ov = to_device(C_ov, require_device())
        self.precision = precision
        self.eps = np.asarray(eps, float)
        self.nocc = nocc
        self.eta = float(eta)
        self.d = (ov_energies(self.eps, nocc) if pair_energies is None
                  else np.asarray(pair_energies, float))
        if self.d.size != self.C_ov.shape[1]:
            raise ValueError(f'C_ov has {self.C_ov.shape[1]} pairs, the pair energies '
                             f'{self.d.size}')
        naux = self.C_ov.shape[0]
        self._cap = max(2, min(2 * len(self.eps), int(cache_bytes // (8 * naux * naux))))
        self._w = OrderedDict()
        self._solves = _ResidueSolves(self._cap)

    def w_minus_identity(self, freq, imaginary=False):
        key = (float(freq), bool(imaginary))
        w = self._w.get(key)
        if w is None:
            chi0 = self._chi0(freq, imaginary)
            dyson_batch(chi0, want_w=True, precision='fp64')
            w = self._w[key] = chi0[0]
            if len(self._w) > self._cap:
                self._w.popitem(last=False)
        else:
            self._w.move_to_end(key)
        return w

    def _chi0(self, freq, imaginary=False):
        f = frequency_factor(self.d, float(freq), imaginary, self.eta)
        return chi0_aux([(self.C_ov, f)], 2.0, precision=self.precision)[None]

    def apply(self, freq, b):
        """W(freq) b = [1 - chi0(freq)]^-1 b, by a solve against the
        frequency's kept Cholesky factor (the LU inverse above the gap)."""
        key = float(freq)
        ent = self._solves.entry(key, lambda: self._chi0(key))
        y = _ResidueSolves.solve(ent, to_device(b, self.C_ov.device))
        return y if isinstance(b, torch.Tensor) else y.cpu().numpy()

    def slope(self, freq, y):
        """y^T [dchi0/dfreq] y = 2 sum_(ia) df/dw (C_ov^T y)_(ia)^2
        (``real_screening.py:87-91``)."""
        z = (self.C_ov.T @ to_device(y, self.C_ov.device)).cpu().numpy()
        return 2.0 * float(frequency_factor(self.d, float(freq), False, self.eta,
                                            slopes=True)[2] @ z ** 2)


def residue_backend(real_screening, C_ov, eps, nocc, eta):
    """The backend the residue term uses: the one given, else the explicit one
    from C_ov (``contour_deformation.py:117-122``)."""
    if real_screening is not None:
        return real_screening
    require_three_index(C_ov, 'the residue term')
    return ExplicitRealScreening(C_ov, eps, nocc, eta)


def wc_explicit(Bp, C_ov, d, nu_points, block=8):
    """wc[k, q] = Bp[:, q]^T (W(i nu_k) - I) Bp[:, q] from the explicit
    imaginary-axis screening (``contour_deformation.py:240-245``): per block
    of frequencies the explicit chi0 (mbpt_chi0_aux), the Dyson step and the
    screening contraction. (nfreq, norb) on the host."""
    dev = require_device()
    Cd = to_device(C_ov, dev)
    Bd = to_device(Bp, dev)
    naux = Cd.shape[0]
    nu = np.asarray(nu_points, float)
    out = []
    for k0 in range(0, len(nu), block):
        ks = nu[k0:k0 + block]
        stack = torch.empty((len(ks), naux, naux), dtype=torch.float64, device=dev)
        for m, v in enumerate(ks):
            chi0_aux([(Cd, frequency_factor(d, float(v), True))], 2.0, out=stack[m])
        dyson_batch(stack, want_w=True, precision='fp64')
        out.append(screening_contraction_device(stack, [Bd])[0].cpu().numpy())
    return np.concatenate(out)


def sigma_cd(p, omega, Bp, eps, nocc, nu_points, nu_weights, residues=None, wbp=None,
             eta=0.0, wc=None, C_ov=None, real_screening=None):
    """Sigma^c_pp(omega) by contour deformation from the state's slice Bp and
    its contracted screening wc (``contour_deformation.py:310-343``):
    the imaginary-axis integral and, for the residue set (recomputed at omega
    when not given), sum_q w_q (b_q^T W(|eps_q - omega|) b_q - b_q^T b_q) with
    `real_screening`'s W (a LaplaceRealScreening or ExplicitRealScreening;
    with C_ov and no backend the explicit one). With neither wc nor wbp the
    imaginary-axis screening is built explicitly from C_ov (`wc_explicit`)."""
    eps = np.asarray(eps, float)
    Bh = Bp.detach().cpu().numpy() if isinstance(Bp, torch.Tensor) else np.asarray(Bp)
    if wc is None:
        if wbp is None:
            require_three_index(C_ov, 'the imaginary-axis screening without wbp or wc')
            wc = wc_explicit(Bp, C_ov, ov_energies(eps, nocc), nu_points)
        else:
            wc = screening_contraction(Bh, wbp)
    wc = wc.detach().cpu().numpy() if isinstance(wc, torch.Tensor) else np.asarray(wc)
    c, _ = cd_integral_weights(omega - eps, nu_points, nu_weights)
    s_int = -float(np.einsum('kq,kq->', c, wc)) / np.pi
    res = residue_set(eps, nocc, omega) if residues is None else residues
    s_res = 0.0
    if res:
        rs = residue_backend(real_screening, C_ov, eps, nocc, eta)
        for q, weight in res:
            b = Bh[:, q]
            y = rs.apply(abs(eps[q] - omega), b)
            s_res += weight * (float(b @ y) - float(b @ b))
    return s_int + s_res


def sigma_cd_slope(p, omega, Bp, eps, nocc, nu_points, nu_weights, residues, wc, eta=0.0,
                   C_ov=None, real_screening=None):
    """dSigma^c_pp/domega in closed form at a frozen residue set
    (``contour_deformation.py:346-373``): the integral weights' derivative
    against wc, and per residue W [dchi0/dfreq] W contracted with b_q on both
    sides, signed by the side of the pole."""
    eps = np.asarray(eps, float)
    Bh = Bp.detach().cpu().numpy() if isinstance(Bp, torch.Tensor) else np.asarray(Bp)
    wc = wc.detach().cpu().numpy() if isinstance(wc, torch.Tensor) else np.asarray(wc)
    _, dc = cd_integral_weights(omega - eps, nu_points, nu_weights)
    slope = -float(np.einsum('kq,kq->', dc, wc)) / np.pi
    if residues:
        rs = residue_backend(real_screening, C_ov, eps, nocc, eta)
        for q, weight in residues:
            gap = eps[q] - omega
            freq = abs(gap)
            y = rs.apply(freq, Bh[:, q])
            slope -= weight * rs.slope(freq, y) * np.sign(gap)
    return slope


# ------------------------------------------------ the scan root finder
# Solvers/qp_equation.py: `solve_qp_equation_scan` (:1396-1420) on a
# `SampledEquation` (:1029-1278) through `find_qp_root` (:155-233) without a
# followed root, as `qp_energy_cd` calls it.

def _qp_search_windows(a):
    """Windows about the bare level, narrowest first: the tier of the
    state's depth, then every wider tier (:1280-1288)."""
    tier = 0
    for k, (depth, _) in enumerate(QP_SEARCH_WINDOW_TIERS):
        if abs(a) > depth:
            tier = k
    return [(a - half, a + half) for _, half in QP_SEARCH_WINDOW_TIERS[tier:]]


def _valid_weight(z, z_min=0.0):
    """Z of a quasiparticle: finite and in (z_min, 1] (:95-102)."""
    z = float(z)
    return bool(np.isfinite(z) and z_min < z <= 1.0)


def _bracketed_newton(fval, l, r, sl, tol, max_iter):
    """The root of f in (l, r), f of sign sl at l, by Newton on the slope
    safeguarded by the bracket: a step leaving it, or not under half the step
    before the last, is a bisection; a step below tol that stays in the
    closed bracket ends it (:376-426, for a costly f)."""
    if sl == 0.0:
        return float(l)
    w = 0.5 * (l + r)
    step = old = r - l
    for _ in range(int(max_iter)):
        f, fp = fval(w)
        if f == 0.0:
            return float(w)
        if np.sign(f) == sl:
            l = w
        else:
            r = w
        dw = -f / fp
        if abs(dw) < tol and l <= w + dw <= r:
            return float(w + dw)
        mid = 0.5 * (l + r)
        if not l < mid < r:
            break
        newton = np.isfinite(dw) and l < w + dw < r and abs(dw) <= 0.5 * abs(old)
        old, step = step, (dw if newton else mid - w)
        w = w + dw if newton else mid
    return float(w)


class _Scan:
    """f(w) = w - a - Sigma(w) known pointwise with a closed-form slope, for
    a positive-weight Sigma; points a refusal type rejects are NaN, the first
    refusal kept (:1071-1092, :1143-1166, :1250-1278)."""

    def __init__(self, func, fprime, tol, max_iter, refusals):
        self.tol, self.max_iter = tol, max_iter
        self.refusals, self.refused = tuple(refusals), None
        self.func, self.fprime = self._guarded(func), self._guarded(fprime)

    def _guarded(self, g):
        def call(w):
            try:
                return g(w)
            except self.refusals as refusal:
                if self.refused is None:
                    self.refused = refusal
                return np.nan
        return call

    def weight(self, w):
        fp = float(self.fprime(w))
        return 1.0 / fp if fp != 0.0 else np.nan

    def solve(self, bracket):
        """[(root, Z)] of a bracket (l, r, f(l), f(r)); empty for a pole."""
        l, r, fl, fr = bracket
        if l == r:
            return [(float(l), self.weight(l))]
        if fl > 0.0 > fr:
            return []                   # f falls: a pole of a positive-weight Sigma
        fval = lambda x: (float(self.func(x)), float(self.fprime(x)))  # noqa: E731
        w = _bracketed_newton(fval, l, r, np.sign(fl), self.tol, self.max_iter)
        fw = fval(w)[0]
        if not abs(fw) <= max(abs(fl), abs(fr)):
            return []                   # |f| grew (a pole) or the point was refused
        return [(float(w), self.weight(w))]

    def cells(self, l, r, fl, fr, depth):
        """Brackets in [l, r]: the cell on a sign change; its halves while
        its secant slope is below QP_SCAN_SECANT_MIN or one end is refused
        and the other not, at most `depth` times (:1250-1266)."""
        if fl * fr < 0.0:
            return [(l, r, fl, fr)]
        edge = np.isnan(fl) != np.isnan(fr)
        if depth == 0 or fl == 0.0 or fr == 0.0 or not (
                edge or fr - fl < QP_SCAN_SECANT_MIN * (r - l)):
            return []
        m = 0.5 * (l + r)
        fm = float(self.func(m))
        return self.cells(l, m, fl, fm, depth - 1) + self.cells(m, r, fm, fr, depth - 1)

    def outward(self, lo, hi, a):
        """The brackets of each grid cell, cells in increasing distance from
        the one holding a, f evaluated as the cells reach a grid point
        (:1110-1129)."""
        grid = np.linspace(lo, hi, QP_GRAPHICAL_N_OMEGA)
        f = {}

        def value(j):
            if j not in f:
                f[j] = float(self.func(grid[j]))
            return f[j]
        c0 = min(max(int(np.searchsorted(grid, a)) - 1, 0), grid.size - 2)
        for d in range(grid.size - 1):
            for c in sorted({c0 - d, c0 + d}):
                if 0 <= c < grid.size - 1:
                    yield self.cells(grid[c], grid[c + 1], value(c), value(c + 1),
                                     QP_SCAN_SPLIT_DEPTH)


def _weighed_outward(scan, lo, hi, a, enough):
    """[(root, Z)] of the cells walked outward from a, until the valid
    weights found leave (plus QP_WEIGHT_SUM_SLACK) no more of their sum, one,
    than the largest of them or `enough` (:312-339)."""
    found, best, weighed = [], -np.inf, 0.0
    for brackets in scan.outward(lo, hi, a):
        for bracket in brackets:
            got = scan.solve(bracket)
            found.append((bracket[0], got))
            for _, z in got:
                if _valid_weight(z):
                    weighed += z
                    best = max(best, z)
        if 1.0 - weighed + QP_WEIGHT_SUM_SLACK <= max(best, enough):
            break
    found.sort(key=lambda lr: lr[0])
    return [rz for _, got in found for rz in got]


def solve_qp_equation_scan(residual, fprime, a, tol=QP_ROOT_TOL, max_iter=QP_ROOT_MAX_ITER,
                           label='', refusals=()):
    """(w, Z) of residual(w) = 0 for a positive-weight self-energy: per
    window, narrowest first, the root of largest valid weight; a weight above
    QP_WINDOW_Z_MIN ends the search, the widest window keeps its largest
    valid weight (the root nearest a if none is valid). No quasiparticle
    where Sigma could be evaluated raises the first refusal; no root at all
    is (NaN, NaN) with a QPNoRoot warning; a root with Z outside (0, 1] is
    kept with a QPWeightOutside warning (:155-273, :1396-1420)."""
    from .gw import QPNoRoot, QPWeightOutside
    scan = _Scan(residual, fprime, tol, max_iter, refusals)
    windows = _qp_search_windows(a)
    found, w, z, quasi = [], np.nan, np.nan, False
    for i, (lo, hi) in enumerate(windows):
        enough = QP_WINDOW_Z_MIN if i + 1 < len(windows) else -np.inf
        found = _weighed_outward(scan, lo, hi, a, enough)
        ok = [k for k, (_, zk) in enumerate(found) if _valid_weight(zk)]
        if ok:
            k = max(ok, key=lambda j: found[j][1])
            if _valid_weight(found[k][1], QP_WINDOW_Z_MIN):
                w, z, quasi = found[k][0], found[k][1], True
                break
    if not quasi:
        if scan.refused is not None:
            raise scan.refused
        if not found:
            warnings.warn(f'{label or "the quasiparticle equation"} has no root in the widest '
                          f'scan window [{windows[-1][0]:.6f}, {windows[-1][1]:.6f}] Ha about '
                          f'{a:.6f} Ha.', QPNoRoot, stacklevel=2)
            return np.nan, np.nan
        ok = [k for k, (_, zk) in enumerate(found) if _valid_weight(zk)]
        k = (max(ok, key=lambda j: found[j][1]) if ok
             else min(range(len(found)), key=lambda j: abs(found[j][0] - a)))
        w, z = found[k]
    if np.isfinite(w) and not 0.0 < z <= 1.0:
        warnings.warn(f'the quasiparticle root of {label or "the quasiparticle equation"} '
                      f'{w!r} Ha has Z = {z!r}, outside (0, 1]: kept', QPWeightOutside,
                      stacklevel=2)
    return float(w), float(z)


def qp_energy_cd(p, Bp, eps, nocc, nu_points, nu_weights, xc_correction=0.0, tol=QP_ROOT_TOL,
                 max_iter=QP_ROOT_MAX_ITER, follow=None, wbp=None, wc=None, C_ov=None,
                 eta=0.0, real_screening=None, branch=None, rescan=True):
    """(eps^QP_p, Z_p, residues) of w = eps_p + xc_correction + Sigma^c(w) by
    contour deformation (``contour_deformation.py:376-436``): the scan about
    the bare level with Newton on the closed-form slope, the residue set
    re-decided at every point and frozen at the root. The imaginary-axis
    screening comes in as wc, as wbp contracted once here, or -- with neither
    -- explicitly from C_ov (`wc_explicit`, contracted once). The residues
    read `real_screening`, else the explicit backend of C_ov (broadened by
    eta), built once for the whole scan: its kept W - I serves the value and
    the slope at one point, as the reference's `_PointApplies` does."""
    if follow is not None or branch is not None:
        raise NotImplementedError('following a root along a walk is outside the device route')
    eps = np.asarray(eps, float)
    Bh = Bp.detach().cpu().numpy() if isinstance(Bp, torch.Tensor) else np.asarray(Bp)
    if wc is None:
        if wbp is not None:
            wc = screening_contraction(Bh, wbp)
        else:
            require_three_index(C_ov, 'the imaginary-axis screening without wbp or wc')
            wc = wc_explicit(Bp, C_ov, ov_energies(eps, nocc), nu_points)
    wc = wc.detach().cpu().numpy() if isinstance(wc, torch.Tensor) else np.asarray(wc)
    if real_screening is not None or C_ov is not None:
        real_screening = residue_backend(real_screening, C_ov, eps, nocc, eta)
    common = dict(eta=eta, C_ov=C_ov, real_screening=real_screening)

    def residual(w):
        return w - eps[p] - xc_correction - sigma_cd(
            p, w, Bh, eps, nocc, nu_points, nu_weights, residues=residue_set(eps, nocc, w),
            wc=wc, **common)

    def fprime(w):
        return 1.0 - sigma_cd_slope(p, w, Bh, eps, nocc, nu_points, nu_weights,
                                    residue_set(eps, nocc, w), wc, **common)
    w, z = solve_qp_equation_scan(residual, fprime, float(eps[p] + xc_correction), tol=tol,
                                  max_iter=max_iter, label=f'orbital {p}',
                                  refusals=(ResidueRefused,))
    return w, z, residue_set(eps, nocc, w)


HARTREE_TO_EV = 27.211386245988  # MBPTcode constants.py:11 (CODATA 2018)


def _roots_on_contour(continuation, states, B, wcs, eps, nocc, nu, nu_w, xc_correction,
                      backend, w0, ntau, nfreq_cd):
    """Each state's root and Z by `qp_energy_cd` on one contour grid, with
    the per-state records (``contour_deformation.py:558-598``)."""
    explicit = continuation == 'cd'
    roots, zs, records = np.zeros(len(states)), np.zeros(len(states)), []
    for i, p in enumerate(states):
        xc = (float(np.asarray(xc_correction).ravel()[i]) if np.ndim(xc_correction)
              else float(xc_correction))
        try:
            w, z, res = qp_energy_cd(int(p), B[i], eps, nocc, nu, nu_w, xc_correction=xc,
                                     wc=wcs[i], real_screening=backend)
        except ResidueRefused as refusal:
            if explicit:
                raise
            raise ResidueRefused(
                f"continuation='laplace' cannot serve orbital {int(p)}: its contour sweeps "
                f'a residue the imaginary-time grid does not represent. {refusal}') from refusal
        roots[i], zs[i] = w, z
        error = None
        if not explicit and res:
            error = max(backend.representation_error(abs(eps[q] - w)) for q, _ in res)
        records.append({'state': int(p), 'residues': len(res),
                        'representation_error': error})
    info = {'continuation': continuation, 'ntau': int(ntau), 'nfreq_cd': int(nfreq_cd),
            'w0_cd': float(w0), 'residue_route_taken': 'explicit' if explicit else 'laplace',
            'states': records}
    return roots, zs, info


def contour_roots(X, D, eps, nocc, states, ntau=CD_NTAU, nfreq_cd=CD_NFREQ, w0_cd=None,
                  e_min_below_gap=None, xc_correction=0.0, mu=None, continuation='laplace',
                  precision='fp64'):
    """(roots in Hartree, Z, per-state records) of the states on one contour
    grid (``contour_deformation.py:558-598, 767-812``): one proj(tau) and one
    W per frequency serve every state's imaginary-axis term, each state's
    root by `qp_energy_cd`. The residues read W at real frequencies from the
    cosh transform of the same proj(tau) (continuation 'laplace', which
    refuses a state whose residues the time grid does not carry) or from the
    explicit particle-hole response of C_ov (continuation 'cd', any state).
    xc_correction: the static term, one per state or one for all. precision
    'mixed' runs the screening contraction and the explicit response as
    split tensor-core products (the Dyson steps and the Laplace residues stay
    FP64)."""
    if continuation not in ('laplace', 'cd'):
        raise ValueError(f"continuation={continuation!r}: choose 'cd' or 'laplace'")
    eps = _eps_host(eps)
    states = np.atleast_1d(np.asarray(states, int))
    explicit = (ExplicitRealScreening(three_index_ov(X, D, eps, nocc), eps, nocc,
                                      precision=precision)
                if continuation == 'cd' else None)
    nu, nu_w, grid, w0 = cd_frequency_grid(eps, nocc, ntau=ntau, nfreq_cd=nfreq_cd,
                                           w0_cd=w0_cd, e_min_below_gap=e_min_below_gap)
    proj = polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    B = three_index_slices(X, D, states)
    wcs = cd_screening_contraction_multi(proj, grid.cosft_wt, list(B), precision=precision)
    backend = LaplaceRealScreening(proj, grid, eps, nocc) if explicit is None else explicit
    del proj
    return _roots_on_contour(continuation, states, B, wcs, eps, nocc, nu, nu_w, xc_correction,
                             backend, w0, ntau, nfreq_cd)


def contour_roots_unrestricted(X_mos, D, spectra, noccs, spin, states, ntau=CD_NTAU,
                               nfreq_cd=CD_NFREQ, w0_cd=None, e_min_below_gap=None,
                               xc_correction=0.0, continuation='laplace', precision='fp64'):
    """`contour_roots` for one spin channel of an unrestricted reference
    (``contour_deformation.py:686-812``): both spins' pair energies side by
    side set the contour grid, proj(tau) is the spin sum (half of each spin's
    restricted sweep at its own mid-gap), the channel's slices and contraction
    read it, and the residues come from its cosh transform on those pair
    energies ('laplace') or from both spins' C_ov side by side at 1/sqrt(2),
    so that the restricted factor 2 counts every pair once ('cd'). spin: 0
    (alpha) or 1 (beta); states are the channel's orbitals."""
    if continuation not in ('laplace', 'cd'):
        raise ValueError(f"continuation={continuation!r}: choose 'cd' or 'laplace'")
    if len(X_mos) != 2 or len(spectra) != 2 or len(noccs) != 2 or spin not in (0, 1):
        raise ValueError('an unrestricted contour takes two spin channels and spin 0 or 1')
    from .space_time import spin_summed
    spectra = [_eps_host(e) for e in spectra]
    noccs = [int(n) for n in noccs]
    pairs = np.concatenate([ov_energies(e, n) for e, n in zip(spectra, noccs)])
    eps, nocc = spectra[spin], noccs[spin]
    states = np.atleast_1d(np.asarray(states, int))
    explicit = None
    if continuation == 'cd':
        C = torch.cat([three_index_ov(X, D, e, n) for X, e, n in zip(X_mos, spectra, noccs)],
                      dim=1)
        C.mul_(1.0 / np.sqrt(2.0))
        explicit = ExplicitRealScreening(C, eps, nocc, pair_energies=pairs, precision=precision)
    nu, nu_w, grid, w0 = cd_frequency_grid(eps, nocc, ntau=ntau, nfreq_cd=nfreq_cd,
                                           w0_cd=w0_cd, e_min_below_gap=e_min_below_gap,
                                           pair_energies=pairs)
    proj = spin_summed(polarizability_tau, X_mos, D, spectra, noccs, grid)
    B = three_index_slices(X_mos[spin], D, states)
    wcs = cd_screening_contraction_multi(proj, grid.cosft_wt, list(B), precision=precision)
    backend = (LaplaceRealScreening(proj, grid, eps, nocc, pair_energies=pairs)
               if explicit is None else explicit)
    del proj
    return _roots_on_contour(continuation, states, B, wcs, eps, nocc, nu, nu_w, xc_correction,
                             backend, w0, ntau, nfreq_cd)


def solve_qp_energy_contour(mf, mol, nocc, states, continuation='cd', numerics=None,
                            w0_cd=None, auxbasis=None, radii=None, counts=None, factors=None,
                            grid_accuracy=None, sigma_x='mf', dm_correction=None,
                            eps_anchor=None, spin_channel='alpha', xc_diagonal=None,
                            precision='fp64'):
    """Drop-in for ``GW/contour_deformation.py:601-820`` on a gas-phase
    reference with pre-built factors: (quasiparticle energies in eV, pole
    strengths, diagnostics). The mean field gives eps (mo_energy); the
    static term <Sigma_x - v_xc> is `xc_diagonal` (zero on a Hartree-Fock
    reference); numerics.quadrature: ntau_cd and nfreq_cd where it has them.
    An unrestricted mean field (mo_energy (2, nmo), nocc (nalpha, nbeta),
    mo_coeff per spin) solves `spin_channel` by `contour_roots_unrestricted`
    from the factors' AO collocation, (X_mo, D, X_ao[, coords]).
    'cd' (the default, as in the reference) reads the residues' W from the
    explicit particle-hole response of C_ov, O(N^4) per residue frequency and
    exact for any state; 'laplace' solves the same contour from the cubic
    cosh transform wherever the time grid carries the residue frequencies,
    and refuses a state by name otherwise, as the reference does. 'sop' (the
    pole model) is outside the device route and refused. precision: as
    `contour_roots`."""
    if continuation not in ('cd', 'laplace'):
        raise NotImplementedError(f"continuation={continuation!r}: the device route runs "
                                  "'cd' (explicit residues) and 'laplace' (cubic residues)")
    if factors is None:
        raise NotImplementedError('building the ISDF factors needs pyscf (integrals and the '
                                  'fit); pass factors=(X_mo, D)')
    eps = np.asarray(getattr(mf, 'mo_energy', mf), float)
    ntau, nfreq = CD_NTAU, CD_NFREQ
    if numerics is not None:
        q = numerics.quadrature
        ntau = getattr(q, 'ntau_cd', ntau)
        nfreq = getattr(q, 'nfreq_cd', nfreq)
    states = np.atleast_1d(np.asarray(states, int))
    xc = 0.0 if xc_diagonal is None else np.asarray(xc_diagonal, float)
    X, D = (factors['X_mo'], factors['D']) if isinstance(factors, dict) else factors[:2]
    if eps.ndim == 2:
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
        if eps_anchor is not None:
            anchor = np.asarray(eps_anchor, float)
            if anchor.shape != eps.shape:
                raise ValueError(f'an unrestricted eps_anchor is one spectrum per spin, shape '
                                 f'{eps.shape}; got {anchor.shape}')
            xc = xc + (anchor[spin][states] - eps[spin][states])
        roots, zs, info = contour_roots_unrestricted(
            X_mos, D, list(eps), tuple(int(n) for n in nocc), spin, states, ntau=ntau,
            nfreq_cd=nfreq, w0_cd=w0_cd, xc_correction=xc, continuation=continuation,
            precision=precision)
        return roots * HARTREE_TO_EV, zs, info
    if eps_anchor is not None:
        xc = xc + (np.asarray(eps_anchor, float)[states] - eps[states])
    roots, zs, info = contour_roots(X, D, eps, nocc, states, ntau=ntau, nfreq_cd=nfreq,
                                    w0_cd=w0_cd, xc_correction=xc, continuation=continuation,
                                    precision=precision)
    return roots * HARTREE_TO_EV, zs, info


def _slice_backward(X, D, p, B_bar, X_bar, D_bar):
    Xd, Dd = to_device(X, B_bar.device), to_device(D, B_bar.device)
    M, norb = Xd.shape
    naux = Dd.shape[1]
    ws = WORKSPACE.get(lib().mbpt_three_index_slice_backward_workspace_bytes(M, norb, naux),
                       B_bar.device)
    Bb = B_bar.contiguous()
    check(lib().mbpt_three_index_slice_backward(ptr(Xd), M, norb, ptr(Dd), naux, int(p), ptr(Bb),
                                                ptr(X_bar), ptr(D_bar), ptr(ws), ws.numel(),
                                                stream_ptr()),
          'mbpt_three_index_slice_backward')


def qp_gradient_space_time(X, D, eps, nocc, grid, nu_points, nu_weights, p, *,
                           residue_route='laplace', mu=None, xc_correction=0.0, w0=None,
                           tol=QP_ROOT_TOL, laplace_tol=LAPLACE_SCREENING_TOL, want_grad=True,
                           tile_gb=None, follow=None, route_out=None, n_poles=None,
                           sop_stride=None, scissor=None, sop_poles=None, comm=None, z0=None):
    """(eps^QP_p, Z, eps_bar, X_bar, D_bar), or (eps^QP_p, Z) with want_grad
    False: the contour-deformation QP energy of state p and its gradient in
    (eps, X, D) (``gradients/gwbse/qp_space_time.py:412-452``), residues by
    the cosh transform of proj(tau) on `grid` (the contour's time grid, mu
    frozen). The root is differentiated implicitly, d eps^QP = Z [d eps_p +
    dSigma^c(w)|_w], the residue set frozen at the root: the integral term's
    adjoint goes to the slice, to W(i nu) (then W W_bar W onto chi0 and
    proj(tau)) and to eps through its weights; each residue's to the slice,
    to chi0 at its real frequency (folded onto proj(tau) by the cosh weights)
    and to eps through its frequency; then the chi0 sweep's and the slice's
    reverses. FP64 on the device; arrays come back as X is held."""
    if residue_route != 'laplace':
        raise NotImplementedError(f'residue_route={residue_route!r}: the device route serves '
                                  "'laplace' (the cubic residues)")
    if any(v is not None for v in (follow, scissor, sop_poles, comm, z0, w0)):
        raise NotImplementedError('walks, scissors, pole models and rank splits are outside '
                                  'the device route')
    dev = require_device()
    eps_h = _eps_host(eps)
    p = int(p)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    proj = polarizability_tau(X, D, eps_h, nocc, grid, mu=mu)
    wmi, _ = screening_minus_identity(proj, grid.cosft_wt)
    B = three_index_slices(X, D, [p])[0]
    wc = screening_contraction_device(wmi, [B])[0]
    lap = LaplaceRealScreening(proj, grid, eps_h, nocc, tol=laplace_tol)
    w, z, res = qp_energy_cd(p, B, eps_h, nocc, nu_points, nu_weights,
                             xc_correction=xc_correction, tol=tol, wc=wc, real_screening=lap)
    if route_out is not None:
        route_out.update(residue_route='laplace', residues=res)
    if not want_grad:
        return w, z
    naux, norb = B.shape
    eps_bar = np.zeros(norb)
    eps_bar[p] += z
    c, dc = cd_integral_weights(w - eps_h, nu_points, nu_weights)
    coeff = -z / np.pi
    wc_h = wc.cpu().numpy()
    eps_bar += -coeff * np.einsum('kq,kq->q', wc_h, dc)
    wc_bar = torch.as_tensor(coeff * c, dtype=torch.float64, device=dev)
    B_bar = torch.zeros_like(B)
    W_bar = torch.empty_like(wmi)
    ws = WORKSPACE.get(lib().mbpt_cd_integral_backward_workspace_bytes(naux, norb), dev)
    Bc = B.contiguous()
    check(lib().mbpt_cd_integral_backward(ptr(wmi), wmi.shape[0], naux, ptr(Bc), norb,
                                          ptr(wc_bar), ptr(B_bar), ptr(W_bar), ptr(ws),
                                          ws.numel(), stream_ptr()),
          'mbpt_cd_integral_backward')
    wsd = WORKSPACE.get(lib().mbpt_dyson_backward_workspace_bytes(naux), dev)
    check(lib().mbpt_dyson_backward(ptr(wmi), ptr(W_bar), naux, wmi.shape[0], ptr(wsd),
                                    wsd.numel(), stream_ptr()), 'mbpt_dyson_backward')
    cw_t = np.ascontiguousarray(np.asarray(grid.cosft_wt, float).T)   # (ntau, nfreq)
    proj_bar = torch.zeros_like(proj)
    for k0 in range(0, cw_t.shape[1], _MAX_J):
        transform(W_bar[k0:k0 + _MAX_J].contiguous(), np.ascontiguousarray(cw_t[:, k0:k0 + _MAX_J]),
                  out=proj_bar, accumulate=True)
    del W_bar
    tau = np.asarray(grid.tau_points, float)
    for q, wt in res:
        f = abs(eps_h[q] - w)
        cf, _ = real_frequency_weights(grid, f)
        b = B[:, q]
        y = lap.apply(f, b)
        B_bar[:, q] += (z * wt * 2.0) * (y - b)
        proj_bar += torch.as_tensor(z * wt * cf, device=dev)[:, None, None] * torch.outer(y, y)[None]
        eps_bar[q] += z * wt * lap.slope(f, y) * np.sign(eps_h[q] - w)
    del tau
    from .adjoint import chi0_backward
    e2, X_bar, D_bar = chi0_backward(proj_bar, X, D, eps_h, nocc, grid.tau_points, mu)
    _slice_backward(X, D, p, B_bar, X_bar, D_bar)
    eps_bar = eps_bar + e2.cpu().numpy()
    if isinstance(X, torch.Tensor):
        return w, z, torch.as_tensor(eps_bar, device=dev), X_bar, D_bar
    return w, z, eps_bar, X_bar.cpu().numpy(), D_bar.cpu().numpy()
