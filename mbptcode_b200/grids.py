"""Imaginary-time / imaginary-frequency axes of the space-time route (host side, FP64).

Everything here is tiny (at most 34 points per axis) and runs once per solve on
the host in FP64; the transform matrices it returns feed the device transforms.
The algorithms follow MBPTcode's grid layer so that a solve built on these
axes uses the same points and weights as the reference route:

* table lookup and narrow-range stretch: ``src/Base/utils/grids/grids.py:78-158``
  (``_table_row``, ``minimax_frequency_grid``, ``minimax_time_grid``);
* modified Gauss-Legendre axis: ``grids.py:161-170``;
* Kaltak-Klimes-Kresse test integral and point-count choice:
  ``src/Base/utils/grids/time_frequency.py:151-215`` and ``:249-272``;
* per-output-row least-squares transform fit (GreenX
  ``get_transformation_weights``): ``time_frequency.py:257-380``;
* self-energy fit ranges: ``time_frequency.py:387-427``;
* the split grid (tau axis at half the Laplace scaling):
  ``time_frequency.py:498-555``;
* the GW route's three axes: ``src/SingleReference/GW/space_time.py:559-618``,
  ``src/SingleReference/GW/imaginary_time.py:95-138``.

The coefficient tables are the GreenX ones (Apache-2.0, see data/NOTICE).
"""
from __future__ import annotations

import contextlib
import json
import os
import threading
import warnings
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

try:
    from threadpoolctl import ThreadpoolController
except ImportError:  # pragma: no cover -- the fits then run on the BLAS's own threads
    ThreadpoolController = None

_DATA = os.path.join(os.path.dirname(__file__), 'data')
_TABLES: dict = {}

# The transform fits are many small independent SVDs (~1000 x 24), one stacked
# SVD per transform, with a single-threaded BLAS.
_BLAS = {'ctrl': None, 'depth': 0, 'limit': None, 'lock': threading.Lock()}


@contextlib.contextmanager
def _single_threaded_blas():
    """One BLAS thread per call while any fit is running (the limit is
    process-wide, so only the outermost entry sets and restores it)."""
    b = _BLAS
    with b['lock']:
        if b['depth'] == 0 and ThreadpoolController is not None:
            if b['ctrl'] is None:
                b['ctrl'] = ThreadpoolController()
            b['limit'] = b['ctrl'].limit(limits=1)
        b['depth'] += 1
    try:
        yield
    finally:
        with b['lock']:
            b['depth'] -= 1
            if b['depth'] == 0 and b['limit'] is not None:
                b['limit'].restore_original_limits()
                b['limit'] = None

# transform kinds, numbered as GreenX numbers them
COSINE_TW, COSINE_WT, SINE_TW, SINE_WT = 1, 2, 3, 4

#: at or above this many input points the fit gets a Tikhonov term
REGULARIZE_FROM = 20
TIKHONOV = 1e-8
#: singular values at or below this fraction of the largest are dropped
FIT_RCOND = 1e-100
FIT_ERROR_WARN = 1e-3
#: padding (below, above) of the two self-energy fit ranges
SELF_ENERGY_PAD = (0.3, 3.0)
#: Laplace-residual target of the automatic point count
DEFAULT_TAU_TARGET = 1e-10
#: Pade sample points and the scale of their Gauss-Legendre axis
DEFAULT_NPADE = 16
DEFAULT_W0 = 1.0


def _table(kind):
    if kind not in _TABLES:
        name = {'tau': 'greenx_minimax_tau.json',
                'omega': 'greenx_minimax_omega.json'}[kind]
        with open(os.path.join(_DATA, name)) as fh:
            _TABLES[kind] = json.load(fh)
    return _TABLES[kind]


def supported_sizes(kind='tau'):
    return sorted(int(k) for k in _table(kind))


def particle_hole_window(eps, nocc):
    """(gap, span, mu): smallest and largest eps_a - eps_i and the mid-gap
    chemical potential (``src/Base/orbital_spaces.py:12-20``)."""
    eps = np.asarray(eps, float)
    homo, lumo = eps[:nocc].max(), eps[nocc:].min()
    return lumo - homo, eps[nocc:].max() - eps[:nocc].min(), 0.5 * (homo + lumo)


def _check_range(e_min, e_max, who):
    if not e_min > 0:
        raise ValueError(f'{who}: e_min = {e_min:.6g} is not positive; the '
                         f'T = 0 grids are scaled by the gap and need one')
    if e_max is not None and not e_max > e_min:
        raise ValueError(f'{who}: e_max = {e_max:.6g} must exceed '
                         f'e_min = {e_min:.6g}')


def _row(entry, n, e_min, e_max):
    """The tabulated row for range e_max/e_min and the narrow-range stretch.

    The first bin whose range exceeds the requested ratio is used (the last
    bin beyond the widest); below the narrowest bin, grids of more than 20
    points slide that bin down by e_ratio (divided by 1.5 when above 1.5).
    """
    ranges = entry['energy_range']
    ratio = e_max / e_min
    pick = len(ranges)
    for i, top in enumerate(ranges):
        if ratio < top:
            pick = i
            break
    stretch = 1.0
    if pick == 0 and n > 20:
        stretch = ranges[0] / ratio
        if stretch > 1.5:
            stretch /= 1.5
    return np.array(entry['aw_erange_matrix'][pick]), stretch


def minimax_frequency_grid(nfreq, e_min, e_max):
    """(points, weights) of the tabulated minimax frequency axis."""
    _check_range(e_min, e_max, 'minimax_frequency_grid')
    tab = _table('omega')
    if str(nfreq) not in tab:
        raise ValueError(f'nfreq={nfreq} is not tabulated; sizes: '
                         f'{supported_sizes("omega")}')
    row, stretch = _row(tab[str(nfreq)], nfreq, e_min, e_max)
    # frequencies carry energy: the stretch divides, e_min multiplies
    return row[:nfreq] / stretch * e_min, row[nfreq:] / stretch * e_min


def minimax_time_grid(ntau, e_min, e_max):
    """(points, weights) with 1/x ~ sum_k w_k exp(-x tau_k) on [e_min, e_max]."""
    _check_range(e_min, e_max, 'minimax_time_grid')
    tab = _table('tau')
    if str(ntau) not in tab:
        raise ValueError(f'ntau={ntau} is not tabulated; sizes: '
                         f'{supported_sizes("tau")}')
    row, stretch = _row(tab[str(ntau)], ntau, e_min, e_max)
    # times carry 1/energy: the stretch multiplies, e_min divides
    return row[:ntau] * stretch / e_min, row[ntau:] * stretch / e_min


def gauss_legendre_grid(nfreq, w0):
    """Gauss-Legendre nodes mapped onto [0, inf) with scale w0."""
    _check_range(w0, None, 'gauss_legendre_grid (w0)')
    x, w = np.polynomial.legendre.leggauss(nfreq)
    return w0 * (1.0 + x) / (1.0 - x), w0 * 2.0 * w / (1.0 - x) ** 2


def pade_nodes(npade=DEFAULT_NPADE, w0=DEFAULT_W0):
    return gauss_legendre_grid(npade, w0)[0]


def laplace_test_error(npoints, ratio, nsample=4001, relative=False):
    """max over x in [1, R] of |1/x - sum_k w_k exp(-x tau_k)| (or relative)."""
    tau, w = minimax_time_grid(npoints, 1.0, float(ratio))
    x = np.exp(np.linspace(0.0, np.log(float(ratio)), nsample))
    approx = np.exp(-np.outer(x, tau)) @ w
    if relative:
        return float(np.abs(1.0 - x * approx).max())
    return float(np.abs(1.0 / x - approx).max())


def minimax_points_for_accuracy(e_min, e_max, target, npoints_max=34,
                                relative=False):
    """(n, residual): smallest tabulated grid meeting `target`, else the best."""
    _check_range(float(e_min), float(e_max), 'minimax_points_for_accuracy')
    ratio = float(e_max) / float(e_min)
    sizes = set(supported_sizes('tau'))
    best = (None, np.inf)
    for n in range(6, npoints_max + 1, 2):
        if n not in sizes:
            continue
        err = laplace_test_error(n, ratio, relative=relative)
        if err < best[1]:
            best = (n, err)
        if err <= target:
            return n, err
    if best[0] is None:
        raise ValueError(f'no tabulated grid fits e_max/e_min = {ratio:.6g}')
    return best


def minimax_points_for_ranges(ratios, target=DEFAULT_TAU_TARGET, npoints_max=34):
    npoints, worst = 0, 0.0
    for ratio in ratios:
        n, err = minimax_points_for_accuracy(1.0, ratio, target, npoints_max)
        npoints, worst = max(npoints, n), max(worst, err)
    return npoints, worst


def _fit_problem(kind, tau, omega, i, x):
    """Target psi(x) and design matrix of output row i of one transform."""
    if kind == COSINE_TW:
        w = omega[i]
        return (2 * x / (x ** 2 + w ** 2),
                np.cos(w * tau)[None, :] * np.exp(-np.outer(x, tau)))
    if kind == COSINE_WT:
        t = tau[i]
        return (np.exp(-x * t),
                np.cos(t * omega)[None, :]
                * (2 * x[:, None] / (x[:, None] ** 2 + omega[None, :] ** 2)))
    if kind == SINE_TW:
        w = omega[i]
        return (2 * w / (x ** 2 + w ** 2),
                np.sin(w * tau)[None, :] * np.exp(-np.outer(x, tau)))
    if kind == SINE_WT:
        t = tau[i]
        return (np.exp(-x * t),
                np.sin(t * omega)[None, :]
                * (2 * omega[None, :] / (x[:, None] ** 2 + omega[None, :] ** 2)))
    raise ValueError(f'unknown transform kind {kind}')


def transform_weights(kind, tau, omega, e_min, e_max, regularization=None,
                      nodes_factor=200, warn=True):
    """(W, max_fit_error): one tau<->omega transform matrix, cos/sin absorbed.

    Each output point is an independent least-squares problem on a
    logarithmic node set over [e_min, e_max]; the pseudo-inverse keeps the
    singular values above FIT_RCOND times the largest, with a Tikhonov filter
    S/(r^2 + S^2) from REGULARIZE_FROM input points on. Rows are (omega, tau)
    for the *_TW kinds and (tau, omega) for the *_WT kinds.
    """
    tau, omega = np.asarray(tau, float), np.asarray(omega, float)
    forward = kind in (COSINE_TW, SINE_TW)
    n_out = len(omega) if forward else len(tau)
    n_in = len(tau) if forward else len(omega)
    reg = regularization
    if reg is None:
        reg = 0.0 if n_in < REGULARIZE_FROM else TIKHONOV
    nx = max((int(np.log10(e_max / e_min)) + 1) * nodes_factor, n_in)
    x = e_min * (e_max / e_min) ** (np.arange(nx) / (nx - 1.0))
    W = np.zeros((n_out, n_in))
    # every row's design matrix in one stack and one stacked SVD (LAPACK per
    # matrix, outside the interpreter lock), then each row's filtered
    # pseudo-inverse exactly as a single row's fit computes it
    probs = [_fit_problem(kind, tau, omega, i, x) for i in range(n_out)]
    A_all = np.stack([A for _, A in probs])
    with _single_threaded_blas():
        U_all, S_all, Vt_all = np.linalg.svd(A_all, full_matrices=False)
    errs = []
    for i, (psi, A) in enumerate(probs):
        U, S, Vt = U_all[i], S_all[i], Vt_all[i]
        keep = S > FIT_RCOND * S[0]
        filt = np.zeros_like(S)
        np.divide(S, reg ** 2 + S ** 2, out=filt, where=keep)
        W[i] = Vt.T @ (filt * (U.T @ psi))
        errs.append(float(np.abs(A @ W[i] - psi).max()))
    worst = 0.0
    for i, err in enumerate(errs):
        if not (np.isfinite(err) and np.isfinite(W[i]).all()):
            raise FloatingPointError(
                f'transform kind {kind}: row {i} of {n_out} is not finite '
                f'(n={n_in}, e_max/e_min={e_max / e_min:.6g}); no W(tau) or '
                f'self-energy can be built on it')
        worst = max(worst, err)
    if warn and not worst <= FIT_ERROR_WARN:
        warnings.warn(f'minimax transform fit reached only {worst:.2e} at '
                      f'{n_in} points over e_max/e_min = {e_max / e_min:.3g}; '
                      f'use more points', RuntimeWarning, stacklevel=2)
    trig = np.cos if kind in (COSINE_TW, COSINE_WT) else np.sin
    phase = trig(np.outer(omega, tau))
    return (W * phase if forward else W * phase.T), worst


def minimax_transform_weights(kind, tau, omega, e_min, e_max, regularization=None,
                              nodes_factor=200, warn=True):
    """The reference's name for `transform_weights`
    (``Base/utils/grids/time_frequency.py:282-380``)."""
    return transform_weights(kind, tau, omega, e_min, e_max, regularization=regularization,
                             nodes_factor=nodes_factor, warn=warn)


@dataclass
class TimeFrequencyGrid:
    """Both imaginary axes and the transforms between them (T = 0 minimax).

    cosft_wt (nfreq, ntau): even tau -> omega; cosft_tw (ntau, nfreq): even
    omega -> tau; sinft_* likewise for odd functions.
    """
    tau_points: np.ndarray
    tau_weights: np.ndarray
    omega_points: np.ndarray
    omega_weights: np.ndarray
    cosft_wt: np.ndarray = None
    cosft_tw: np.ndarray = None
    sinft_wt: np.ndarray = None
    sinft_tw: np.ndarray = None
    fit_errors: dict = field(default_factory=dict)
    meta: dict = field(default_factory=dict)

    @property
    def ntau(self):
        return len(self.tau_points)

    @property
    def nfreq(self):
        return len(self.omega_points)

    @classmethod
    def minimax_split(cls, ntau, e_min, e_max, omega_points, omega_weights,
                      regularization=None, with_sine=True, with_inverse=True):
        """Minimax tau axis of `ntau` points (half the Laplace scaling, the
        time-frequency pair's 1/(2 e_min)) onto a caller's frequency axis."""
        tau, tw = minimax_time_grid(ntau, e_min, e_max)
        tau, tw = 0.5 * tau, 0.5 * tw
        omega_points = np.asarray(omega_points, float)
        kinds = [('cosft_wt', COSINE_TW)]
        if with_inverse:
            kinds.append(('cosft_tw', COSINE_WT))
        if with_sine:
            kinds.append(('sinft_wt', SINE_TW))
            if with_inverse:
                kinds.append(('sinft_tw', SINE_WT))
        mats, errs = {}, {}
        # the transforms' rows all go to the fit pool at once
        with _single_threaded_blas(), ThreadPoolExecutor(max_workers=len(kinds)) as outer:
            futs = {name: outer.submit(transform_weights, kind, tau, omega_points, e_min,
                                       e_max, regularization)
                    for name, kind in kinds}
            for name, f in futs.items():
                mats[name], errs[name] = f.result()
        return cls(tau, tw, omega_points, np.asarray(omega_weights, float),
                   fit_errors=errs,
                   meta={'e_min': e_min, 'e_max': e_max, 'ntau': ntau,
                         'nfreq': len(omega_points)}, **mats)

    @classmethod
    def minimax(cls, npoints, e_min, e_max, regularization=None, with_sine=True):
        w, ww = minimax_frequency_grid(npoints, e_min, e_max)
        return cls.minimax_split(npoints, e_min, e_max, w, ww,
                                 regularization=regularization,
                                 with_sine=with_sine)


def self_energy_fit_ranges_from_window(eps, mu, w_lo, w_hi, pad=SELF_ENERGY_PAD):
    lo, hi = pad
    dG = np.abs(np.asarray(eps) - mu)
    return ((lo * w_lo, hi * w_hi),
            (lo * (float(dG.min()) + w_lo), hi * (float(dG.max()) + w_hi)))


def sigma_fit_ranges(eps, nocc, mu=None):
    """(rW, rS): fit range of W - I (padded window) and of Sigma (sums of
    |eps - mu| and the window, padded)."""
    eps = np.asarray(eps, float)
    occ, virt = eps[:nocc], eps[nocc:]
    if mu is None:
        mu = 0.5 * (occ.max() + virt.min())
    w_lo, w_hi = virt.min() - occ.max(), virt.max() - occ.min()
    return self_energy_fit_ranges_from_window(eps, mu, w_lo, w_hi)


def screening_frequency_grid(ntau, eps, nocc, mu=None):
    """Minimax frequencies over rW, where W(i omega) is sampled."""
    rW, _ = sigma_fit_ranges(eps, nocc, mu=mu)
    return minimax_frequency_grid(ntau, *rW)


def minimax_points_for_gw(eps, nocc, mu=None, target=DEFAULT_TAU_TARGET,
                          npoints_max=34):
    """(n, residual) resolving the chi0 window, rW and rS at once."""
    gap, span, mid = particle_hole_window(eps, nocc)
    mu = mid if mu is None else mu
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    return minimax_points_for_ranges((span / gap, rW[1] / rW[0], rS[1] / rS[0]),
                                     target=target, npoints_max=npoints_max)


def sigma_transforms(eps, nocc, tau_points, omega_in, omega_out, mu=None, intermediate=None):
    """(Ctw, C, S): the omega -> tau weights of W - I over rW and the tau ->
    omega cosine and sine weights of Sigma over rS, on the caller's axes
    (``Base/utils/grids/time_frequency.py:430-448``). Frozen per geometry, as
    the reference treats them: not differentiated."""
    if intermediate is not None:
        raise NotImplementedError('an intermediate-orbital mask is outside the device route')
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    Ctw = transform_weights(COSINE_WT, tau_points, omega_in, *rW)[0]
    C = transform_weights(COSINE_TW, tau_points, omega_out, *rS)[0]
    S = transform_weights(SINE_TW, tau_points, omega_out, *rS)[0]
    return Ctw, C, S


def transition_range(spectra, noccs):
    """(smallest, largest) particle-hole energy over every spin channel
    (``src/Base/orbital_spaces.py:23-29``)."""
    windows = [particle_hole_window(e, n) for e, n in zip(spectra, noccs)]
    return min(w[0] for w in windows), max(w[1] for w in windows)


def minimax_points_for_bse(eps, nocc, tau_target=DEFAULT_TAU_TARGET):
    """(ntau, residual) of the static screening's time grid: only chi0 is
    transformed, so the chi0 transition range alone sizes it
    (``LinearResponse/space_time.py:971-981``)."""
    gap, span, _ = particle_hole_window(eps, nocc)
    return minimax_points_for_accuracy(gap, span, target=tau_target)


def static_screening_grid(eps, nocc, ntau=None, tau_target=DEFAULT_TAU_TARGET):
    """The one-frequency (omega = 0, weight 1) minimax split on which the
    static screening is built, cosine tau -> omega weights only
    (``LinearResponse/space_time.py:984-1000``). ntau None or 'auto' sizes
    it by `minimax_points_for_bse`."""
    e_min, e_max, _ = particle_hole_window(eps, nocc)
    if ntau is None or (isinstance(ntau, str) and ntau.lower() == 'auto'):
        ntau, _ = minimax_points_for_bse(eps, nocc, tau_target=tau_target)
    return TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, [0.0], [1.0],
                                           with_sine=False, with_inverse=False)


@dataclass
class SpaceTimeAxes:
    """The axes of one space-time GW solve.

    mu: the mid-gap (restricted), or one per spin channel (unrestricted);
    grid: chi0's tau axis onto the screening frequencies, with the cosine
    tau -> omega weights cosft_wt only (the route's one use of the grid; the
    full four-matrix grid is TimeFrequencyGrid.minimax_split on the same
    arguments);
    tau_sigma: the self-energy's own tau axis (half the rS minimax points);
    Ctw (ntau, nfreq): omega -> tau cosine weights of W - I over rW;
    C, S (npade, ntau): tau -> i omega cosine / sine weights of Sigma over rS;
    pade_freq: the Pade sample frequencies.
    """
    ntau: int
    mu: float | tuple
    grid: TimeFrequencyGrid
    tau_sigma: np.ndarray
    Ctw: np.ndarray
    C: np.ndarray
    S: np.ndarray
    pade_freq: np.ndarray
    ranges: tuple
    tau_fit_error: float = None


def space_time_axes(eps, nocc, ntau='auto', pade_freq=None, anchor=None,
                    tau_target=DEFAULT_TAU_TARGET):
    """All axes and weights of the restricted route, as the reference driver
    builds them (``GW/space_time.py:559-618`` and
    ``GW/imaginary_time.py:459-472``). `anchor` sizes an automatic ntau
    (the mean-field spectrum of an evGW run)."""
    eps = np.asarray(eps, float)
    e_min, e_max, mu = particle_hole_window(eps, nocc)
    tau_err = None
    if ntau is None or (isinstance(ntau, str) and ntau.lower() == 'auto'):
        a = eps if anchor is None else np.asarray(anchor, float)
        ntau, tau_err = minimax_points_for_gw(
            a, nocc, mu=particle_hole_window(a, nocc)[2], target=tau_target)
    if int(ntau) not in supported_sizes('omega'):
        raise ValueError(f'ntau = {ntau} has no tabulated frequency grid')
    ntau = int(ntau)
    freq, fw = screening_frequency_grid(ntau, eps, nocc, mu=mu)
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    tau_sigma = 0.5 * minimax_time_grid(ntau, *rS)[0]
    pade = pade_nodes() if pade_freq is None else np.asarray(pade_freq, float)
    # the seven transform fits are independent: all in flight at once
    with _single_threaded_blas(), ThreadPoolExecutor(max_workers=4) as outer:
        f_grid = outer.submit(TimeFrequencyGrid.minimax_split, ntau, e_min, e_max, freq, fw,
                              with_sine=False, with_inverse=False)
        f_ctw = outer.submit(transform_weights, COSINE_WT, tau_sigma, freq, *rW, warn=False)
        f_c = outer.submit(transform_weights, COSINE_TW, tau_sigma, pade, *rS, warn=False)
        f_s = outer.submit(transform_weights, SINE_TW, tau_sigma, pade, *rS, warn=False)
        grid, (Ctw, _), (C, _), (S, _) = (f_grid.result(), f_ctw.result(), f_c.result(),
                                          f_s.result())
    return SpaceTimeAxes(ntau, mu, grid, tau_sigma, Ctw, C, S, pade,
                         (rW, rS), tau_err)


def unrestricted_fit_ranges(spectra, noccs):
    """(rW, rS) of an unrestricted reference (``GW/imaginary_time.py:141-155``):
    the restricted rule on both spin channels together, each channel at its
    own mid-gap, rW from the union of the transitions and rS the hull of the
    channels' self-energy ranges."""
    w_lo, w_hi = transition_range(spectra, noccs)
    parts = [self_energy_fit_ranges_from_window(e, 0.5 * (e[n - 1] + e[n]), w_lo, w_hi)
             for e, n in ((np.asarray(e, float), n) for e, n in zip(spectra, noccs))]
    rW = parts[0][0]
    return rW, (min(rS[0] for _, rS in parts), max(rS[1] for _, rS in parts))


def unrestricted_screening_frequency_grid(ntau, spectra, noccs):
    """Minimax frequencies over the two-spin rW (``GW/imaginary_time.py:158-163``)."""
    rW, _ = unrestricted_fit_ranges(spectra, noccs)
    return minimax_frequency_grid(ntau, *rW)


def minimax_points_for_gw_unrestricted(spectra, noccs, target=DEFAULT_TAU_TARGET,
                                       npoints_max=34):
    """`minimax_points_for_gw` over both spin channels' ranges together
    (``GW/imaginary_time.py:166-173``)."""
    w_lo, w_hi = transition_range(spectra, noccs)
    rW, rS = unrestricted_fit_ranges(spectra, noccs)
    return minimax_points_for_ranges((w_hi / w_lo, rW[1] / rW[0], rS[1] / rS[0]),
                                     target=target, npoints_max=npoints_max)


def space_time_axes_unrestricted(spectra, noccs, ntau='auto', pade_freq=None, anchors=None,
                                 tau_target=DEFAULT_TAU_TARGET):
    """The axes of the unrestricted route (``GW/space_time.py:559-618`` with two
    channels): chi0's time grid over both spins' transitions, W's frequencies
    and the self-energy's fit ranges over both channels, so that one W serves
    either channel. `mu` is the tuple of the channels' own mid-gaps, on which
    each channel samples its self-energy. `anchors` (one spectrum per spin)
    size an automatic ntau."""
    spectra = [np.asarray(e, float) for e in spectra]
    noccs = [int(n) for n in noccs]
    e_min, e_max = transition_range(spectra, noccs)
    tau_err = None
    if ntau is None or (isinstance(ntau, str) and ntau.lower() == 'auto'):
        a = spectra if anchors is None else [np.asarray(x, float) for x in anchors]
        ntau, tau_err = minimax_points_for_gw_unrestricted(a, noccs, target=tau_target)
    if int(ntau) not in supported_sizes('omega'):
        raise ValueError(f'ntau = {ntau} has no tabulated frequency grid')
    ntau = int(ntau)
    freq, fw = unrestricted_screening_frequency_grid(ntau, spectra, noccs)
    rW, rS = unrestricted_fit_ranges(spectra, noccs)
    tau_sigma = 0.5 * minimax_time_grid(ntau, *rS)[0]
    pade = pade_nodes() if pade_freq is None else np.asarray(pade_freq, float)
    with _single_threaded_blas(), ThreadPoolExecutor(max_workers=4) as outer:
        f_grid = outer.submit(TimeFrequencyGrid.minimax_split, ntau, e_min, e_max, freq, fw,
                              with_sine=False, with_inverse=False)
        f_ctw = outer.submit(transform_weights, COSINE_WT, tau_sigma, freq, *rW, warn=False)
        f_c = outer.submit(transform_weights, COSINE_TW, tau_sigma, pade, *rS, warn=False)
        f_s = outer.submit(transform_weights, SINE_TW, tau_sigma, pade, *rS, warn=False)
        grid, (Ctw, _), (C, _), (S, _) = (f_grid.result(), f_ctw.result(), f_c.result(),
                                          f_s.result())
    mus = tuple(particle_hole_window(e, n)[2] for e, n in zip(spectra, noccs))
    return SpaceTimeAxes(ntau, mus, grid, tau_sigma, Ctw, C, S, pade, (rW, rS), tau_err)
