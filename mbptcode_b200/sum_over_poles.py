"""The contour's self-energy as a sum over auxiliary poles (continuation 'sop').

MBPTcode ``GW/sum_over_poles.py``: W on the imaginary axis, as the screening
contraction wc[k, q] = B_p[:, q]^T [W(i nu_k) - I] B_p[:, q] already gives it,
is modelled by M common poles Om_m,

    wc[k, q] ~= sum_m A[m, q] (-2 Om_m / (nu_k^2 + Om_m^2)),

and the frequency convolution then closes:

    Sigma^c_pp(w) = sum_{s, m} A[m, s] / (w - d[s, m]),
    d[s, m] = eps_s - Om_m (occupied s), eps_s + Om_m (virtual s).

The poles are placed by vector fitting (Gustavsen and Semlyen, 1999) in the
variable u = z^2, where the model is real and even: the linear least squares
for the amplitudes of f and of a weight function on shared poles, the new
poles the zeros of that weight (the eigenvalues of diag(u) - 1 b^T), clipped
to the particle-hole range and merged where they coalesce. The amplitudes are
then the fixed linear map A = F^+ wc. The quasiparticle equation
w = eps_p + xc + Sigma(w) has known poles, so every real root is found interval by
interval (`pole_sum_roots`), the root of largest valid weight kept, or with
`follow` the one continuing a walk's branch between the same two labelled
poles.

Everything here is host FP64 algebra on a few hundred numbers per state,
fed by the device-made screening contraction; the screening itself is never
evaluated off the imaginary axis on this route.
"""
from __future__ import annotations

import warnings

import numpy as np
import scipy.linalg

# MBPTcode src/Base/numerics/constants.py
SOP_CLEARANCE_MIN = 0.05          # :514
SOP_FIT_RCOND = 1e-12             # :518
SOP_POLE_MERGE_TOL = 1e-3         # :537
SOP_N_POLES = 12                  # :541
SOP_FIT_STRIDE = 8                # :545
QP_WINDOW_Z_MIN = 0.5             # :553
QP_ROOT_TOL = 1e-10               # :1596
QP_POLE_OFFSET = 1e-3             # :462
QP_POLE_INTERVAL_SAMPLES = 3      # :1604
QP_GRAPHICAL_N_OMEGA = 150        # :273
QP_GRAPHICAL_MAX_BISECTION = 100  # :274


class VectorFitFallback(RuntimeWarning):
    """The vector fit's least squares needed another LAPACK driver."""


def _ov_energies(eps, nocc):
    eps = np.asarray(eps, float)
    return (eps[nocc:][None, :] - eps[:nocc][:, None]).ravel()


def _residue_set(eps, nocc, w):
    from .contour import residue_set
    return residue_set(eps, nocc, w)


def qp_start(eps, p, nocc, offset=QP_POLE_OFFSET):
    """eps_p moved `offset` toward the chemical potential: where a state is
    judged before its root is known (``Solvers/qp_equation.py:87-92``)."""
    return float(eps[p] + (offset if p < nocc else -offset))


# ---------------------------------------------------------------- the model
def initial_poles(n_poles, gap, e_max):
    """n_poles log-spaced on [gap, e_max] (``sum_over_poles.py:61-70``)."""
    if not 0.0 < gap < e_max:
        raise ValueError(f'poles need 0 < gap < e_max, got {gap} and {e_max}')
    return np.logspace(np.log10(gap), np.log10(e_max), int(n_poles))


def pole_basis(nu_points, poles):
    """F[k, m] = -2 Om_m / (nu_k^2 + Om_m^2), the model's imaginary-axis
    columns (real: the two terms of a pole pair combine)."""
    nu = np.asarray(nu_points, float)[:, None]
    om = np.asarray(poles, float)[None, :]
    return -2.0 * om / (nu * nu + om * om)


def pole_pseudoinverse(nu_points, poles, rcond=SOP_FIT_RCOND):
    """F^+, the map from wc to amplitudes (one operator for the fit and for
    anything differentiated through it)."""
    return np.linalg.pinv(pole_basis(nu_points, poles), rcond=rcond)


def pole_amplitudes(wc, poles, nu_points, rcond=SOP_FIT_RCOND):
    """A (n_poles, norb) = F^+ wc."""
    return pole_pseudoinverse(nu_points, poles, rcond) @ np.asarray(wc, float)


def _lstsq(block, rhs):
    """Least squares by LAPACK's divide-and-conquer SVD; where it does not
    converge, by the QR-iteration SVD, then by pivoted QR."""
    try:
        return np.linalg.lstsq(block, rhs, rcond=None)[0]
    except np.linalg.LinAlgError as exc:
        failed = exc
    cut = np.finfo(float).eps * max(block.shape)
    for driver in ('gelss', 'gelsy'):
        warnings.warn(f'vector fitting: the least squares failed on a {block.shape} block '
                      f'({failed}); solved by {driver} instead', VectorFitFallback,
                      stacklevel=3)
        try:
            return scipy.linalg.lstsq(block, rhs, cond=cut, lapack_driver=driver)[0]
        except np.linalg.LinAlgError as exc:
            failed = exc
    raise failed


def merge_poles(poles, tol=SOP_POLE_MERGE_TOL):
    """Sorted poles with every chain of neighbours closer than tol (relative
    to the previous one) replaced by its root-mean-square, so that no two
    columns of the least squares coincide (``sum_over_poles.py:131-152``)."""
    om = np.sort(np.asarray(poles, float))
    if tol is None or om.size < 2:
        return om
    out, chain = [], [om[0]]
    for w in om[1:]:
        if w - chain[-1] <= tol * chain[-1]:
            chain.append(w)
            continue
        out.append(chain[0] if len(chain) == 1 else float(np.sqrt(np.mean(np.square(chain)))))
        chain = [w]
    out.append(chain[0] if len(chain) == 1 else float(np.sqrt(np.mean(np.square(chain)))))
    return np.array(out)


def fit_poles(wc, nu_points, poles, n_iter=5, stride=1, bounds=None, state=None,
              merge_tol=SOP_POLE_MERGE_TOL):
    """The poles after n_iter vector-fitting passes in u = z^2 on every
    stride-th column of wc (``sum_over_poles.py:155-211``): per pass the
    amplitudes of every column and the weight's residues b solved together,
    the new u the eigenvalues of diag(Om^2) - 1 b^T, clipped to bounds^2."""
    wc = np.asarray(wc, float)
    if not np.isfinite(wc).all():
        bad = np.unique(np.argwhere(~np.isfinite(wc))[:, 1])
        raise FloatingPointError(
            'W_c on the imaginary axis is not finite'
            f'{"" if state is None else f" for orbital {state}"}: columns '
            f'{bad[:10].tolist()}{" ..." if bad.size > 10 else ""} of {wc.shape[1]}; no pole '
            'model is fitted to it')
    om = np.asarray(poles, float).copy()
    lo, hi = bounds if bounds is not None else (om[0], om[-1])
    u = -np.asarray(nu_points, float) ** 2
    cols = wc[:, ::max(int(stride), 1)]
    nk, nc = cols.shape
    rhs = cols.T.ravel()
    for _ in range(int(n_iter)):
        if merge_tol is not None:
            om = merge_poles(om, merge_tol)
        npl = om.size
        kern = 1.0 / (u[:, None] - (om * om)[None, :])
        block = np.zeros((nk * nc, nc * npl + npl))
        for j in range(nc):
            rows = slice(j * nk, (j + 1) * nk)
            block[rows, j * npl:(j + 1) * npl] = kern
            block[rows, nc * npl:] = -cols[:, j][:, None] * kern
        b = _lstsq(block, rhs)[nc * npl:]
        zeros = np.linalg.eigvals(np.diag(om * om) - np.outer(np.ones(npl), b))
        om = np.sqrt(np.sort(np.clip(np.real(zeros), lo * lo, hi * hi)))
    return om if merge_tol is None else merge_poles(om, merge_tol)


def sop_from_wc(wc, nu_points, eps, nocc, n_poles=SOP_N_POLES, relocate=True,
                stride=SOP_FIT_STRIDE, e_max=None, pair_energies=None, state=None):
    """(poles, amplitudes) of one state from its wc (nfreq, norb): poles
    log-spaced over the particle-hole energies, relocated by `fit_poles`
    inside them, then A = F^+ wc (``sum_over_poles.py:349-367``).
    pair_energies: the screening's particle-hole energies where they are not
    (eps, nocc)'s (both spins of an unrestricted reference)."""
    if hasattr(wc, 'detach'):
        wc = wc.detach().cpu().numpy()
    d = _ov_energies(eps, nocc) if pair_energies is None else np.asarray(pair_energies, float)
    gap, top = float(d.min()), float(e_max if e_max is not None else d.max())
    poles = initial_poles(n_poles, gap, top)
    if relocate:
        poles = fit_poles(wc, nu_points, poles, stride=stride, bounds=(gap, top), state=state)
    return poles, pole_amplitudes(wc, poles, nu_points)


def denominators(omega, poles, eps, nocc):
    """D[q, m] = omega - eps_q + Om_m (occupied q), - Om_m (virtual q)."""
    sign = np.where(np.arange(len(eps)) < nocc, 1.0, -1.0)
    return ((omega - np.asarray(eps, float))[:, None]
            + sign[:, None] * np.asarray(poles, float)[None, :])


def pole_denominators(poles, eps, nocc):
    """d[s, m], the real-axis poles of Sigma: eps_s - Om_m (occupied s),
    eps_s + Om_m (virtual s)."""
    sign = np.where(np.arange(len(eps)) < nocc, 1.0, -1.0)
    return np.asarray(eps, float)[:, None] - sign[:, None] * np.asarray(poles, float)[None, :]


def pole_clearance(omega, poles, eps, nocc):
    """min |D| / min Om: how near the model is to a resonance of its own."""
    return float(np.abs(denominators(omega, poles, eps, nocc)).min() / np.min(poles))


def pole_condition(omega, eps, nocc, limit):
    """(ok, reach): the farthest pole of G the contour sweeps at omega, in
    units of limit, and whether it is below one (Eq. 27 of the pole model)."""
    swept = _residue_set(eps, nocc, omega)
    reach = max((abs(eps[q] - omega) for q, _ in swept), default=0.0) / limit
    return bool(reach < 1.0), float(reach)


def compressible(omega, eps, nocc, pair_energies=None):
    """(ok, reach) of the compression condition against the particle-hole
    gap E_g (the lowest neutral excitation's dRPA bound): every pole the
    contour sweeps must lie within one gap of omega
    (``sum_over_poles.py:232-265``)."""
    limit = float((_ov_energies(eps, nocc) if pair_energies is None
                   else np.asarray(pair_energies, float)).min())
    return pole_condition(omega, eps, nocc, limit)


def sigma_sop(omega, amplitudes, poles, eps, nocc, check=True, out=None):
    """Sigma^c_pp(omega) of the pole model, closed form. check: warn where
    the compression condition excludes the state or the model is resonant
    at omega (the names go to `out`, 'compression_excluded' with the reach
    and 'resonant' with the clearance)."""
    if check:
        ok, reach = compressible(omega, eps, nocc)
        if not ok:
            if out is not None:
                out['compression_excluded'] = reach
            warnings.warn(f'omega = {omega:.4f} sweeps a pole {reach:.2f} gaps away: the '
                          'compression condition excludes this state, where single '
                          'excitations of W matter and no number of model poles converges; '
                          'use the real-axis route.', RuntimeWarning, stacklevel=2)
        clear = pole_clearance(omega, poles, eps, nocc)
        if clear < SOP_CLEARANCE_MIN:
            if out is not None:
                out['resonant'] = float(clear)
            warnings.warn(f'the pole model is resonant at omega = {omega:.4f}: its closest '
                          f'denominator is {clear:.2g} of the lowest model pole.',
                          RuntimeWarning, stacklevel=2)
    return float(np.sum(np.asarray(amplitudes, float).T / denominators(omega, poles, eps, nocc)))


def sigma_sop_slope(omega, amplitudes, poles, eps, nocc):
    """dSigma^c_pp/domega of the pole model at fixed amplitudes."""
    d = denominators(omega, poles, eps, nocc)
    return -float(np.sum(np.asarray(amplitudes, float).T / (d * d)))


# ------------------------------------------------ roots of a sum of poles
def _prepare(num, pol):
    """(num, pol, labels): sorted by pole; with any negative weight,
    coinciding poles summed into the first of them; zero weights dropped
    (positive weights: only positive ones kept). labels: indices as given."""
    num = np.asarray(num, float).ravel()
    pol = np.asarray(pol, float).ravel()
    order = np.argsort(pol, kind='stable')
    if (num < 0.0).any():
        upol, first = np.unique(pol[order], return_index=True)
        unum = np.add.reduceat(num[order], first) if num.size else num
        keep = unum != 0.0
        return unum[keep], upol[keep], order[first][keep], True
    num, pol, lab = num[order], pol[order], order
    keep = num > 0.0
    return num[keep], pol[keep], lab[keep], False


def _values(num, pol, a, w, block=1 << 22):
    """(f, f') of f(w) = w - a - sum num/(w - pol) on the points w."""
    w = np.asarray(w, float)
    f, fp = np.empty(w.size), np.empty(w.size)
    rows = max(1, block // max(pol.size, 1))
    for r0 in range(0, w.size, rows):
        inv = 1.0 / (w[r0:r0 + rows, None] - pol[None, :])
        r = num[None, :] * inv
        f[r0:r0 + rows] = w[r0:r0 + rows] - a - r.sum(1)
        fp[r0:r0 + rows] = 1.0 + (r * inv).sum(1)
    return f, fp


def _newton_all(num, pol, a, L, R, SL, tol, max_iter=QP_GRAPHICAL_MAX_BISECTION):
    """The root in each bracket (L, R) (f of sign SL at L, of the other at R),
    all brackets at once: a Newton step that leaves the bracket is a
    bisection, and so is every second step that has not halved the bracket;
    a step below tol ends a bracket only strictly inside it; one a bit wide
    ends at its point (``qp_equation.py:376-426``, the cheap-f rules)."""
    L, R = np.array(L, float), np.array(R, float)
    SL = np.asarray(SL, float)
    W = 0.5 * (L + R)
    width = R - L
    out = np.full(L.size, np.nan)
    live = SL != 0.0
    out[~live] = L[~live]
    for it in range(int(max_iter)):
        idx = np.nonzero(live)[0]
        if idx.size == 0:
            break
        f, fp = _values(num, pol, a, W[idx])
        w = W[idx]
        zero = f == 0.0
        same = np.sign(f) == SL[idx]
        L[idx] = np.where(same, w, L[idx])
        R[idx] = np.where(same, R[idx], w)
        l, r = L[idx], R[idx]
        with np.errstate(divide='ignore', invalid='ignore'):
            dw = -f / fp
            conv = (np.abs(dw) < tol) & (l < w + dw) & (w + dw < r)
        mid = 0.5 * (l + r)
        stuck = ~((l < mid) & (mid < r))
        with np.errstate(invalid='ignore'):
            newton = np.isfinite(dw) & (l < w + dw) & (w + dw < r)
        if it % 2:
            newton &= ~(r - l > 0.5 * width[idx])
            width[idx] = r - l
        stop = zero | conv | stuck
        out[idx] = np.where(zero, w, np.where(conv, w + dw, w))
        W[idx] = np.where(stop, w, np.where(newton, w + dw, mid))
        live[idx[stop]] = False
    out[live] = W[live]
    return out


def _turning_split(num, pol, a, l, r, s, sp, tol):
    """Between two nodes where f has sign s and turns toward zero, the point
    where f' = 0 by Newton on f' inside (l, r); where f has the other sign on
    the way, the two brackets either side of it (0 or 2 crossings)."""
    x0, x1 = l, r
    w, width = 0.5 * (l + r), r - l
    for it in range(QP_GRAPHICAL_MAX_BISECTION):
        inv = 1.0 / (w - pol)
        q = num * inv
        qi = q * inv
        fm, fpm, fppm = w - a - q.sum(), 1.0 + qi.sum(), -2.0 * (qi * inv).sum()
        if np.sign(fm) != s:
            return [(x0, w, s), (w, x1, -s)]
        if np.sign(fpm) == sp:
            l = w
        else:
            r = w
        dw = -fpm / fppm if fppm != 0.0 else np.inf
        if abs(dw) < tol or not l < 0.5 * (l + r) < r:
            return []
        newton = l < w + dw < r
        if it % 2 and r - l > 0.5 * width:
            newton = False
        if it % 2:
            width = r - l
        w = w + dw if newton else 0.5 * (l + r)
    return []


def pole_sum_roots(num, pol, a, tol=QP_ROOT_TOL):
    """Every real root of f(w) = w - a - sum_i num_i/(w - pol_i) that the
    interval search finds, as (w, Z, m) with m the interval (pol[m],
    pol[m+1]) of the prepared poles (-1 and n-1 the outer ones), and the
    prepared (num, pol, labels). Between neighbouring poles of positive
    weight f rises from -inf to +inf: one root. Any interval is sampled at
    interior nodes (3 inside, 150 on an outer one) with the poles' known
    limits at its ends: a sign change is a bracket, and two nodes of one
    sign between which f turns toward zero are split at its turning point
    where f changes sign there (``qp_equation.py:429-683``). Z = 1/f'."""
    num, pol, lab, signed = _prepare(num, pol)
    a = float(a)
    n = num.size
    if n == 0:
        return [(a, 1.0, -1)], (num, pol, lab)
    reach = np.sqrt(np.abs(num).sum()) * (1.0 + 1e-9) + 1e-12
    lo_end, hi_end = min(a, pol[0]) - reach, max(a, pol[-1]) + reach
    brackets = []                     # (l, r, sign of f at l, interval)
    for m in range(-1, n):
        if m >= 0:
            l, sl, spl = pol[m], -np.sign(num[m]), np.sign(num[m])
        else:
            l, sl, spl = lo_end, -1.0, None
        if m + 1 < n:
            r, sr, spr = pol[m + 1], np.sign(num[m + 1]), np.sign(num[m + 1])
        else:
            r, sr, spr = hi_end, 1.0, None
        if not l < r:
            continue
        if not signed and 0 <= m < n - 1:
            brackets.append((l, r, -1.0, m))       # rising from -inf to +inf
            continue
        k = QP_POLE_INTERVAL_SAMPLES if 0 <= m < n - 1 else QP_GRAPHICAL_N_OMEGA
        x = l + (r - l) * np.arange(1, k + 1) / (k + 1)
        f, fp = _values(num, pol, a, x)
        if spl is None:
            spl = np.sign(_values(num, pol, a, [l])[1][0])
        if spr is None:
            spr = np.sign(_values(num, pol, a, [r])[1][0])
        xs = np.concatenate([[l], x, [r]])
        sf = np.concatenate([[sl], np.sign(f), [sr]])
        sfp = np.concatenate([[spl], np.sign(fp), [spr]])
        for i in range(xs.size - 1):
            if sf[i] == 0.0:
                brackets.append((xs[i], xs[i], 0.0, m))
            elif sf[i] != sf[i + 1]:
                if sf[i + 1] != 0.0:
                    brackets.append((xs[i], xs[i + 1], sf[i], m))
            elif sfp[i] == -sf[i] and sfp[i + 1] == sf[i]:
                brackets += [br + (m,) for br in _turning_split(num, pol, a, xs[i], xs[i + 1],
                                                                sf[i], sfp[i], tol)]
    if not brackets:
        return [], (num, pol, lab)
    L = np.array([b[0] for b in brackets])
    R = np.array([b[1] for b in brackets])
    S = np.array([b[2] for b in brackets])
    w = _newton_all(num, pol, a, L, R, S, tol)
    _, fp = _values(num, pol, a, w)
    with np.errstate(divide='ignore'):
        z = 1.0 / fp
    return [(float(w[i]), float(z[i]), brackets[i][3]) for i in range(len(brackets))], \
        (num, pol, lab)


def _valid(z, z_min=0.0):
    return bool(np.isfinite(z) and z_min < z <= 1.0)


def solve_qp_equation_poles(num, pol, a, tol=QP_ROOT_TOL, label='', follow=None, out=None):
    """(w, Z) of w = a + sum_i num_i/(w - pol_i) (``qp_equation.py:1423-1441``):
    the root of largest valid weight (Z in (0, 1]), or the root nearest a if
    none is valid; with follow = (w, (lo, hi)) the valid root nearest w
    between the poles labelled lo and hi (indices into num; None for an
    open side; labels None: the interval holding w), the largest weight
    again where that branch has gone. out: a dict that receives 'labels' of
    the root kept, 'largest', 'followed', 'flipped', 'no_root',
    'z_outside'; without it a RuntimeWarning where the largest weight has
    left a followed root."""
    from .gw import QPNoRoot, QPWeightOutside
    roots, (pn, pp, lab) = pole_sum_roots(num, pol, a, tol)
    n = pn.size
    what = label or 'the quasiparticle equation'

    def labels_of(m):
        if n == 0:
            return (None, None)
        return (None if m < 0 else int(lab[m]), None if m + 1 >= n else int(lab[m + 1]))
    ok = [i for i, (_, z, _) in enumerate(roots) if _valid(z)]
    if ok:
        best = max(ok, key=lambda i: roots[i][1])
    elif roots:
        best = min(range(len(roots)), key=lambda i: abs(roots[i][0] - a))
    else:
        best = None
    largest = followed = None
    if follow is None:
        if best is None:
            warnings.warn(f'{what} has no real root.', QPNoRoot, stacklevel=2)
            w, z, labels = np.nan, np.nan, None
        else:
            w, z, m = roots[best]
            labels = labels_of(m)
    else:
        fw, flab = (follow if isinstance(follow, (tuple, list)) else (follow, None))
        fw = float(fw)
        span = None
        if n == 0:
            span = [-1]
        elif flab is None:
            span = [int(np.searchsorted(pp, fw)) - 1]
        else:
            ends = []
            for side, lb in zip((-1, n), flab):
                if lb is None:
                    ends.append(side)
                    continue
                at = np.flatnonzero(lab == int(lb))
                ends.append(int(at[0]) if at.size == 1 else None)
            if None not in ends and ends[0] < ends[1]:
                span = range(ends[0], ends[1])
        got = ([(i, r) for i, r in enumerate(roots) if r[2] in span and _valid(r[1])]
               if span is not None else [])
        if got:
            i, (w, z, m) = min(got, key=lambda ir: abs(ir[1][0] - fw))
            labels, followed = labels_of(m), True
            largest = None if best is None else (roots[best][0], roots[best][1])
        else:
            followed = False
            if best is None:
                warnings.warn(f'{what}: the branch followed from {fw:.6f} Ha has gone and '
                              'the equation has no real root.', QPNoRoot, stacklevel=2)
                w, z, labels = np.nan, np.nan, None
            else:
                w, z, m = roots[best]
                labels = labels_of(m)
            largest = (float(w), float(z))
    w, z = float(w), float(z)
    zout = bool(np.isfinite(w) and not 0.0 < z <= 1.0)
    if zout:
        warnings.warn(f'the quasiparticle root of {what} {w!r} Ha has Z = {z!r}, outside '
                      '(0, 1]: kept', QPWeightOutside, stacklevel=2)
    flipped = followed is not None and (
        (not followed) or (largest is not None and abs(largest[0] - w) > tol
                           and largest[1] > z))
    if out is not None:
        out.update(labels=labels, largest=largest, followed=followed, flipped=flipped,
                   no_root=not np.isfinite(w), z_outside=zout)
    elif flipped:
        msg = (f'{what}: the branch the previous geometry kept has gone; the root of largest '
               f'weight is kept again, {w:.10f} Ha (Z = {z:.4f}).' if not followed else
               f'{what}: the followed root {w:.10f} Ha has Z = {z:.4f}; the largest weight '
               f'is now {largest[1]:.4f} at {largest[0]:.10f} Ha; the branch is kept.')
        warnings.warn(msg, RuntimeWarning, stacklevel=2)
    return w, z


def qp_energy_sop(p, amplitudes, poles, eps, nocc, xc_correction=0.0, tol=QP_ROOT_TOL,
                  follow=None, branch=None):
    """(eps^QP_p, Z_p) of w = eps_p + xc_correction + Sigma^c(w) on the pole
    model (``sum_over_poles.py:326-346``): Sigma's poles d[s, m] with weights
    A[m, s], labelled s * n_poles + m, by `solve_qp_equation_poles`."""
    num = np.asarray(amplitudes, float).T.ravel()
    pol = pole_denominators(poles, eps, nocc).ravel()
    return solve_qp_equation_poles(num, pol, float(eps[p] + xc_correction), tol=tol,
                                   label=f'orbital {p}', follow=follow, out=branch)
