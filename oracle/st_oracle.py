"""CPU oracle of MBPTcode's space-time ISDF RPA/GW route -- TEST INFRASTRUCTURE.

This module is the checker, never the product: only tests/, the smoke check
and bench.py's CPU-baseline leg may import it. It restates, in FP64 NumPy,
the reference's algorithm for the route, each function citing the reference
file:line it follows (paths inside MBPTcode). Its results are pinned against
golden vectors produced by the reference itself (tests/golden/, generated by
tests/golden/make_golden.py, which imports the reference), so the GPU path is
compared with numbers that the reference computes.

The time/frequency axes come from mbptcode_b200.grids, whose tables and
least-squares transform fits are pinned bitwise to the reference's in the
same fixtures.
"""
from __future__ import annotations

import numpy as np

# reference constants (src/Base/numerics/constants.py)
ISDF_TILE_GB = 4.0                   # :292
BYTES_PER_GB = 1e9                   # :17
QP_GRAPHICAL_TOL = 1e-8              # :272
QP_GRAPHICAL_N_OMEGA = 150           # :273
QP_GRAPHICAL_MAX_BISECTION = 100     # :274
QP_Z_DERIV_STEP = 1e-3               # :276
QP_WINDOW_Z_MIN = 0.5                # :553
QP_SEARCH_WINDOW_TIERS = ((0.0, 0.5), (1.5, 1.0), (4.0, 2.0))   # :1464
QP_SCAN_SECANT_MIN = 0.5             # :1613
QP_SCAN_SPLIT_DEPTH = 6              # :1614
EVGW_MAX_CYCLE, EVGW_TOL = 30, 1e-5  # :187-188
EVGW_DIIS_SIZE, EVGW_DIIS_START = 8, 2   # :197-198


# ---------------------------------------------------------------------------
# chi0 sweep (src/SingleReference/LinearResponse/space_time.py)
# ---------------------------------------------------------------------------

def particle_hole_window(eps, nocc):
    """src/Base/orbital_spaces.py:12-20."""
    eps = np.asarray(eps, float)
    homo, lumo = eps[:nocc].max(), eps[nocc:].min()
    return lumo - homo, eps[nocc:].max() - eps[:nocc].min(), 0.5 * (homo + lumo)


def split_branches(X, eps, nocc, mu=None):
    """space_time.py:448-475: contiguous X_o, X_v and mu-shifted energies."""
    eps = np.asarray(eps, float)
    if mu is None:
        mu = particle_hole_window(eps, nocc)[2]
    X_o = np.ascontiguousarray(X[:, :nocc])
    X_v = np.ascontiguousarray(X[:, nocc:])
    return X_o, X_v, eps[:nocc] - mu, eps[nocc:] - mu, mu


def tile_rows(M, tile_gb, per_row_bytes):
    """space_time.py:413-416."""
    return max(1, min(M, int(tile_gb * BYTES_PER_GB / max(per_row_bytes, 1))))


def polarizability_projected_tau(X_o, X_v, e_o, e_v, D, tau, tile_gb=ISDF_TILE_GB):
    """space_time.py:478-530: proj(tau) = -2 D^T (Go o Gv) D, grid-row tiled."""
    M = X_o.shape[0]
    rows = tile_rows(M, tile_gb, 3 * M * 8)
    out = np.zeros((D.shape[1], D.shape[1]))
    eo_t, ev_t = np.exp(e_o * tau), np.exp(-e_v * tau)
    for p0 in range(0, M, rows):
        p1 = min(p0 + rows, M)
        Go = (X_o[p0:p1] * eo_t) @ X_o.T
        Gv = (X_v[p0:p1] * ev_t) @ X_v.T
        Go *= Gv
        out += D[p0:p1].T @ (Go @ D)
    out *= -2.0
    return out


def polarizability_projected_sweep(X, D, eps, nocc, tau_points, mu=None,
                                   tile_gb=ISDF_TILE_GB):
    """space_time.py:533-560: proj(tau) for every tau, (ntau, naux, naux)."""
    X_o, X_v, e_o, e_v, _ = split_branches(X, eps, nocc, mu)
    return np.stack([polarizability_projected_tau(X_o, X_v, e_o, e_v, D, t, tile_gb)
                     for t in np.asarray(tau_points, float)])


def chi0_imaginary_frequency(X, D, eps, nocc, grid, mu=None, tile_gb=ISDF_TILE_GB):
    """space_time.py:607-651: chi0(i w_f) = sum_tau cosft_wt[f, tau] proj(tau)."""
    X_o, X_v, e_o, e_v, _ = split_branches(X, eps, nocc, mu)
    chi0 = np.zeros((grid.nfreq, D.shape[1], D.shape[1]))
    for k, tau in enumerate(grid.tau_points):
        proj = polarizability_projected_tau(X_o, X_v, e_o, e_v, D, tau, tile_gb)
        chi0 += grid.cosft_wt[:, k, None, None] * proj
    return chi0


def dyson_screening(chi0, correlation=False):
    """space_time.py:956-968: W = [I - chi0]^-1 (minus I when correlation)."""
    W = np.linalg.inv(np.eye(chi0.shape[-1]) - chi0)
    if correlation:
        W[np.diag_indices_from(W)] -= 1.0
    return W


def static_screening_matrix(X, D, eps, nocc, grid, mu=None):
    """space_time.py:1003-1050 on one rank: chi0 on the one-frequency static
    grid (tau addends summed in tau order), then W = [1 - chi0]^-1."""
    return dyson_screening(chi0_imaginary_frequency(X, D, eps, nocc, grid, mu=mu)[0])


def static_screening_matrix_unrestricted(X_mos, D, spectra, noccs, grid):
    """space_time.py:1053-1066 and spin_summed :774-796: half the restricted
    chi0 of each spin (at its own mid-gap) summed, then the Dyson inverse.
    `grid` is the two-spin static grid (transition range of both spins)."""
    chi0 = sum(chi0_imaginary_frequency(X, D, e, n, grid,
                                        mu=particle_hole_window(e, n)[2])[0]
               for X, e, n in zip(X_mos, spectra, noccs))
    return dyson_screening(0.5 * chi0)


def dielectric_log_determinant(one_minus_c, where, flags=None):
    """space_time.py:1073-1097: log|det|, flagging a non-positive determinant."""
    sign, logdet = np.linalg.slogdet(one_minus_c)
    if not sign > 0 and flags is not None:
        flags.setdefault('nonpositive_det', []).append(where)
    return logdet


def rpa_correlation_energy(X, D, eps, nocc, grid, mu=None, flags=None,
                           want_proj=False):
    """space_time.py:1100-1183 (serial, gas phase):
    E_c = (1/2pi) sum_w w_w [log det(I - chi0_w) + tr chi0_w]."""
    proj = polarizability_projected_sweep(X, D, eps, nocc, grid.tau_points, mu)
    blk = np.tensordot(grid.cosft_wt, proj, axes=(1, 0))
    e_c = 0.0
    for k in range(grid.nfreq):
        c = blk[k]
        logdet = dielectric_log_determinant(np.eye(c.shape[0]) - c, k, flags)
        e_c += grid.omega_weights[k] * (logdet + np.trace(c))
    e_c /= 2.0 * np.pi
    return (e_c, proj) if want_proj else e_c


# ---------------------------------------------------------------------------
# screened interaction and self-energy (src/SingleReference/GW/imaginary_time.py)
# ---------------------------------------------------------------------------

def transform_screened(Ctw, W_omega):
    """imaginary_time.py:181-195: Wt(tau) = sum_w Ctw[tau, w] (W(i w) - I)."""
    n = W_omega.shape[-1]
    blk = W_omega.copy()
    blk[(slice(None),) + np.diag_indices(n)] -= 1.0
    return np.tensordot(Ctw, blk, axes=(1, 0))


def sigma_branch_sums(X, D, Wt_tau, eps, nocc, tau_sigma, mu, states):
    """imaginary_time.py:39-92 (SigmaPairs.add, one block pair) over every tau:
    Sigma^<_pp(tau) = sum_PQ X_s[P,p] (Go o Zt)_PQ X_s[Q,p] and
    Sigma^>_pp(tau) = -sum_PQ X_s[P,p] (Gv o Zt)_PQ X_s[Q,p], Zt = D Wt D^T.
    Equal to the MO diagonal of the AO build of :403-533 taken with X_ao = X,
    mo_coeff = I (`sigma_ao_to_mo_diagonal` :581-587). Returns (2, ntau, S)."""
    X_o, X_v, e_o, e_v, _ = split_branches(X, eps, nocc, mu)
    X_s = np.ascontiguousarray(X[:, np.atleast_1d(states)])
    sig = np.zeros((2, len(tau_sigma), X_s.shape[1]))
    for k, tau in enumerate(tau_sigma):
        Zt = (D @ Wt_tau[k]) @ D.T
        G = (X_o * np.exp(e_o * tau)) @ X_o.T
        G *= Zt
        sig[0, k] = np.einsum('Pp,Pp->p', X_s, G @ X_s)
        G = (X_v * np.exp(-e_v * tau)) @ X_v.T
        G *= Zt
        sig[1, k] = -np.einsum('Pp,Pp->p', X_s, G @ X_s)
    return sig


def sigma_frequency(sig, C, S):
    """imaginary_time.py:525-532 / :559-561: Sigma_c(i w_p) =
    -1/2 [C (S> + S<) + i S (S> - S<)], returned as (nstates, npade)."""
    sig_l, sig_g = sig
    return -0.5 * ((sig_g + sig_l).T @ C.T + 1j * ((sig_g - sig_l).T @ S.T))


# ---------------------------------------------------------------------------
# Pade continuation (src/Base/utils/grids/analytic_continuation.py)
# ---------------------------------------------------------------------------

def thiele_coefficients(z, f):
    """analytic_continuation.py:15-22."""
    n = len(z)
    g = np.zeros((n, n), dtype=complex)
    g[:, 0] = f
    for i in range(1, n):
        g[i:, i] = (g[i - 1, i - 1] - g[i:, i - 1]) / ((z[i:] - z[i - 1]) * g[i:, i - 1])
    return g.diagonal().copy()


def pade_eval(zq, z, a):
    """analytic_continuation.py:25-31."""
    r = a[-1] * np.ones_like(np.asarray(zq, dtype=complex))
    for i in range(len(a) - 2, -1, -1):
        r = a[i] / (1.0 + (zq - z[i]) * r)
    return r


def greedy_pade_order(z, f):
    """analytic_continuation.py:34-61."""
    remaining = list(range(len(z)))
    order = [int(np.argmin(np.abs(z)))]
    remaining.remove(order[0])
    while remaining:
        best_j, best = None, np.inf
        for j in remaining:
            trial = order + [j]
            score = abs(thiele_coefficients(z[trial], f[trial])[-1])
            if np.isfinite(score) and score < best:
                best, best_j = score, j
        if best_j is None:
            raise FloatingPointError('greedy Pade ordering: no finite next '
                                     'coefficient')
        order.append(best_j)
        remaining.remove(best_j)
    return np.array(order)


class PadeFit:
    """analytic_continuation.py:64-89 (greedy, all points)."""

    def __init__(self, z, f, greedy=True):
        if greedy:
            o = greedy_pade_order(z, f)
            z, f = z[o], f[o]
        self.z, self.f = z, f
        self.coefficients = thiele_coefficients(z, f)

    def __call__(self, zq):
        return pade_eval(zq, self.z, self.coefficients)


# ---------------------------------------------------------------------------
# QP root finder (src/Solvers/qp_equation.py, sampled equation, no fprime)
# ---------------------------------------------------------------------------

class _Counted:
    def __init__(self, f):
        self.f, self.n = f, 0

    def __call__(self, w):
        self.n += 1
        return self.f(w)


def _search_windows(a):
    """qp_equation.py:1280-1288."""
    tier = 0
    for k, (depth, _) in enumerate(QP_SEARCH_WINDOW_TIERS):
        if abs(a) > depth:
            tier = k
    return [(a - half, a + half) for _, half in QP_SEARCH_WINDOW_TIERS[tier:]]


def _refine_root(func, a, b, tol, max_bisection):
    """qp_equation.py:1319-1333."""
    fa = func(a)
    for _ in range(max_bisection):
        c = 0.5 * (a + b)
        fc = func(c)
        if fa * fc <= 0.0:
            b = c
        else:
            a, fa = c, fc
        if abs(b - a) <= tol:
            break
    return 0.5 * (a + b)


def pole_strength(func, w, h=QP_Z_DERIV_STEP):
    """qp_equation.py:1336-1350."""
    d = (func(w + h) - func(w - h)) / (2.0 * h)
    if d == 0.0 or not np.isfinite(d):
        return np.nan
    return 1.0 / d


def _cells(func, l, r, fl, fr, depth):
    """qp_equation.py:1256-1271 (no refusals)."""
    if fl * fr < 0.0:
        return [(l, r, fl, fr)]
    if depth == 0 or fl == 0.0 or fr == 0.0 or not (fr - fl < QP_SCAN_SECANT_MIN * (r - l)):
        return []
    m = 0.5 * (l + r)
    fm = float(func(m))
    return _cells(func, l, m, fl, fm, depth - 1) + _cells(func, m, r, fm, fr, depth - 1)


def _solve_bracket(func, bracket):
    """qp_equation.py:1138-1157 with fprime None and positive_weight False."""
    l, r, fl, fr = bracket
    if l == r:
        return [(float(l), float(pole_strength(func, l)))]
    w = _refine_root(func, r, l, QP_GRAPHICAL_TOL, QP_GRAPHICAL_MAX_BISECTION)
    fw = float(func(w))
    if not abs(fw) <= max(abs(fl), abs(fr)):
        return []
    return [(float(w), float(pole_strength(func, w)))]


def _valid(z, z_min=0.0):
    """qp_equation.py:85-94 (`quasiparticle_weight`)."""
    z = float(z)
    return bool(np.isfinite(z) and z_min < z <= 1.0)


def _select(found):
    """qp_equation.py:97-109 with z_min 0 and no `near`."""
    ok = [i for i, (_, z) in enumerate(found) if _valid(z)]
    if not ok:
        return None
    return max(ok, key=lambda i: found[i][1])


def solve_qp_equation_pole_strength(func, a):
    """qp_equation.py:1353-1393 -> find_qp_root :155-232 -> _largest_root
    :236-268 -> _weighed_roots :277-305 on a SampledEquation :1029-1271
    (every bracket of a window is refined: its Z bounds are all infinite).

    Returns (root, Z, quasiparticle)."""
    found, k = [], None
    windows = _search_windows(a)
    for lo, hi in windows:
        grid = np.linspace(lo, hi, QP_GRAPHICAL_N_OMEGA)
        f = np.array([func(w) for w in grid])
        brackets = []
        for i in range(1, grid.size):
            brackets += _cells(func, grid[i - 1], grid[i], f[i - 1], f[i],
                               QP_SCAN_SPLIT_DEPTH)
        found = []
        for br in brackets:
            found += _solve_bracket(func, br)
        k = _select(found)
        if k is not None and _valid(found[k][1], QP_WINDOW_Z_MIN):
            return found[k][0], found[k][1], True
    if not found:
        return np.nan, np.nan, False
    if k is None:
        k = min(range(len(found)), key=lambda i: abs(found[i][0] - a))
    return found[k][0], found[k][1], False


def imaginary_axis_sample_points(freq_points, nocc, p, mu):
    """GW/qp_solve.py:698-703."""
    sign = -1.0 if p < nocc else 1.0
    return mu + 1j * sign * np.asarray(freq_points)


def solve_qp_from_imaginary_axis(eps_p, xc, z_fit, sigma_iw, greedy=True,
                                 counter=None):
    """GW/qp_solve.py:529-558: Pade-continue Sigma_c and solve
    w = eps_p + xc + Re Sigma_c(w) for the root of largest Z."""
    fit = PadeFit(z_fit, sigma_iw, greedy=greedy)

    def residual(w):
        return w - eps_p - xc - fit(np.array([w], dtype=complex))[0].real
    func = _Counted(residual)
    root, z, qp = solve_qp_equation_pole_strength(func, eps_p)
    if counter is not None:
        counter.append(func.n)
    return root, z, fit


def finish_qp(sigma, eps, nocc, states, mu, pade_freq, xc_diag=None,
              greedy=True, counts=None):
    """GW/qp_solve.py:575-695 on a restricted gas-phase reference with the
    static term handed in (xc_diagonal; 0 for an HF reference, :311).
    sigma (nstates, npade) on the positive branch; occupied states take the
    conjugate (:659). Returns (roots, Z)."""
    states = np.atleast_1d(states)
    xc = np.zeros(len(states)) if xc_diag is None else np.asarray(xc_diag, float)
    roots, zs = np.empty(len(states)), np.empty(len(states))
    for i, p in enumerate(states):
        z_fit = imaginary_axis_sample_points(pade_freq, nocc, int(p), mu)
        s_p = np.conj(sigma[i]) if p < nocc else sigma[i]
        roots[i], zs[i], _ = solve_qp_from_imaginary_axis(
            float(eps[p]), xc[i], z_fit, s_p, greedy=greedy, counter=counts)
    return roots, zs


# ---------------------------------------------------------------------------
# the route (src/SingleReference/GW/space_time.py:768-863, serial restricted)
# ---------------------------------------------------------------------------

def gw_space_time(X, D, eps, nocc, states, axes, eps_anchor=None, xc_diag=None,
                  timings=None, counts=None):
    """chi0 -> Dyson -> Wt(tau) -> Sigma_c diagonal -> QP roots, on the axes
    `axes` (mbptcode_b200.grids.space_time_axes). Returns a dict with chi0,
    W_minus_I, Wt, sigma (nstates, npade), roots and Z."""
    import time
    eps = np.asarray(eps, float)
    mu = axes.mu
    t0 = time.perf_counter()
    chi0 = chi0_imaginary_frequency(X, D, eps, nocc, axes.grid, mu)
    t1 = time.perf_counter()
    W = np.stack([dyson_screening(c, correlation=True) for c in chi0])
    t2 = time.perf_counter()
    Wt = np.tensordot(axes.Ctw, W, axes=(1, 0))
    sig = sigma_branch_sums(X, D, Wt, eps, nocc, axes.tau_sigma, mu, states)
    sigma = sigma_frequency(sig, axes.C, axes.S)
    t3 = time.perf_counter()
    anchor = eps if eps_anchor is None else np.asarray(eps_anchor, float)
    roots, z = finish_qp(sigma, anchor, nocc, states, mu, axes.pade_freq,
                         xc_diag, counts=counts)
    t4 = time.perf_counter()
    if timings is not None:
        timings.update(t_chi0=t1 - t0, t_dyson=t2 - t1, t_sigma=t3 - t2,
                       t_qp=t4 - t3)
    return {'chi0': chi0, 'W_minus_I': W, 'Wt': Wt, 'branch': sig,
            'sigma': sigma, 'roots': roots, 'z': z}


def gw_space_time_unrestricted(X_mos, D, spectra, noccs, states, axes):
    """GW/space_time.py:866-1009 (serial): chi0 = half of each spin's
    restricted chi0 at its own mid-gap (space_time.py:774-796), one W, then
    per channel the restricted Sigma sweep on that channel's orbitals and its
    QP roots sampled through the channel's mid-gap. `axes`: the two-spin axes
    (mbptcode_b200.grids.space_time_axes_unrestricted; axes.mu per channel).
    states: per channel. Returns {'W_minus_I', 'sigma': [..], 'roots': [..],
    'z': [..]}."""
    chi0 = 0.5 * sum(chi0_imaginary_frequency(X, D, np.asarray(e, float), n, axes.grid, m)
                     for X, e, n, m in zip(X_mos, spectra, noccs, axes.mu))
    W = np.stack([dyson_screening(c, correlation=True) for c in chi0])
    Wt = np.tensordot(axes.Ctw, W, axes=(1, 0))
    out = {'W_minus_I': W, 'sigma': [], 'roots': [], 'z': []}
    for X, e, n, m, st in zip(X_mos, spectra, noccs, axes.mu, states):
        e = np.asarray(e, float)
        sig = sigma_branch_sums(X, D, Wt, e, n, axes.tau_sigma, m, st)
        sigma = sigma_frequency(sig, axes.C, axes.S)
        roots, z = finish_qp(sigma, e, n, st, m, axes.pade_freq)
        for k, v in (('sigma', sigma), ('roots', roots), ('z', z)):
            out[k].append(v)
    return out


# ---------------------------------------------------------------------------
# dRPA adjoint (src/gradients/rpa/space_time_adjoint.py:136-218, 473-563)
# ---------------------------------------------------------------------------

def polarizability_backward(proj_bar, X, D, eps, nocc, tau_points, mu=None):
    """space_time_adjoint.py:167-218 with one row tile: the reverse of the
    chi0 sweep, G(tau) recomputed per tau."""
    X_o, X_v, e_o, e_v, _ = split_branches(X, eps, nocc, mu)
    eps_bar = np.zeros(len(eps))
    X_bar = np.zeros_like(X)
    D_bar = np.zeros_like(D)
    for k, tau in enumerate(tau_points):
        pb = 0.5 * (proj_bar[k] + proj_bar[k].T)
        E = -2.0 * (D @ pb)
        w, u = np.exp(e_o * tau), np.exp(-e_v * tau)
        Go = (X_o * w) @ X_o.T
        Gv = (X_v * u) @ X_v.T
        Pi = Go * Gv
        D_bar += 2.0 * (Pi @ E)
        Pi_bar = E @ D.T
        GoX = (Pi_bar * Gv) @ X_o
        GvX = (Pi_bar * Go) @ X_v
        X_bar[:, :nocc] += 2.0 * GoX * w
        X_bar[:, nocc:] += 2.0 * GvX * u
        eps_bar[:nocc] += tau * w * np.einsum('bi,bi->i', X_o, GoX)
        eps_bar[nocc:] -= tau * u * np.einsum('ba,ba->a', X_v, GvX)
    return eps_bar, X_bar, D_bar


# ---------------------------------------------------------------------------
# self-energy diagonal in the auxiliary basis and its reverse
# (GW/imaginary_time.py:632-661, 731-768; space_time_adjoint.py:593-691, 795-875)
# ---------------------------------------------------------------------------

def three_index_slice(X, D, p):
    """LinearResponse/space_time.py:804-815: B_p[P, q] = sum_k D[k,P] X[k,p] X[k,q]."""
    return D.T @ (X[:, p:p + 1] * X)


def screened_interaction_tau(proj_tau, grid, Ctw):
    """Wt(tau) = sum_w Ctw[tau, w] ([1 - chi0_w]^-1 - I), chi0 from proj(tau)."""
    chi0 = np.tensordot(grid.cosft_wt, proj_tau, axes=(1, 0))
    W = np.stack([dyson_screening(c, correlation=True) for c in chi0])
    return np.tensordot(Ctw, W, axes=(1, 0))


def selfenergy_diag(X, D, eps, nocc, grid, states, transforms, mu):
    """GW/imaginary_time.py:731-768 (serial): Sigma^c_pp(i omega_out) and the
    cache (proj_tau, Wt_tau, Bs), from the states' three-index slices."""
    Ctw, C, S = transforms
    eps = np.asarray(eps, float)
    _, _, e_o, e_v, _ = split_branches(X, eps, nocc, mu)
    proj = polarizability_projected_sweep(X, D, eps, nocc, grid.tau_points, mu)
    Wt = screened_interaction_tau(proj, grid, Ctw)
    states = np.atleast_1d(states)
    Bs = np.stack([three_index_slice(X, D, int(p)) for p in states])
    sig_l = np.zeros((len(grid.tau_points), len(states)))
    sig_g = np.zeros_like(sig_l)
    for k, tau in enumerate(grid.tau_points):
        w, u = np.exp(e_o * tau), np.exp(-e_v * tau)
        for s in range(len(states)):
            bYb = np.einsum('Pq,Pq->q', Bs[s], Wt[k] @ Bs[s])
            sig_l[k, s] = bYb[:nocc] @ w
            sig_g[k, s] = -(bYb[nocc:] @ u)
    sigma = -0.5 * ((sig_g + sig_l).T @ C.T + 1j * ((sig_g - sig_l).T @ S.T))
    return sigma, (proj, Wt, Bs)


def screened_interaction_tau_backward(Wt_bar, proj_tau, grid, Ctw):
    """space_time_adjoint.py:652-691 (serial): chi0_bar = W W_bar W per
    frequency, W rebuilt from proj(tau), folded back onto tau."""
    chi0 = np.tensordot(grid.cosft_wt, proj_tau, axes=(1, 0))
    Wbar = np.tensordot(Ctw, Wt_bar, axes=(0, 0))
    eye = np.eye(chi0.shape[-1])
    for f in range(len(chi0)):
        Wf = np.linalg.inv(eye - chi0[f])
        Wbar[f] = Wf @ Wbar[f] @ Wf
    return np.tensordot(grid.cosft_wt.T, Wbar, axes=(1, 0))


def three_index_slice_backward(X, D, p, Bp_bar, X_bar, D_bar):
    """space_time_adjoint.py:593-624 with one row tile, accumulating."""
    xp = X[:, p, None]
    G = D @ Bp_bar
    term = xp * G
    term[:, p] += np.einsum('kq,kq->k', G, X)
    X_bar += term
    D_bar += xp * (X @ Bp_bar.T)


def selfenergy_diag_backward(a_re, a_im, X, D, eps, nocc, grid, states, transforms, mu,
                             cache):
    """space_time_adjoint.py:795-875 (serial): (eps_bar, X_bar, D_bar) of
    sum a_re Re Sigma + a_im Im Sigma."""
    Ctw, C, S = transforms
    eps = np.asarray(eps, float)
    _, _, e_o, e_v, _ = split_branches(X, eps, nocc, mu)
    proj, Wt, Bs = cache
    states = np.atleast_1d(states)
    ac, bs = a_re @ C, a_im @ S
    sg_bar = -0.5 * (ac + bs).T
    sl_bar = -0.5 * (ac - bs).T
    eps_bar = np.zeros_like(eps)
    Bs_bar = np.zeros_like(Bs)
    Wt_bar = np.zeros_like(Wt)
    c = np.empty(X.shape[1])
    for k, tau in enumerate(grid.tau_points):
        w, u = np.exp(e_o * tau), np.exp(-e_v * tau)
        for s in range(len(states)):
            b = Bs[s]
            Y = Wt[k] @ b
            c[:nocc] = sl_bar[k, s] * w
            c[nocc:] = -sg_bar[k, s] * u
            Bs_bar[s] += 2.0 * Y * c
            Wt_bar[k] += (b * c) @ b.T
            bYb = np.einsum('Pq,Pq->q', b, Y)
            eps_bar[:nocc] += sl_bar[k, s] * tau * w * bYb[:nocc]
            eps_bar[nocc:] += sg_bar[k, s] * tau * u * bYb[nocc:]
    proj_bar = screened_interaction_tau_backward(Wt_bar, proj, grid, Ctw)
    eps2, X_bar, D_bar = polarizability_backward(proj_bar, X, D, eps, nocc, grid.tau_points,
                                                 mu)
    for s, p in enumerate(states):
        three_index_slice_backward(X, D, int(p), Bs_bar[s], X_bar, D_bar)
    return eps_bar + eps2, X_bar, D_bar


def rpa_energy_and_adjoint(X, D, eps, nocc, grid, mu=None):
    """space_time_adjoint.py:473-563, gas phase: (E_c, eps_bar, X_bar, D_bar)."""
    e_c, proj = rpa_correlation_energy(X, D, eps, nocc, grid, mu, want_proj=True)
    blk = np.tensordot(grid.cosft_wt, proj, axes=(1, 0))
    eye = np.eye(proj.shape[-1])
    for k in range(grid.nfreq):
        scale = grid.omega_weights[k] / (2.0 * np.pi)
        blk[k] = scale * (eye - np.linalg.inv(eye - blk[k]).T)
    proj_bar = np.tensordot(grid.cosft_wt, blk, axes=(0, 0))
    eps_bar, X_bar, D_bar = polarizability_backward(proj_bar, X, D, eps, nocc,
                                                    grid.tau_points, mu)
    return e_c, eps_bar, X_bar, D_bar


# ---------------------------------------------------------------------------
# evGW (src/SingleReference/GW/evGW.py:78-229) with Pulay DIIS
# ---------------------------------------------------------------------------

class PulayDIIS:
    """Pulay's direct inversion in the iterative subspace (Chem. Phys. Lett.
    73, 393 (1980)): the iterate that minimises the norm of the linearly
    combined residuals under sum c = 1. Before `start` updates it passes the
    iterate through; it keeps the last `size` pairs. This follows the
    schedule the reference's evGW loop drives (evGW.py:181, 209-210)."""

    def __init__(self, size, start):
        self.size, self.start, self.seen = size, start, 0
        self.vecs, self.errs = [], []

    def update(self, vec, err):
        if self.seen < self.start:
            self.seen += 1
            return vec
        self.seen += 1
        self.vecs.append(np.array(vec, float))
        self.errs.append(np.array(err, float))
        if len(self.vecs) > self.size:
            self.vecs.pop(0)
            self.errs.pop(0)
        n = len(self.vecs)
        B = np.zeros((n + 1, n + 1))
        B[:n, :n] = [[e1 @ e2 for e2 in self.errs] for e1 in self.errs]
        B[n, :n] = B[:n, n] = -1.0
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        c = np.linalg.solve(B, rhs)[:n]
        return sum(ci * v for ci, v in zip(c, self.vecs))


def evgw(X, D, eps0, nocc, ntau, tol=EVGW_TOL, max_cycle=EVGW_MAX_CYCLE,
         diis_size=EVGW_DIIS_SIZE, diis_start=EVGW_DIIS_START, counts=None):
    """evGW.py:78-229 restricted, every orbital updated, screening 'updated':
    each cycle builds G, chi0 and W from the iterate, anchors the equation on
    eps0 (GW/space_time.py:706-712) and converges on HOMO/LUMO."""
    from mbptcode_b200.grids import space_time_axes
    eps0 = np.asarray(eps0, float)
    n = len(eps0)
    tested = [nocc - 1, nocc]
    eps = eps0.copy()
    acc = PulayDIIS(diis_size, diis_start) if diis_size else None
    history = []
    converged = False
    for _ in range(max_cycle):
        axes = space_time_axes(eps, nocc, ntau=ntau, anchor=eps0)
        out = gw_space_time(X, D, eps, nocc, np.arange(n), axes,
                            eps_anchor=eps0, counts=counts)
        eps_new = out['roots']
        res = eps_new - eps
        delta = float(np.abs(res[tested]).max())
        history.append(delta)
        if delta < tol:
            eps = eps_new
            converged = True
            break
        eps = acc.update(eps_new, res) if acc is not None else eps_new
    return eps, {'cycles': len(history), 'converged': converged,
                 'history': history}


# ---------------------------------------------------------------------------
# contour deformation (src/SingleReference/GW/contour_deformation.py,
# GW/real_screening.py): the imaginary-axis screening contraction, the
# Laplace real-frequency screening and Sigma^c(omega)
# ---------------------------------------------------------------------------

def cd_integral_weights(de, nu, wt, on_contour_tol=1e-10, with_slope=False):
    """contour_deformation.py:150-202: quadrature weights of the Lorentzian
    with its singular part (wc(0) times de/(de^2+nu^2) a^2/(a^2+nu^2))
    integrated in closed form; wc(0) from the two smallest nodes. With
    with_slope also their derivative in de."""
    de, nu, wt = (np.asarray(a, float) for a in (de, nu, wt))
    den = de[None, :] ** 2 + nu[:, None] ** 2
    g = de[None, :] / den
    dg = (nu[:, None] ** 2 - de[None, :] ** 2) / den ** 2
    c, dc = wt[:, None] * g, wt[:, None] * dg
    order = np.argsort(nu)
    k1, k2 = order[0], order[1]
    n1, n2 = nu[k1] ** 2, nu[k2] ** 2
    a = 4.0 * float(np.median(nu))
    h = wt * a * a / (a * a + nu ** 2)
    side = np.where(np.abs(de) < on_contour_tol, 0.0, np.sign(de))
    err = 0.5 * np.pi * side * a / (a + np.abs(de)) - h @ g
    derr = -0.5 * np.pi * a / (a + np.abs(de)) ** 2 - h @ dg
    for k, coef in ((k1, n2 / (n2 - n1)), (k2, -n1 / (n2 - n1))):
        c[k] += coef * err
        dc[k] += coef * derr
    return (c, dc) if with_slope else c


def cd_screening_contraction(proj_tau, cosft_wt, Bps):
    """contour_deformation.py:248-290 (serial): per frequency chi0 =
    cosft_wt proj(tau), W B - B by a solve, wc[k, q] = B[:,q].(W B - B)[:,q]."""
    chi0 = np.tensordot(cosft_wt, proj_tau, axes=(1, 0))
    eye = np.eye(chi0.shape[-1])
    out = [np.zeros((len(chi0), B.shape[1])) for B in Bps]
    for k in range(len(chi0)):
        for wc, B in zip(out, Bps):
            wc[k] = np.einsum('Pq,Pq->q', B, np.linalg.solve(eye - chi0[k], B) - B)
    return out


def residue_set(eps, nocc, omega, tol=1e-10):
    """real_screening.py:157-168."""
    out = []
    for q, e in enumerate(eps):
        gap = e - omega
        if abs(gap) < tol:
            out.append((q, -0.5 if q < nocc else 0.5))
        elif q < nocc and gap > 0.0:
            out.append((q, -1.0))
        elif q >= nocc and gap < 0.0:
            out.append((q, 1.0))
    return out


class LaplaceRefused(ValueError):
    """real_screening.py:128-146: a real frequency the time grid's bare
    quadrature does not carry (error of y sum w e^{-y tau} = 1 above 1e-8
    on y = d -+ freq, LinearResponse/space_time.py:908-931)."""


def laplace_check(eps, nocc, tau, tau_w, freq, tol=1e-8, pair_energies=None):
    eps = np.asarray(eps, float)
    d = (ov_energies(eps, nocc) if pair_energies is None
         else np.asarray(pair_energies, float))
    y = np.concatenate([d - freq, d + freq])
    if y.min() <= 0.0 or not float(np.abs(
            (np.exp(-np.outer(y, tau)) @ tau_w) * y - 1.0).max()) < tol:
        raise LaplaceRefused(freq)


def laplace_screening_slope(proj_tau, tau, tau_w, freq, y):
    """real_screening.py:152-154: y^T [sum_k 2 w_k tau_k sinh(freq tau_k)
    proj(tau_k)] y."""
    dc = 2.0 * np.asarray(tau_w) * np.asarray(tau) * np.sinh(freq * np.asarray(tau))
    return float(y @ np.tensordot(dc, proj_tau, axes=(0, 0)) @ y)


def sigma_cd_slope(p, omega, Bp, eps, nocc, nu, nu_w, wc, proj_tau, tau, tau_w,
                   pair_energies=None):
    """contour_deformation.py:346-373 with the Laplace residue backend (the
    representability check of real_screening.py:132-145 on each frequency;
    pair_energies: both spins' of an unrestricted reference)."""
    eps = np.asarray(eps, float)
    _, dc = cd_integral_weights(omega - eps, nu, nu_w, with_slope=True)
    slope = -float(np.einsum('kq,kq->', dc, wc)) / np.pi
    for q, weight in residue_set(eps, nocc, omega):
        gap = eps[q] - omega
        freq = abs(gap)
        laplace_check(eps, nocc, tau, tau_w, freq, pair_energies=pair_energies)
        y = laplace_screening_apply(proj_tau, tau, tau_w, freq, Bp[:, q])
        slope -= weight * laplace_screening_slope(proj_tau, tau, tau_w, freq, y) * np.sign(gap)
    return slope


def laplace_screening_apply(proj_tau, tau, tau_w, freq, b):
    """real_screening.py:147-150 with :184-209: W(freq) b, chi0(freq) =
    sum_k 2 w_k cosh(freq tau_k) proj(tau_k), below the gap."""
    c = 2.0 * np.asarray(tau_w) * np.cosh(freq * np.asarray(tau))
    chi0 = np.tensordot(c, proj_tau, axes=(0, 0))
    return np.linalg.solve(np.eye(chi0.shape[0]) - chi0, b)


def sigma_cd(p, omega, Bp, eps, nocc, nu, nu_w, wc, proj_tau, tau, tau_w, pair_energies=None):
    """contour_deformation.py:310-343 with the Laplace residue backend."""
    eps = np.asarray(eps, float)
    c = cd_integral_weights(omega - eps, nu, nu_w)
    s = -float(np.einsum('kq,kq->', c, wc)) / np.pi
    for q, weight in residue_set(eps, nocc, omega):
        b = Bp[:, q]
        laplace_check(eps, nocc, tau, tau_w, abs(eps[q] - omega), pair_energies=pair_energies)
        y = laplace_screening_apply(proj_tau, tau, tau_w, abs(eps[q] - omega), b)
        s += weight * (b @ y - b @ b)
    return s


# the explicit particle-hole backend of continuation 'cd'

def frequency_factor(d, w, imaginary, eta=0.0, slopes=False):
    """LinearResponse/imaginary_frequency.py:25-59: the bubble's frequency
    factor for pair energies d at w, (f, df/dd, df/dw) with slopes. Imaginary
    axis -2d/(d^2 + w^2); real axis 1/(w - d) - 1/(w + d), broadened by eta."""
    d = np.asarray(d, float)
    if imaginary:
        den = d * d + w * w
        f = -2.0 * d / den
        return (f, -2.0 * (w * w - d * d) / den ** 2, None) if slopes else f
    a, b = w - d, w + d
    if eta == 0.0:
        f = 1.0 / a - 1.0 / b
        return (f, 1.0 / a ** 2 + 1.0 / b ** 2, -1.0 / a ** 2 + 1.0 / b ** 2) if slopes else f
    da, db = a * a + eta * eta, b * b + eta * eta
    f = a / da - b / db
    if not slopes:
        return f
    return (f, (a * a - eta * eta) / da ** 2 + (b * b - eta * eta) / db ** 2,
            (eta * eta - a * a) / da ** 2 - (eta * eta - b * b) / db ** 2)


def ov_energies(eps, nocc):
    """Base/orbital_spaces.py:31-34: d[(i, a)] = eps_a - eps_i, i major."""
    eps = np.asarray(eps, float)
    return (eps[nocc:][None, :] - eps[:nocc][:, None]).ravel()


def three_index_ov(X, D, eps, nocc):
    """LinearResponse/space_time.py:833-851: C_ov[P, (i, a)] =
    sum_k D[k, P] X[k, i] X[k, a], (naux, nocc * nvirt)."""
    Xo, Xv = X[:, :nocc], X[:, nocc:]
    return D.T @ (Xo[:, :, None] * Xv[:, None, :]).reshape(X.shape[0], -1)


def explicit_screening_apply(C_ov, d, freq, b, eta=0.0, imaginary=False):
    """real_screening.py:84-85 with :171-181: W(freq) b, W = [1 - chi0]^-1,
    chi0 = 2 (C_ov f) C_ov^T -- by a solve (the reference inverts)."""
    chi0 = 2.0 * (C_ov * frequency_factor(d, freq, imaginary, eta)) @ C_ov.T
    return np.linalg.solve(np.eye(len(chi0)) - chi0, b)


def explicit_screening_slope(C_ov, d, freq, y, eta=0.0):
    """real_screening.py:87-91: y^T [dchi0/dfreq] y = 2 sum df/dw (C_ov^T y)^2."""
    z = C_ov.T @ y
    return 2.0 * float(frequency_factor(d, freq, False, eta, slopes=True)[2] @ z ** 2)


def wc_explicit(Bp, C_ov, d, nu):
    """contour_deformation.py:240-245: wc[k, q] = B[:, q]^T (W(i nu_k) - I)
    B[:, q] from the explicit imaginary-axis screening."""
    out = np.zeros((len(nu), Bp.shape[1]))
    for k, v in enumerate(nu):
        out[k] = np.einsum('Pq,Pq->q', Bp, explicit_screening_apply(C_ov, d, v, Bp,
                                                                    imaginary=True) - Bp)
    return out


def sigma_cd_explicit(p, omega, Bp, eps, nocc, nu, nu_w, wc, C_ov, eta=0.0,
                      pair_energies=None):
    """contour_deformation.py:310-343 with the explicit residue backend."""
    eps = np.asarray(eps, float)
    d = ov_energies(eps, nocc) if pair_energies is None else np.asarray(pair_energies, float)
    c = cd_integral_weights(omega - eps, nu, nu_w)
    s = -float(np.einsum('kq,kq->', c, wc)) / np.pi
    for q, weight in residue_set(eps, nocc, omega):
        b = Bp[:, q]
        y = explicit_screening_apply(C_ov, d, abs(eps[q] - omega), b, eta)
        s += weight * (b @ y - b @ b)
    return s


def sigma_cd_slope_explicit(p, omega, Bp, eps, nocc, nu, nu_w, wc, C_ov, eta=0.0,
                            pair_energies=None):
    """contour_deformation.py:346-373 with the explicit residue backend."""
    eps = np.asarray(eps, float)
    d = ov_energies(eps, nocc) if pair_energies is None else np.asarray(pair_energies, float)
    _, dc = cd_integral_weights(omega - eps, nu, nu_w, with_slope=True)
    slope = -float(np.einsum('kq,kq->', dc, wc)) / np.pi
    for q, weight in residue_set(eps, nocc, omega):
        gap = eps[q] - omega
        y = explicit_screening_apply(C_ov, d, abs(gap), Bp[:, q], eta)
        slope -= weight * explicit_screening_slope(C_ov, d, abs(gap), y, eta) * np.sign(gap)
    return slope


def self_energy_matrix(X_ao, D, W_omega, mo_coeff, eps, nocc, tau_points, omega_in, omega_out,
                       mu, tau_indices=None):
    """GW/imaginary_time.py:403-533 in one block: the full AO Sigma^c(i w_out),
    G from the MO collocation X_ao mo_coeff, the outer indices AO."""
    from mbptcode_b200.grids import (COSINE_TW, COSINE_WT, SINE_TW, sigma_fit_ranges,
                                     transform_weights)
    eps = np.asarray(eps, float)
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    Ctw = transform_weights(COSINE_WT, tau_points, omega_in, *rW, warn=False)[0]
    C = transform_weights(COSINE_TW, tau_points, omega_out, *rS, warn=False)[0]
    S = transform_weights(SINE_TW, tau_points, omega_out, *rS, warn=False)[0]
    Wt = transform_screened(Ctw, W_omega)
    X_mo = X_ao @ mo_coeff
    X_o, X_v = X_mo[:, :nocc], X_mo[:, nocc:]
    e_o, e_v = eps[:nocc] - mu, eps[nocc:] - mu
    nao = X_ao.shape[1]
    out = np.zeros((len(omega_out), nao, nao), dtype=complex)
    which = range(len(tau_points)) if tau_indices is None else tau_indices
    for k in which:
        tau = tau_points[k]
        Zt = (D @ Wt[k]) @ D.T
        s_l = X_ao.T @ (((X_o * np.exp(e_o * tau)) @ X_o.T) * Zt) @ X_ao
        s_g = -X_ao.T @ (((X_v * np.exp(-e_v * tau)) @ X_v.T) * Zt) @ X_ao
        for w in range(len(omega_out)):
            out.real[w] += C[w, k] * (s_g + s_l)
            out.imag[w] += S[w, k] * (s_g - s_l)
    return -0.5 * out


def qp_gradient_laplace(X, D, eps, nocc, tau, tau_w, cosft_wt, nu, nu_w, p, mu, root, z):
    """gradients/gwbse/qp_space_time.py:412-452 for one state on the Laplace
    residue route, given its root and Z: (eps_bar, X_bar, D_bar) of
    eps^QP_p = Z [d eps_p + dSigma^c(w)|_w] (implicit differentiation, the
    residue set frozen at the root), with
      the integral term's adjoint on wc (-Z/pi c) carried to B_p (2 (W-I) B
      wc_bar), to W(i nu) (B diag(wc_bar) B^T, then W W_bar W onto chi0 and
      proj(tau)) and to eps through the weights' de-derivative
      (contour_deformation_adjoint.py, qp_space_time.py:328-361);
      each residue's adjoint on b_q (2 w_q (y - b)), its rank-one adjoint
      w_q y y^T on chi0 at the real frequency folded onto proj(tau) by the
      cosh weights, and the frequency's eps dependence through the slope;
      then the chi0 sweep's reverse and the slice's (:593-624)."""
    eps = np.asarray(eps, float)
    proj = polarizability_projected_sweep(X, D, eps, nocc, tau, mu)
    chi0 = np.tensordot(cosft_wt, proj, axes=(1, 0))
    naux = proj.shape[-1]
    eye = np.eye(naux)
    B = three_index_slice(X, D, p)
    eps_bar = np.zeros_like(eps)
    eps_bar[p] += z
    c, dc = cd_integral_weights(root - eps, nu, nu_w, with_slope=True)
    coeff = -z / np.pi
    B_bar = np.zeros_like(B)
    chi0_bar = np.zeros_like(chi0)
    for k in range(len(chi0)):
        Wm = np.linalg.inv(eye - chi0[k]) - eye
        Y = Wm @ B
        wck = np.einsum('Pq,Pq->q', B, Y)
        wcb = coeff * c[k]
        B_bar += 2.0 * Y * wcb
        Wk = eye + Wm
        chi0_bar[k] = Wk @ ((B * wcb) @ B.T) @ Wk
        eps_bar += -coeff * wck * dc[k]
    proj_bar = np.tensordot(cosft_wt.T, chi0_bar, axes=(1, 0))
    for q, wt in residue_set(eps, nocc, root):
        f = abs(eps[q] - root)
        cf = 2.0 * np.asarray(tau_w) * np.cosh(f * np.asarray(tau))
        dcf = 2.0 * np.asarray(tau_w) * np.asarray(tau) * np.sinh(f * np.asarray(tau))
        b = B[:, q]
        y = np.linalg.solve(eye - np.tensordot(cf, proj, axes=(0, 0)), b)
        B_bar[:, q] += z * wt * 2.0 * (y - b)
        proj_bar += (z * wt) * cf[:, None, None] * np.outer(y, y)[None]
        slope = float(y @ np.tensordot(dcf, proj, axes=(0, 0)) @ y)
        eps_bar[q] += z * wt * slope * np.sign(eps[q] - root)
    e2, X_bar, D_bar = polarizability_backward(proj_bar, X, D, eps, nocc, tau, mu)
    three_index_slice_backward(X, D, p, B_bar, X_bar, D_bar)
    return eps_bar + e2, X_bar, D_bar


# ---------------------------------------------------------------------------
# separable-RI fit from supplied inputs (src/Base/factorization/separable_ri.py)
# ---------------------------------------------------------------------------

def isdf_fit_products(ao, second, w, aux, FD, regularization=4e-7):
    """separable_ri.py:664-900 with explicit arrays: the Gram matrix of the
    product pairs and auxiliary functions, balanced by its diagonal,
    regularised, solved by Cholesky against F D^T (separable_ri.py:1616-1653)."""
    import scipy.linalg
    B = ao[:, second] * w[None, :]
    S = (ao @ ao.T) * (B @ B.T) + aux @ aux.T
    scale = np.sqrt(np.diag(S))
    scale[scale == 0] = 1.0
    d = 1.0 / scale
    G = S * d[:, None] * d[None, :]
    G[np.diag_indices_from(G)] += regularization
    cho = scipy.linalg.cho_factor(G, lower=True)
    return scipy.linalg.cho_solve(cho, (FD * d[None, :]).T).T * d[None, :]


def aux_metric_root(V, floor=1e-12):
    """separable_ri.py:1802-1929: V^(1/2) on the eigenvalues above floor x max."""
    w, v = np.linalg.eigh(V)
    keep = w > floor * w.max()
    return (v[:, keep] * np.sqrt(w[keep])) @ v[:, keep].T
