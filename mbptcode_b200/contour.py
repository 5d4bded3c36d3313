"""Contour-deformation correlation self-energy on the B200.

Keeps the kernel seams of MBPTcode's ``src/SingleReference/GW/contour_deformation.py``
and ``GW/real_screening.py`` (names, arguments, the residue backends'
apply/slope protocol, refusals) on a design of its own:

    Sigma^c_pp(omega) = Sigma^int + Sigma^res,
    Sigma^int = -(1/pi) sum_kq c[k, q](omega) wc[k, q],
    wc[k, q]  = B_p[:, q]^T (W(i nu_k) - I) B_p[:, q],
    Sigma^res = sum_q r_q(omega) (b_q^T W(|eps_q - omega|) b_q - b_q^T b_q),

B_p = D^T diag(X[:, p]) X the state's three-index slice, W = [1 - chi0]^-1,
c the Gauss-Legendre weights of the Lorentzian kernel with its singular part
integrated in closed form, r_q the residue weights of the poles of G the
deformation sweeps.

The quasiparticle equation w = eps_p + xc + Sigma^c(w) is solved for every
requested state at once. The search follows the reference's rules (windows
narrowest first, the 150-point grid walked outward from the bare level,
cells halved where the secant slope hides a pole, brackets refined by Newton
on the closed-form slope inside the bracket, the walk ended by the weight
sum, the root of largest Z kept), but it runs as a lockstep over states and
cells: each round gathers every (state, frequency) point the search needs --
a wave of grid cells, one level of halving, one Newton step of every open
bracket -- and evaluates them in one device call. The walk is then replayed
in the reference's order, so the roots are the ones its sequential scan
finds; points of a wave beyond where a walk stops are evaluated and dropped.

One evaluation call: the imaginary-axis term and its slope for all points by
one kernel (mbpt_cd_integral_terms); the residues as one batch of linear
systems [1 - chi0(f)] y = b, one column per (point, residue) pair, solved by
preconditioned conjugate gradients with one FP64 product over the whole
batch per iteration (chi0(f) = sum_k c_k(f) proj(tau_k) for the Laplace
backend, 2 C_ov F C_ov^T for the explicit one) and Cholesky factors of
1 - chi0 at a few anchor frequencies as preconditioners; a column whose
frequency lies above the particle-hole gap (1 - chi0 indefinite, explicit
backend only) or that does not converge is solved directly against its own
frequency's factorisation. The Laplace backend's representability test of
every frequency runs on the device (mbpt_laplace_representation_error).
"""
from __future__ import annotations

import warnings
from collections import OrderedDict

import numpy as np
import torch

from ._lib import MODES, WORKSPACE, check, lib, ptr, require_device, stream_ptr
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

# the residue solves: relative residual of the conjugate-gradient solution,
# iterations before a column is solved directly, anchor spacing in units of
# the lowest particle-hole energy, columns per batched product
PCG_TOL, PCG_MAX_ITER = 1e-13, 60
ANCHOR_STEP = 1.0 / 32.0
PCG_COLUMNS = 2048


class ResidueRefused(ValueError):
    """A real frequency the imaginary-time representation does not carry
    (``real_screening.py:49-54``)."""


# ------------------------------------------------------------ the contour grid

def gap_scaled_w0(eps, nocc, scale=0.5):
    """w0 = scale (eps_LUMO - eps_HOMO) (``Base/utils/grids/grids.py:173-186``)."""
    lo, _ = _transition_edges(eps, nocc, None)
    if not lo > 0:
        raise ValueError(f'gap_scaled_w0: the gap {lo:.6g} is not positive')
    return scale * lo


def _transition_edges(eps, nocc, pair_energies):
    """(lowest, highest) particle-hole energy: of the pair energies when
    given (both spins of an unrestricted reference), else of (eps, nocc)."""
    if pair_energies is not None:
        d = np.asarray(pair_energies, float)
        return float(d.min()), float(d.max())
    gap, span, _ = particle_hole_window(np.asarray(eps, float), nocc)
    return float(gap), float(span)


def cd_grid_range(eps, nocc, e_min_below_gap=None, pair_energies=None):
    """(e_min, e_max) of the contour's time grid (``contour_deformation.py:439-468``):
    the grid reaches `e_min_below_gap` (default: half the lowest particle-hole
    energy) below the lowest particle-hole energy, so that the residues' real
    frequencies up to that depth stay representable, and up to the highest."""
    lo, hi = _transition_edges(eps, nocc, pair_energies)
    depth = 0.5 * lo if e_min_below_gap is None else float(e_min_below_gap)
    if not lo - depth > 0:
        raise ValueError(f'e_min_below_gap {depth} exceeds the gap {lo:.4f}: the imaginary-'
                         f'time grid would be asked to represent e^{{-y tau}} at y <= 0')
    return lo - depth, hi


def cd_frequency_grid(eps, nocc, ntau=CD_NTAU, nfreq_cd=CD_NFREQ, w0_cd=None,
                      e_min_below_gap=None, pair_energies=None):
    """(nu, nu_weights, grid, w0) (``contour_deformation.py:471-503``): the
    Gauss-Legendre imaginary frequencies of scale w0 (default half the
    lowest particle-hole energy) and the minimax time grid over
    `cd_grid_range`, mapped onto them by its cosine weights alone."""
    e_min, e_max = cd_grid_range(eps, nocc, e_min_below_gap, pair_energies)
    w0 = (0.5 * _transition_edges(eps, nocc, pair_energies)[0] if w0_cd is None
          else float(w0_cd))
    nu, nu_weights = gauss_legendre_grid(int(nfreq_cd), w0=w0)
    grid = TimeFrequencyGrid.minimax_split(int(ntau), e_min, e_max, nu, nu_weights,
                                           with_sine=False, with_inverse=False)
    return nu, nu_weights, grid, w0


# --------------------------------------------- the imaginary-axis quadrature

class LorentzianQuadrature:
    """The weights c_k(d) of -(1/pi) int_0^inf g(d, nu) wc(nu) dnu on the
    Gauss-Legendre nodes nu_k, g = d / (d^2 + nu^2), d = omega - eps_q
    (``contour_deformation.py:150-202``). The kernel peaks at nu ~ |d|, which
    the nodes cannot resolve for small |d|; its part wc(0) a^2 / (a^2 + nu^2)
    is integrated exactly, (pi/2) sign(d) a / (a + |d|), with a = 4 median(nu)
    and wc(0) extrapolated linearly in nu^2 from the two nodes nearest zero,
    and only the remainder by quadrature. A pole on the contour (|d| below
    the on-contour tolerance) takes sign 0, as its residue is taken at half
    weight."""

    def __init__(self, nu, nu_w, on_tol=RESIDUE_ON_CONTOUR_TOL):
        self.nu = np.asarray(nu, float)
        self.w = np.asarray(nu_w, float)
        self.on_tol = float(on_tol)
        self.a = 4.0 * float(np.median(self.nu))
        k1, k2 = np.argsort(self.nu)[:2]
        s1, s2 = self.nu[k1] ** 2, self.nu[k2] ** 2
        # wc(0) ~ e1 wc(nu_k1) + e2 wc(nu_k2), linear in nu^2
        self.k1, self.k2 = int(k1), int(k2)
        self.e1, self.e2 = s2 / (s2 - s1), -s1 / (s2 - s1)
        # the model's quadrature weights h_k
        self.h = self.w * self.a ** 2 / (self.a ** 2 + self.nu ** 2)
        self._dev = None

    def weights(self, d):
        """(c, dc), each (nfreq, len(d)): the weights and their d derivative."""
        d = np.atleast_1d(np.asarray(d, float))
        n2 = (self.nu ** 2)[:, None]
        den = d[None, :] ** 2 + n2
        g = d[None, :] / den
        dg = (n2 - d[None, :] ** 2) / den ** 2
        span = self.a + np.abs(d)
        side = np.where(np.abs(d) < self.on_tol, 0.0, np.sign(d))
        corr = 0.5 * np.pi * side * self.a / span - self.h @ g
        dcorr = -0.5 * np.pi * self.a / span ** 2 - self.h @ dg
        c, dc = self.w[:, None] * g, self.w[:, None] * dg
        for k, e in ((self.k1, self.e1), (self.k2, self.e2)):
            c[k] += e * corr
            dc[k] += e * dcorr
        return c, dc

    def device(self, dev):
        if self._dev is None:
            self._dev = (torch.as_tensor(self.nu, device=dev),
                         torch.as_tensor(self.w, device=dev))
        return self._dev


def cd_integral_weights(de, nu_points, nu_weights):
    """(c, dc), (nfreq, norb): Sigma^int = -(1/pi) sum c wc for de = omega -
    eps, and its derivative in de (``contour_deformation.py:150-202``)."""
    return LorentzianQuadrature(nu_points, nu_weights).weights(de)


def integral_terms(wc, eps, quad, slots, omega):
    """(value, slope) of Sigma^int at the points (slots[j], omega[j]) on the
    device: wc (nslots, nfreq, norb) device FP64, slots int, omega float.
    Host arrays back."""
    dev = wc.device
    slots = np.ascontiguousarray(slots, dtype=np.int32)
    omega = np.ascontiguousarray(omega, dtype=float)
    nq = len(omega)
    if nq == 0:
        return np.zeros(0), np.zeros(0)
    nu, nw = quad.device(dev)
    ed = to_device(eps, dev)
    sd = torch.as_tensor(slots, device=dev)
    od = torch.as_tensor(omega, device=dev)
    out = torch.empty((2, nq), dtype=torch.float64, device=dev)
    wcc = wc.contiguous()
    check(lib().mbpt_cd_integral_terms(ptr(wcc), wcc.shape[0], wcc.shape[1], wcc.shape[2],
                                       ptr(ed), ptr(nu), ptr(nw), quad.k1, quad.k2,
                                       float(quad.e1), float(quad.e2), float(quad.a),
                                       float(quad.on_tol), ptr(sd), ptr(od), nq, ptr(out[0]),
                                       ptr(out[1]), stream_ptr()), 'mbpt_cd_integral_terms')
    h = out.cpu().numpy()
    return h[0], h[1]


# ----------------------------------------------------------------- residues

def residue_weights(eps, nocc, omega, tol=RESIDUE_ON_CONTOUR_TOL):
    """r[j, q] for the points omega[j] (``real_screening.py:157-168``): the
    poles of G the deformation sweeps -- -1 for an occupied level above
    omega, +1 for a virtual level below it, -1/2 / +1/2 for a level on the
    contour (|eps_q - omega| < tol), 0 otherwise. (len(omega), norb)."""
    eps = np.asarray(eps, float)
    om = np.atleast_1d(np.asarray(omega, float))
    gap = eps[None, :] - om[:, None]
    occ = (np.arange(eps.size) < nocc)[None, :]
    r = np.where(occ & (gap > 0.0), -1.0, 0.0) + np.where(~occ & (gap < 0.0), 1.0, 0.0)
    on = np.abs(gap) < tol
    return np.where(on, np.where(occ, -0.5, 0.5), r)


def residue_set(eps, nocc, omega, tol=RESIDUE_ON_CONTOUR_TOL):
    """[(q, weight)] of the residues at one omega, in increasing q
    (``real_screening.py:157-168``)."""
    r = residue_weights(eps, nocc, [omega], tol)[0]
    return [(int(q), float(r[q])) for q in np.nonzero(r)[0]]


def real_frequency_weights(grid, omega):
    """(c, dc): chi0(omega) = sum_k c_k proj(tau_k) at a real omega below the
    gap, c_k = 2 w_k cosh(omega tau_k) on the grid's bare Laplace quadrature,
    and its omega derivative (``real_screening.py:184-209``)."""
    t = np.asarray(grid.tau_points, float)
    w = 2.0 * np.asarray(grid.tau_weights, float)
    om = np.asarray(omega, float)
    if om.ndim == 0:
        return w * np.cosh(om * t), w * t * np.sinh(om * t)
    return (w[:, None] * np.cosh(np.outer(t, om)),
            (w * t)[:, None] * np.sinh(np.outer(t, om)))


def laplace_representation_error(grid, eps, nocc, freq, pair_energies=None):
    """max over y = d -+ freq of |y sum_k w_k e^{-y tau_k} - 1| on the pair
    energies d (those of (eps, nocc), or pair_energies), inf where freq
    reaches the gap (``LinearResponse/space_time.py:908-931``); host FP64."""
    d = ov_energies(eps, nocc) if pair_energies is None else np.asarray(pair_energies, float)
    y = np.concatenate([d - freq, d + freq])
    if y.min() <= 0.0:
        return np.inf
    q = np.exp(-np.outer(y, grid.tau_points)) @ grid.tau_weights
    return float(np.abs(q * y - 1.0).max())


# -------------------------------------- batched solves of [1 - chi0(f)] y = b

class _FactorCache:
    """1 - chi0(f) factorised per key, kept for the latest keys within a byte
    budget: ('chol', L) for a positive definite matrix (the Dyson step's FP64
    Cholesky factor, solved by mbpt_chol_solve), ('w', W - I) from the LU
    inverse otherwise."""

    def __init__(self, budget_bytes, naux):
        self.cap = max(2, int(budget_bytes // (8 * naux * naux)))
        self._c = OrderedDict()

    def get(self, key):
        ent = self._c.get(key)
        if ent is not None:
            self._c.move_to_end(key)
        return ent

    def build(self, keys, chi0_of, spd_expected=True):
        """Factorise 1 - chi0 for each key (chi0_of(keys) -> (n, naux, naux)
        device tensor, consumed): one batched Cholesky when spd_expected,
        the LU inverse for any key that is not positive definite."""
        if not keys:
            return
        redo = list(range(len(keys)))
        if spd_expected:
            chi = chi0_of(keys)
            _, _, info, _ = dyson_batch(chi, want_w=False, precision='fp64')
            redo = [i for i in range(len(keys)) if info[i] != 0]
            for i, k in enumerate(keys):
                if info[i] == 0:
                    self._put(k, ('chol', chi[i]))
        if redo:
            again = chi0_of([keys[i] for i in redo])
            dyson_batch(again, want_w=True, precision='fp64')
            for j, i in enumerate(redo):
                self._put(keys[i], ('w', again[j]))

    def _put(self, key, ent):
        self._c[key] = ent
        while len(self._c) > self.cap:
            self._c.popitem(last=False)


def _apply_factor(ent, R):
    """M^-1 R for the columns of R (naux, k): two triangular solves against a
    Cholesky factor, or R + (W - I) R from an LU inverse."""
    kind, m = ent
    if kind == 'w':
        return R + m @ R
    y = R.T.contiguous()
    check(lib().mbpt_chol_solve(ptr(m), m.shape[0], ptr(y), y.shape[0], stream_ptr()),
          'mbpt_chol_solve')
    return y.T


class _BatchedScreening:
    """The solver half of a residue backend: Y[:, j] = [1 - chi0(f_j)]^-1
    B[:, j] for a batch of frequencies at once. Subclasses give chi0(f) as a
    dense matrix for a set of frequencies (`_chi0_dense`), chi0(f_j) x_j for
    all columns at once (`_chi0_apply`), and the slope y^T chi0'(f) y."""

    naux = 0
    lowest = 0.0          # lowest particle-hole energy: the edge of the SPD region

    def _init_solver(self, cache_bytes):
        self._factors = _FactorCache(0.5 * cache_bytes, self.naux)
        self._direct = _FactorCache(0.5 * cache_bytes, self.naux)
        self.stats = {'columns': 0, 'pcg_iterations': 0, 'direct': 0, 'anchors': 0}

    def _anchor_of(self, f):
        """The anchor cell of a frequency below the lowest particle-hole
        energy: cells of ANCHOR_STEP times it, each anchored at its middle,
        so no anchor reaches the gap."""
        return int(np.floor(f / (ANCHOR_STEP * self.lowest)))

    def _anchor_freq(self, i):
        return (i + 0.5) * ANCHOR_STEP * self.lowest

    def solve(self, freqs, B):
        """Y (naux, n) on the device for frequencies freqs (n,) and
        right-hand sides B (naux, n)."""
        freqs = np.asarray(freqs, float)
        n = len(freqs)
        Y = torch.empty_like(B)
        if n == 0:
            return Y
        self.stats['columns'] += n
        spd = freqs < self.lowest
        direct = np.nonzero(~spd)[0]
        it = np.nonzero(spd)[0]
        if it.size:
            done, X = self._pcg(freqs[it], B[:, torch.as_tensor(it, device=B.device)])
            Y[:, torch.as_tensor(it, device=B.device)] = X
            direct = np.concatenate([direct, it[~done]])
        if direct.size:
            self._solve_direct(freqs, B, Y, direct)
        return Y

    def _solve_direct(self, freqs, B, Y, cols):
        self.stats['direct'] += len(cols)
        keys = sorted({float(freqs[c]) for c in cols})
        need = [k for k in keys if self._direct.get(k) is None]
        for i in range(0, len(need), 8):
            part = need[i:i + 8]
            self._direct.build(part, self._chi0_dense, spd_expected=part[-1] < self.lowest)
        for k in keys:
            sel = [c for c in cols if float(freqs[c]) == k]
            idx = torch.as_tensor(sel, device=B.device)
            ent = self._direct.get(k)
            if ent is None:       # evicted by a later build of this call: rebuild alone
                self._direct.build([k], self._chi0_dense, spd_expected=k < self.lowest)
                ent = self._direct.get(k)
            Y[:, idx] = _apply_factor(ent, B[:, idx])

    def _pcg(self, freqs, B):
        """Conjugate gradients on [1 - chi0(f_j)] y_j = b_j, all columns at
        once, each preconditioned by the Cholesky factor of 1 - chi0 at its
        nearest anchor frequency. Returns (converged mask, Y)."""
        anchors = np.array([self._anchor_of(f) for f in freqs])
        groups = {}
        for j, a in enumerate(anchors):
            groups.setdefault(int(a), []).append(j)
        need = [a for a in groups if self._factors.get(a) is None]
        self.stats['anchors'] += len(need)
        for i in range(0, len(need), 8):
            self._factors.build(need[i:i + 8],
                                lambda keys: self._chi0_dense([self._anchor_freq(a)
                                                               for a in keys]))
        dev = B.device
        gidx = {a: torch.as_tensor(js, device=dev) for a, js in groups.items()}

        def precond(R):
            Z = torch.empty_like(R)
            for a, idx in gidx.items():
                ent = self._factors.get(a)
                if ent is None:
                    self._factors.build([a], lambda keys: self._chi0_dense(
                        [self._anchor_freq(k) for k in keys]))
                    ent = self._factors.get(a)
                Z[:, idx] = _apply_factor(ent, R[:, idx])
            return Z

        def op(X):
            return X - self._chi0_apply(freqs, X)

        bnorm = torch.linalg.vector_norm(B, dim=0)
        bnorm = torch.where(bnorm > 0, bnorm, torch.ones_like(bnorm))
        X = precond(B)
        R = B - op(X)
        Z = precond(R)
        P = Z.clone()
        rz = (R * Z).sum(0)
        done = torch.zeros(len(freqs), dtype=torch.bool, device=dev)
        for it in range(PCG_MAX_ITER):
            done = torch.linalg.vector_norm(R, dim=0) <= PCG_TOL * bnorm
            if bool(done.all()):
                break
            self.stats['pcg_iterations'] += 1
            Q = op(P)
            pq = (P * Q).sum(0)
            alpha = torch.where(done, torch.zeros_like(rz), rz / torch.where(pq != 0, pq, 1.0))
            X = X + alpha * P
            R = R - alpha * Q
            Z = precond(R)
            rz_new = (R * Z).sum(0)
            beta = torch.where(rz != 0, rz_new / torch.where(rz != 0, rz, 1.0),
                               torch.zeros_like(rz))
            P = Z + beta * P
            rz = rz_new
        done = torch.linalg.vector_norm(R, dim=0) <= PCG_TOL * bnorm
        return done.cpu().numpy(), X

    # the reference's per-frequency protocol (``real_screening.py``)
    def apply(self, freq, b):
        """W(freq) b = [1 - chi0(freq)]^-1 b for one frequency; b (naux,) or
        (naux, k), host or device, returned as given."""
        self._refuse([float(freq)])
        dev = self._device()
        bd = to_device(b, dev)
        cols = bd[:, None] if bd.dim() == 1 else bd
        y = self.solve(np.full(cols.shape[1], float(freq)), cols.contiguous())
        y = y[:, 0] if bd.dim() == 1 else y
        return y if isinstance(b, torch.Tensor) else y.cpu().numpy()

    def slope(self, freq, y):
        """y^T [dchi0/dfreq] y at one frequency."""
        yd = to_device(y, self._device())
        return float(self.slopes(np.array([float(freq)]), yd[:, None])[0])

    def _refuse(self, freqs):
        """Raise ResidueRefused for a frequency this backend cannot serve."""

    def refused(self, freqs):
        """Boolean mask of the frequencies this backend cannot serve."""
        return np.zeros(len(freqs), dtype=bool)


class LaplaceRealScreening(_BatchedScreening):
    """W at real frequencies below the particle-hole gap from proj(tau)
    (``real_screening.py:94-154``): chi0(f) = sum_k 2 w_k cosh(f tau_k)
    proj(tau_k) on the grid's bare Laplace quadrature. A frequency the grid
    does not carry (quadrature error of 1/y at or above tol on the pair
    energies) is refused (ResidueRefused). pair_energies: the particle-hole
    energies proj(tau) was summed over, when they are not the ones (eps,
    nocc) spans (both spins of an unrestricted reference). cache_bytes bounds
    the factorisations kept (anchors and direct solves)."""

    def __init__(self, proj_tau, grid, eps, nocc, tol=LAPLACE_SCREENING_TOL,
                 pair_energies=None, cache_bytes=4e9):
        dev = require_device()
        self.proj_tau = to_device(proj_tau, dev)
        self.grid = grid
        self.eps = np.asarray(eps, float)
        self.nocc = nocc
        self.tol = tol
        self.pair_energies = (None if pair_energies is None
                              else np.asarray(pair_energies, float))
        d = (ov_energies(self.eps, nocc) if self.pair_energies is None
             else self.pair_energies)
        self.lowest = float(d.min())
        self.naux = self.proj_tau.shape[-1]
        self._d = torch.as_tensor(d, dtype=torch.float64, device=dev)
        self._tau = torch.as_tensor(np.asarray(grid.tau_points, float), device=dev)
        self._tw = torch.as_tensor(np.asarray(grid.tau_weights, float), device=dev)
        self._flat = self.proj_tau.reshape(-1, self.naux)
        self._errors = {}
        self._init_solver(cache_bytes)

    def _device(self):
        return self.proj_tau.device

    def errors(self, freqs):
        """The representation error of each frequency (device kernel, kept
        per frequency)."""
        freqs = np.asarray(freqs, float)
        new = sorted({float(f) for f in freqs if float(f) not in self._errors})
        if new:
            dev = self._device()
            fd = torch.as_tensor(new, dtype=torch.float64, device=dev)
            out = torch.empty_like(fd)
            check(lib().mbpt_laplace_representation_error(
                ptr(self._d), self._d.numel(), ptr(self._tau), ptr(self._tw),
                self._tau.numel(), ptr(fd), len(new), ptr(out), stream_ptr()),
                'mbpt_laplace_representation_error')
            for f, e in zip(new, out.cpu().numpy()):
                self._errors[f] = float(e)
        return np.array([self._errors[float(f)] for f in freqs])

    def representation_error(self, freq):
        """max over y = d -+ freq of |y sum_k w_k e^{-y tau_k} - 1|, inf where
        freq reaches the gap (``LinearResponse/space_time.py:908-931``)."""
        return float(self.errors([freq])[0])

    def refused(self, freqs):
        return ~(self.errors(freqs) < self.tol)

    def _refuse(self, freqs):
        bad = self.refused(freqs)
        if bad.any():
            f = float(np.asarray(freqs)[bad][0])
            raise ResidueRefused(
                f'real frequency {f:.4f} Ha is not carried by the tau grid: bare-quadrature '
                f'error {self.representation_error(f):.1e} against tol {self.tol:.0e}; '
                f'gap - freq = {self.lowest - f:.4f} Ha, the grid\'s e_min is '
                f'{self.grid.meta.get("e_min", float("nan")):.4f}. Build the grid with '
                f'e_min <= gap - freq, or use the explicit backend.')

    def _chi0_dense(self, freqs):
        c, _ = real_frequency_weights(self.grid, np.asarray(freqs, float))
        return _rows_transform(self.proj_tau, np.ascontiguousarray(c.T))

    def _stacked(self, coef, X):
        """sum_k proj(tau_k) (X with column j scaled by coef[k, j]): one FP64
        product over the time points stacked along K (proj(tau) is
        symmetric, so its stacked rows serve as the transposed operand)."""
        T = coef.shape[0]
        cd = torch.as_tensor(np.ascontiguousarray(coef), device=X.device)
        out = torch.empty_like(X)
        for j0 in range(0, X.shape[1], PCG_COLUMNS):
            Xs = X[:, j0:j0 + PCG_COLUMNS]
            Z = (cd[:, None, j0:j0 + PCG_COLUMNS] * Xs[None]).reshape(T * self.naux, -1)
            out[:, j0:j0 + PCG_COLUMNS] = self._flat.T @ Z
        return out

    def _chi0_apply(self, freqs, X):
        c, _ = real_frequency_weights(self.grid, freqs)
        return self._stacked(c, X)

    def slopes(self, freqs, Y):
        """y_j^T [dchi0/df](f_j) y_j for each column (host array)."""
        if Y.shape[1] == 0:
            return np.zeros(0)
        _, dc = real_frequency_weights(self.grid, np.asarray(freqs, float))
        return (Y * self._stacked(dc, Y)).sum(0).cpu().numpy()

    def w_minus_identity(self, freq):
        """W(freq) - I as a dense device matrix (FP64)."""
        self._refuse([float(freq)])
        chi = self._chi0_dense([float(freq)])
        dyson_batch(chi, want_w=True, precision='fp64')
        return chi[0]


class ExplicitRealScreening(_BatchedScreening):
    """W at a real frequency from the particle-hole block C_ov, explicitly
    (``real_screening.py:57-91``, continuation 'cd'): chi0(f) = 2 C_ov F(f)
    C_ov^T with the bubble's frequency factor F (broadened by eta, off by
    default). Below the lowest particle-hole energy the batch is solved by
    preconditioned conjugate gradients (two FP64 products with C_ov per
    iteration); above it, where 1 - chi0 is indefinite, each frequency's
    explicit chi0 (mbpt_chi0_aux) goes through the Dyson step's LU inverse.
    pair_energies: the pair index of C_ov when it is not the one (eps, nocc)
    spans. precision 'mixed' forms the dense chi0 of the anchors and of the
    direct solves as one split BF16x3 product (the iterations stay FP64, so
    the solution does too, except for the direct columns)."""

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
        self.naux = self.C_ov.shape[0]
        self.lowest = float(self.d.min())
        self._dd = torch.as_tensor(self.d, device=self.C_ov.device)
        self._init_solver(cache_bytes)

    def _device(self):
        return self.C_ov.device

    def _chi0(self, freq, imaginary=False):
        f = frequency_factor(self.d, float(freq), imaginary, self.eta)
        return chi0_aux([(self.C_ov, f)], 2.0, precision=self.precision)[None]

    def _chi0_dense(self, freqs):
        out = torch.empty((len(freqs), self.naux, self.naux), dtype=torch.float64,
                          device=self.C_ov.device)
        for i, f in enumerate(freqs):
            chi0_aux([(self.C_ov, frequency_factor(self.d, float(f), False, self.eta))], 2.0,
                     out=out[i], precision=self.precision)
        return out

    def _factor(self, freqs, slopes):
        """F[pair, j] (or dF/df) of the bubble at real f_j, on the device."""
        f = torch.as_tensor(np.asarray(freqs, float), device=self._dd.device)[None, :]
        a, b = f - self._dd[:, None], f + self._dd[:, None]
        if self.eta == 0.0:
            return (1.0 / b ** 2 - 1.0 / a ** 2) if slopes else (1.0 / a - 1.0 / b)
        e2 = self.eta ** 2
        da, db = a ** 2 + e2, b ** 2 + e2
        if slopes:
            return (e2 - a ** 2) / da ** 2 - (e2 - b ** 2) / db ** 2
        return a / da - b / db

    def _chi0_apply(self, freqs, X):
        out = torch.empty_like(X)
        for j0 in range(0, X.shape[1], PCG_COLUMNS):
            Z = self.C_ov.T @ X[:, j0:j0 + PCG_COLUMNS]
            Z *= self._factor(freqs[j0:j0 + PCG_COLUMNS], False)
            out[:, j0:j0 + PCG_COLUMNS] = 2.0 * (self.C_ov @ Z)
        return out

    def slopes(self, freqs, Y):
        """y_j^T [dchi0/df](f_j) y_j = 2 sum_pairs dF/df (C_ov^T y_j)^2."""
        if Y.shape[1] == 0:
            return np.zeros(0)
        out = []
        for j0 in range(0, Y.shape[1], PCG_COLUMNS):
            Z = self.C_ov.T @ Y[:, j0:j0 + PCG_COLUMNS]
            out.append(2.0 * (self._factor(freqs[j0:j0 + PCG_COLUMNS], True) * Z * Z).sum(0))
        return torch.cat(out).cpu().numpy()

    def w_minus_identity(self, freq, imaginary=False):
        """W(freq) - I as a dense device matrix (the Dyson step: Cholesky
        below the gap, LU above it)."""
        chi = self._chi0(freq, imaginary)
        dyson_batch(chi, want_w=True, precision='fp64')
        return chi[0]


# ----------------------------------------------------- the self-energy batch

class ContourEquation:
    """f(w) = w - a_s - Sigma^c_s(w) and f'(w) for a set of states s (slots),
    evaluated for many (slot, w) points per call. B: (nslots, naux, norb)
    slices, wc: (nslots, nfreq, norb) contracted screening, bare: a_s =
    eps_p + xc per slot, backend: the residues' screening (None: a state
    whose points sweep no residue needs none)."""

    def __init__(self, B, wc, eps, nocc, quad, bare, backend):
        dev = require_device()
        self.B = to_device(B, dev)
        self.wc = to_device(wc, dev)
        if self.B.dim() == 2:
            self.B = self.B[None]
        if self.wc.dim() == 2:
            self.wc = self.wc[None]
        self.eps = np.asarray(eps, float)
        self.nocc = nocc
        self.quad = quad
        self.bare = np.atleast_1d(np.asarray(bare, float))
        self.backend = backend
        self.points = 0

    def sigma(self, slots, w, want_slope=True, residues=None):
        """(Sigma, dSigma/dw, refused) at the points; residues: one fixed set
        [(q, weight)] for every point instead of the points' own."""
        slots = np.asarray(slots, int)
        w = np.asarray(w, float)
        self.points += len(w)
        val, slope = integral_terms(self.wc, self.eps, self.quad, slots, w)
        if residues is None:
            R = residue_weights(self.eps, self.nocc, w)
        else:
            R = np.zeros((len(w), self.eps.size))
            for q, weight in residues:
                R[:, q] = weight
        jj, qq = np.nonzero(R)
        refused = np.zeros(len(w), dtype=bool)
        if jj.size == 0:
            return val, slope, refused
        if self.backend is None:
            require_three_index(None, 'the residue term')
        gap = self.eps[qq] - w[jj]
        f = np.abs(gap)
        bad = self.backend.refused(f)
        if bad.any():
            refused[np.unique(jj[bad])] = True
        keep = ~refused[jj]
        jj, qq, f, gap = jj[keep], qq[keep], f[keep], gap[keep]
        r = R[jj, qq]
        dev = self.B.device
        cols = self.B[torch.as_tensor(slots[jj], device=dev), :,
                      torch.as_tensor(qq, device=dev)].T.contiguous()
        Y = self.backend.solve(f, cols)
        by = (cols * Y).sum(0).cpu().numpy()
        bb = (cols * cols).sum(0).cpu().numpy()
        np.add.at(val, jj, r * (by - bb))
        if want_slope:
            s = self.backend.slopes(f, Y)
            np.add.at(slope, jj, -r * s * np.sign(gap))
        val[refused] = np.nan
        slope[refused] = np.nan
        return val, slope, refused

    def __call__(self, slots, w, want_slope=True):
        """(f, f', refused) at the points."""
        slots = np.asarray(slots, int)
        s, ds, refused = self.sigma(slots, w, want_slope)
        return np.asarray(w, float) - self.bare[slots] - s, 1.0 - ds, refused


# ------------------------------------- proj(tau), slices and the contraction

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


# ------------------------------------------------------------ the lockstep scan
# The rules are those of MBPTcode's `solve_qp_equation_scan` on a
# `SampledEquation` with a closed-form slope and positive weights
# (``Solvers/qp_equation.py:155-273, 1029-1420``), which the contour route
# (`qp_energy_cd`) uses without a followed root.

def _windows(a):
    """[(lo, hi)] about the bare level a, narrowest first: the tier of the
    state's depth |a| and every wider one (``qp_equation.py:1280-1288``)."""
    tier = max((k for k, (depth, _) in enumerate(QP_SEARCH_WINDOW_TIERS) if abs(a) > depth),
               default=0)
    return [(a - half, a + half) for _, half in QP_SEARCH_WINDOW_TIERS[tier:]]


def _valid(z, z_min=0.0):
    """Z of a quasiparticle: finite and in (z_min, 1] (``qp_equation.py:95-102``)."""
    z = float(z)
    return bool(np.isfinite(z) and z_min < z <= 1.0)


def _walk_order(c0, ncells):
    """The cells in the order the outward walk reaches them: the one holding
    the bare level, then at each distance the lower neighbour and the upper."""
    order = [c0]
    for d in range(1, ncells):
        order.extend(c for c in (c0 - d, c0 + d) if 0 <= c < ncells)
    return order


class _Walk:
    """One state's walk over one window's grid."""

    def __init__(self, slot, a, lo, hi, enough):
        self.slot, self.a, self.enough = slot, a, enough
        self.grid = np.linspace(lo, hi, QP_GRAPHICAL_N_OMEGA)
        c0 = min(max(int(np.searchsorted(self.grid, a)) - 1, 0), self.grid.size - 2)
        self.order = _walk_order(c0, self.grid.size - 1)
        self.pos, self.f, self.bad = 0, {}, {}
        self.found, self.weighed, self.best = [], 0.0, -np.inf
        self.refusal = None
        self.done = False


class _FollowWalk:
    """One state's search, over one window's grid, for the valid root nearest
    a root followed from a previous geometry: rings of cells outward from
    the cell holding it, until the next ring lies farther from it than the
    nearest root found."""

    def __init__(self, slot, target, lo, hi):
        self.slot, self.t, self.lo, self.hi = slot, float(target), lo, hi
        self.grid = np.linspace(lo, hi, QP_GRAPHICAL_N_OMEGA)
        self.c0 = min(max(int(np.searchsorted(self.grid, target)) - 1, 0), self.grid.size - 2)
        self.d = 0
        self.f, self.bad = {}, {}
        self.solved = {}            # (l, r) of a bracket -> [(w, Z)]
        self.best = None
        self.refusal = None
        self.done = False

    def ring(self):
        n = self.grid.size - 1
        return sorted(c for c in {self.c0 - self.d, self.c0 + self.d} if 0 <= c < n)


class _LockstepScan:
    """The scan of many states at once. equation(slots, w, want_slope) ->
    (f, f', refusals {index: exception}) evaluates f(w) = w - a - Sigma(w)
    and its slope at every point of a round. positive_weight: Sigma is a sum
    of poles of positive weight, so a bracket where f falls holds a pole and
    is passed over, and the valid weights of all roots sum to one, which ends
    a window's walk early; without it every bracket of a window is solved."""

    def __init__(self, equation, tol=QP_ROOT_TOL, max_iter=QP_ROOT_MAX_ITER,
                 positive_weight=True):
        self.eq, self.tol, self.max_iter = equation, tol, int(max_iter)
        self.positive_weight = bool(positive_weight)
        self.rounds = 0

    def _eval(self, slots, w, want_slope):
        if len(w) == 0:
            return np.zeros(0), np.zeros(0), {}
        self.rounds += 1
        f, fp, bad = self.eq(np.asarray(slots, int), np.asarray(w, float), want_slope)
        return np.asarray(f, float), np.asarray(fp, float), bad

    # -- brackets of a set of cells: the cell on a sign change; its halves
    # while its secant slope is below QP_SCAN_SECANT_MIN or one end is refused
    # and the other not, at most QP_SCAN_SPLIT_DEPTH times; one level of
    # halving of every open cell per round
    def _brackets(self, cells):
        """cells: [(key, slot, l, r, fl, fr)] -> {key: [(path, l, r, fl, fr)]},
        {key: refusal or None} of the halving points."""
        out = {key: [] for key, *_ in cells}
        bad = {key: None for key, *_ in cells}
        items = [(key, slot, '', l, r, fl, fr, QP_SCAN_SPLIT_DEPTH)
                 for key, slot, l, r, fl, fr in cells]
        while items:
            split = []
            for key, slot, path, l, r, fl, fr, depth in items:
                if fl * fr < 0.0:
                    out[key].append((path, l, r, fl, fr))
                    continue
                edge = np.isnan(fl) != np.isnan(fr)
                if depth == 0 or fl == 0.0 or fr == 0.0 or not (
                        edge or fr - fl < QP_SCAN_SECANT_MIN * (r - l)):
                    continue
                split.append((key, slot, path, l, r, fl, fr, depth))
            if not split:
                break
            mids = [0.5 * (it[3] + it[4]) for it in split]
            fm, _, refused = self._eval([it[1] for it in split], mids, False)
            items = []
            for i, (key, slot, path, l, r, fl, fr, depth) in enumerate(split):
                if i in refused and bad[key] is None:
                    bad[key] = refused[i]
                m = mids[i]
                items.append((key, slot, path + '0', l, m, fl, fm[i], depth - 1))
                items.append((key, slot, path + '1', m, r, fm[i], fr, depth - 1))
        return out, bad

    # -- roots of brackets: Newton on the closed-form slope inside the
    # bracket, one step of every open bracket per round (``qp_equation.py:376-426``
    # for a costly f): a step that leaves the bracket, or is not under half
    # the step before the last, is a bisection; a step below tol that stays
    # in the closed bracket ends it; a bracket one ulp wide ends at its point
    def _roots(self, brackets):
        """brackets: [(slot, l, r, fl, fr)] -> ([] or [(w, Z)] each, refusal
        per bracket)."""
        n = len(brackets)
        roots, bad = [None] * n, [None] * n
        live, at = [], {}
        for i, (slot, l, r, fl, fr) in enumerate(brackets):
            if l == r:
                at[i] = float(l)
            elif self.positive_weight and fl > 0.0 > fr:
                roots[i] = []          # f falls: a pole of a positive-weight Sigma
            else:
                live.append(i)
        if live:
            slots = np.array([brackets[i][0] for i in live])
            L = np.array([brackets[i][1] for i in live], float)
            R = np.array([brackets[i][2] for i in live], float)
            SL = np.sign([brackets[i][3] for i in live])
            W = 0.5 * (L + R)
            old = R - L
            step = R - L
            result = np.full(len(live), np.nan)
            active = np.ones(len(live), dtype=bool)
            for _ in range(self.max_iter):
                idx = np.nonzero(active)[0]
                if idx.size == 0:
                    break
                f, fp, refused = self._eval(slots[idx], W[idx], True)
                for k, e in refused.items():
                    if bad[live[idx[k]]] is None:
                        bad[live[idx[k]]] = e
                w = W[idx]
                with np.errstate(divide='ignore', invalid='ignore'):
                    dw = -f / fp
                zero = f == 0.0
                same = np.sign(f) == SL[idx]
                L[idx] = np.where(same, w, L[idx])
                R[idx] = np.where(same, R[idx], w)
                l, r = L[idx], R[idx]
                with np.errstate(invalid='ignore'):
                    conv = (np.abs(dw) < self.tol) & (l <= w + dw) & (w + dw <= r)
                mid = 0.5 * (l + r)
                stuck = ~((l < mid) & (mid < r))
                with np.errstate(invalid='ignore'):
                    newton = (np.isfinite(dw) & (l < w + dw) & (w + dw < r)
                              & (np.abs(dw) <= 0.5 * np.abs(old[idx])))
                stop = zero | conv | stuck
                result[idx] = np.where(zero, w, np.where(conv, w + dw, w))
                go = ~stop
                old[idx] = np.where(go, step[idx], old[idx])
                step[idx] = np.where(go, np.where(newton, dw, mid - w), step[idx])
                W[idx] = np.where(go, np.where(newton, w + dw, mid), w)
                active[idx[stop]] = False
            result = np.where(active, W, result)
            for j, i in enumerate(live):
                at[i] = float(result[j])
        if at:
            keys = list(at)
            f, fp, refused = self._eval([brackets[i][0] for i in keys],
                                        [at[i] for i in keys], True)
            for j, i in enumerate(keys):
                if j in refused and bad[i] is None:
                    bad[i] = refused[j]
                fl, fr = brackets[i][3], brackets[i][4]
                if brackets[i][1] != brackets[i][2] and not abs(f[j]) <= max(abs(fl), abs(fr)):
                    roots[i] = []      # |f| grew (a pole) or the point was refused
                else:
                    z = 1.0 / fp[j] if fp[j] != 0.0 else np.nan
                    roots[i] = [(at[i], float(z))]
        return roots, bad

    def walk(self, walks):
        """Walk every window in waves of cells that double, all walks at
        once; each walk stops once the valid weights found leave, plus
        QP_WEIGHT_SUM_SLACK, no more of their sum (one) than the largest of
        them or than its window's `enough`."""
        size = 1
        while True:
            live = [wk for wk in walks if not wk.done]
            if not live:
                return
            chunk = {id(wk): wk.order[wk.pos:wk.pos + size] for wk in live}
            # the grid points the wave's cells end on
            need = []
            for wk in live:
                pts = sorted({i for c in chunk[id(wk)] for i in (c, c + 1)} - set(wk.f))
                need += [(wk, i) for i in pts]
            f, _, refused = self._eval([wk.slot for wk, _ in need],
                                       [wk.grid[i] for wk, i in need], False)
            for j, (wk, i) in enumerate(need):
                wk.f[i] = float(f[j])
                if j in refused:
                    wk.bad[i] = refused[j]
            cells = [((id(wk), c), wk.slot, wk.grid[c], wk.grid[c + 1], wk.f[c], wk.f[c + 1])
                     for wk in live for c in chunk[id(wk)]]
            brk, bad_split = self._brackets(cells)
            flat, owner = [], []
            for (key, slot, *_rest) in cells:
                for path, l, r, fl, fr in sorted(brk[key]):
                    flat.append((slot, l, r, fl, fr))
                    owner.append(key)
            roots, bad_root = self._roots(flat)
            per_cell = {}
            for k, key in enumerate(owner):
                per_cell.setdefault(key, []).append((flat[k][1], roots[k], bad_root[k]))
            # replay each walk in the reference's order up to where it stops
            for wk in live:
                for c in chunk[id(wk)]:
                    key = (id(wk), c)
                    for e in (wk.bad.get(c), wk.bad.get(c + 1), bad_split.get(key)):
                        if e is not None and wk.refusal is None:
                            wk.refusal = e
                    for l, got, e in per_cell.get(key, []):
                        if e is not None and wk.refusal is None:
                            wk.refusal = e
                        wk.found.append((l, got))
                        for _, z in got:
                            if _valid(z):
                                wk.weighed += z
                                wk.best = max(wk.best, z)
                    wk.pos += 1
                    if self.positive_weight and (
                            1.0 - wk.weighed + QP_WEIGHT_SUM_SLACK <= max(wk.best, wk.enough)):
                        wk.done = True
                        break
                if wk.pos >= len(wk.order):
                    wk.done = True
            size *= 2

    # -- following a root: the nearest valid root to it, every state in lockstep
    def _cells_of(self, items):
        """items: [(walk, cell)] -> {(id(walk), cell): [(l, r, fl, fr)]} with the
        grid points the cells end on evaluated first (kept on each walk)."""
        need = []
        for wk, c in items:
            need += [(wk, i) for i in (c, c + 1) if i not in wk.f and (wk, i) not in need]
        f, _, refused = self._eval([wk.slot for wk, _ in need], [wk.grid[i] for wk, i in need],
                                   False)
        for j, (wk, i) in enumerate(need):
            wk.f[i] = float(f[j])
            if j in refused:
                wk.bad[i] = refused[j]
        cells = [((id(wk), c), wk.slot, wk.grid[c], wk.grid[c + 1], wk.f[c], wk.f[c + 1])
                 for wk, c in items]
        brk, bad = self._brackets(cells)
        out = {}
        for (key, *_r), (wk, c) in zip(cells, items):
            for e in (wk.bad.get(c), wk.bad.get(c + 1), bad.get(key)):
                if e is not None and wk.refusal is None:
                    wk.refusal = e
            out[key] = [(l, r, fl, fr) for _, l, r, fl, fr in sorted(brk[key])]
        return out

    def follow_walk(self, walks):
        """Advance every walk ring by ring until each has stopped."""
        while True:
            items = []
            for wk in walks:
                if wk.done:
                    continue
                cells = wk.ring()
                if not cells:
                    wk.done = True
                    continue
                near = min(max(wk.grid[c] - wk.t, wk.t - wk.grid[c + 1], 0.0) for c in cells)
                if wk.best is not None and near > abs(wk.best[0] - wk.t):
                    wk.done = True
                    continue
                items += [(wk, c) for c in cells]
            if not items:
                return
            per_cell = self._cells_of(items)
            flat, owner = [], []
            for wk, c in items:
                for br in per_cell[(id(wk), c)]:
                    flat.append((wk.slot,) + br)
                    owner.append(wk)
            roots, bad = self._roots(flat)
            for k, wk in enumerate(owner):
                if bad[k] is not None and wk.refusal is None:
                    wk.refusal = bad[k]
                wk.solved[(flat[k][1], flat[k][2])] = roots[k]
                for w, z in roots[k]:
                    if _valid(z) and (wk.best is None or abs(w - wk.t) < abs(wk.best[0] - wk.t)):
                        wk.best = (w, z)
            for wk in {id(wk): wk for wk, _ in items}.values():
                wk.d += 1

    def _largest_beside(self, wk, a):
        """(w, Z) of the largest valid weight of the window beside a followed
        root below QP_WINDOW_Z_MIN: the brackets solved already as found, any
        other solved where the weight at its secant root (1/f' there) beats
        the largest so far; cells outward from a until the weights found
        leave no more of their sum than that (positive weight), or all."""
        top, weighed = wk.best, 0.0
        for got in wk.solved.values():
            for w, z in got:
                if _valid(z):
                    weighed += z
                    if z > top[1]:
                        top = (w, z)
        n = wk.grid.size - 1
        if self.positive_weight:
            c0 = min(max(int(np.searchsorted(wk.grid, a)) - 1, 0), n - 1)
            groups = [[c] for c in _walk_order(c0, n)]
        else:
            groups = [list(range(n))]
        for cells in groups:
            if self.positive_weight and 1.0 - weighed + QP_WEIGHT_SUM_SLACK <= top[1]:
                break
            per_cell = self._cells_of([(wk, c) for c in cells])
            for c in cells:
                for l, r, fl, fr in per_cell[(id(wk), c)]:
                    if (l, r) in wk.solved:
                        continue
                    x = l if l == r else l - fl * (r - l) / (fr - fl)
                    _, fp, _ = self._eval([wk.slot], [x], True)
                    z = 1.0 / fp[0] if fp[0] != 0.0 else np.nan
                    if not _valid(z) or z <= top[1]:
                        continue
                    got, _ = self._roots([(wk.slot, l, r, fl, fr)])
                    wk.solved[(l, r)] = got[0]
                    for w, zz in got[0]:
                        if _valid(zz):
                            weighed += zz
                            if zz > top[1]:
                                top = (w, zz)
        return top

    def follow(self, slots, bare, targets, rescan=True):
        """Per state: None where no window about its bare level holds a valid
        root near its target (``qp_equation.py:1155-1193``), else (w, Z,
        largest, refusal): the valid root nearest the target on the narrowest
        window that holds the target (a wider one while that root lies
        farther from the target than the window's edge), and beside it the
        largest valid weight of that window -- the root itself above
        QP_WINDOW_Z_MIN, else `_largest_beside`, or () with rescan off."""
        n = len(slots)
        res = [None] * n
        wins = [_windows(float(a)) for a in bare]

        def holding(i, start):
            return next((k for k in range(start, len(wins[i]))
                         if wins[i][k][0] <= targets[i] <= wins[i][k][1]), None)
        level = [holding(i, 0) for i in range(n)]
        pending = [i for i in range(n) if level[i] is not None]
        while pending:
            walks = [_FollowWalk(slots[i], targets[i], *wins[i][level[i]]) for i in pending]
            self.follow_walk(walks)
            nxt = []
            for i, wk in zip(pending, walks):
                last = level[i] + 1 == len(wins[i])
                t = float(targets[i])
                if wk.best is not None and (abs(wk.best[0] - t) <= min(t - wk.lo, wk.hi - t)
                                            or last):
                    if _valid(wk.best[1], QP_WINDOW_Z_MIN):
                        largest = wk.best
                    else:
                        largest = self._largest_beside(wk, float(bare[i])) if rescan else ()
                    res[i] = (wk.best[0], wk.best[1], largest, wk.refusal)
                    continue
                k = holding(i, level[i] + 1)
                if k is not None:
                    level[i] = k
                    nxt.append(i)
            pending = nxt
        return res

    def solve(self, slots, bare):
        """Per state: (w, Z, refusal, found roots of its last window), the
        root of largest valid weight in the narrowest window that holds one
        above QP_WINDOW_Z_MIN; a state without one keeps its widest window's
        largest valid weight, or the root nearest its bare level."""
        n = len(slots)
        out = [None] * n
        pending = list(range(n))
        wins = [_windows(float(a)) for a in bare]
        level = [0] * n
        refusal = [None] * n
        found = [[] for _ in range(n)]
        while pending:
            walks = []
            for i in pending:
                lo, hi = wins[i][level[i]]
                last = level[i] + 1 == len(wins[i])
                walks.append(_Walk(slots[i], float(bare[i]), lo, hi,
                                   -np.inf if last else QP_WINDOW_Z_MIN))
            self.walk(walks)
            nxt = []
            for i, wk in zip(pending, walks):
                if wk.refusal is not None and refusal[i] is None:
                    refusal[i] = wk.refusal
                wk.found.sort(key=lambda lr: lr[0])
                found[i] = [rz for _, got in wk.found for rz in got]
                ok = [k for k, (_, z) in enumerate(found[i]) if _valid(z)]
                if ok:
                    k = max(ok, key=lambda j: found[i][j][1])
                    if _valid(found[i][k][1], QP_WINDOW_Z_MIN):
                        out[i] = (found[i][k][0], found[i][k][1], True)
                        continue
                if level[i] + 1 < len(wins[i]):
                    level[i] += 1
                    nxt.append(i)
            pending = nxt
        result = []
        for i in range(n):
            if out[i] is not None:
                result.append((out[i][0], out[i][1], None, found[i]))
                continue
            if refusal[i] is not None:
                result.append((np.nan, np.nan, refusal[i], found[i]))
                continue
            if not found[i]:
                result.append((np.nan, np.nan, None, found[i]))
                continue
            ok = [k for k, (_, z) in enumerate(found[i]) if _valid(z)]
            k = (max(ok, key=lambda j: found[i][j][1]) if ok
                 else min(range(len(found[i])), key=lambda j: abs(found[i][j][0] - bare[i])))
            result.append((found[i][k][0], found[i][k][1], None, found[i]))
        return result


def _report_root(w, z, refusal, bare, label):
    """Raise the refusal of a state without a quasiparticle, warn for no root
    or for Z outside (0, 1], as ``qp_equation.py:236-273`` does."""
    from .gw import QPNoRoot, QPWeightOutside
    if refusal is not None:
        raise refusal
    if not np.isfinite(w):
        lo, hi = _windows(bare)[-1]
        warnings.warn(f'{label or "the quasiparticle equation"} has no root in the widest '
                      f'scan window [{lo:.6f}, {hi:.6f}] Ha about {bare:.6f} Ha.', QPNoRoot,
                      stacklevel=3)
    elif not 0.0 < z <= 1.0:
        warnings.warn(f'the quasiparticle root of {label or "the quasiparticle equation"} '
                      f'{w!r} Ha has Z = {z!r}, outside (0, 1]: kept', QPWeightOutside,
                      stacklevel=3)


def _branch_flipped(w, z, largest, followed, tol):
    """Whether a followed root is not the largest weight here
    (``qp_equation.py:145-152``): its branch has gone, or another root more
    than tol away carries more weight."""
    if followed is None:
        return False
    return (not followed) or (largest is not None and abs(largest[0] - w) > tol
                              and largest[1] > z)


def _scan_one(equation, a, follow=None, tol=QP_ROOT_TOL, max_iter=QP_ROOT_MAX_ITER, label='',
              out=None, positive_weight=True, rescan=True):
    """(w, Z) of one equation (the scan's protocol) about the bare level a,
    optionally following a previous root (``qp_equation.py:155-237, 342-356``):
    the valid root nearest it where a window holds one, else the largest
    weight again (its branch has gone). out: a dict that receives the branch
    ('labels', 'largest', 'followed', 'flipped', 'no_root', 'z_outside');
    without it a warning where the largest weight has left the followed
    root."""
    from .gw import QPNoRoot, QPWeightOutside
    scan = _LockstepScan(equation, tol, max_iter, positive_weight)
    what = label or 'the quasiparticle equation'
    largest = followed = None
    if follow is None:
        (w, z, refusal, _), = scan.solve([0], [float(a)])
        _report_root(w, z, refusal, float(a), label)
    else:
        target = float(follow[0] if isinstance(follow, (tuple, list)) else follow)
        got = scan.follow([0], [float(a)], [target], rescan)[0]
        if got is not None:
            w, z, largest, _ = got
            largest, followed = (largest or None), True
        else:
            (w, z, refusal, _), = scan.solve([0], [float(a)])
            if refusal is not None:
                raise refusal
            if not np.isfinite(w):
                lo, hi = _windows(float(a))[-1]
                warnings.warn(f'{what}: the branch followed from {target:.6f} Ha has gone and '
                              f'no root lies in the widest scan window [{lo:.6f}, {hi:.6f}] '
                              f'Ha about {float(a):.6f} Ha.', QPNoRoot, stacklevel=3)
            largest, followed = (float(w), float(z)), False
        if np.isfinite(w) and not 0.0 < z <= 1.0:
            warnings.warn(f'the quasiparticle root of {what} {w!r} Ha has Z = {z!r}, outside '
                          f'(0, 1]: kept', QPWeightOutside, stacklevel=3)
    w, z = float(w), float(z)
    flipped = _branch_flipped(w, z, largest, followed, tol)
    if out is not None:
        out.update(labels=None, largest=largest, followed=followed, flipped=flipped,
                   no_root=not np.isfinite(w),
                   z_outside=bool(np.isfinite(w) and not 0.0 < z <= 1.0))
    elif flipped:
        if not followed:
            msg = (f'{what}: the branch the previous geometry kept has gone; the root of '
                   f'largest weight is kept again, {w:.10f} Ha (Z = {z:.4f}).')
        else:
            msg = (f'{what}: the followed root {w:.10f} Ha has Z = {z:.4f}; the largest '
                   f'weight is now {largest[1]:.4f} at {largest[0]:.10f} Ha; the branch is '
                   f'kept.')
        warnings.warn(msg, RuntimeWarning, stacklevel=3)
    return w, z


def solve_qp_equation_scan(residual, fprime, a, follow=None, tol=QP_ROOT_TOL,
                           max_iter=QP_ROOT_MAX_ITER, label='', refusals=(), out=None,
                           positive_weight=False, rescan=True):
    """(w, Z) of residual(w) = 0 for a self-energy known pointwise,
    residual and fprime host callables (``qp_equation.py:1396-1420``).
    Points where either raises one of `refusals` count as unknown. No
    quasiparticle where the self-energy could be evaluated raises the first
    refusal; no root at all is (NaN, NaN) with a QPNoRoot warning; a root
    with Z outside (0, 1] is kept with a QPWeightOutside warning.
    positive_weight: Sigma a sum of poles of positive weight (a bracket
    where f falls is a pole; the walk ends once the weights found leave no
    more), else every bracket of a window is solved. follow, out, rescan:
    a previous root to follow, the dict its branch goes to, and whether a
    weak followed root's window is searched for the largest weight beside
    it (`_scan_one`)."""
    refusals = tuple(refusals)

    def equation(slots, w, want_slope):
        f = np.empty(len(w))
        fp = np.full(len(w), np.nan)
        bad = {}
        for j, x in enumerate(w):
            try:
                f[j] = residual(float(x))
                if want_slope:
                    fp[j] = fprime(float(x))
            except refusals as e:
                f[j], fp[j] = np.nan, np.nan
                bad[j] = e
        return f, fp, bad
    return _scan_one(equation, a, follow, tol, max_iter, label, out, positive_weight, rescan)


def _contour_equation_callable(eq):
    """Adapt a ContourEquation to the scan's (f, f', refusals) protocol."""
    def equation(slots, w, want_slope):
        f, fp, refused = eq(slots, w, want_slope)
        bad = {}
        for j in np.nonzero(refused)[0]:
            try:
                eq.backend._refuse(np.abs(eq.eps - w[j])[
                    residue_weights(eq.eps, eq.nocc, [w[j]])[0] != 0])
            except ResidueRefused as e:
                bad[int(j)] = e
        return f, fp, bad
    return equation


def solve_contour_roots(eq, labels=None, tol=QP_ROOT_TOL, max_iter=QP_ROOT_MAX_ITER,
                        warn=True):
    """(roots, Z, refusals) of every slot of a ContourEquation, all states'
    searches in lockstep. warn: report no-root / Z-outside per state (a
    refusal is returned, not raised)."""
    n = len(eq.bare)
    scan = _LockstepScan(_contour_equation_callable(eq), tol, max_iter)
    res = scan.solve(list(range(n)), eq.bare)
    roots = np.array([r[0] for r in res], float)
    zs = np.array([r[1] for r in res], float)
    refusals = [r[2] for r in res]
    if warn:
        for i, (w, z, e, _) in enumerate(res):
            if e is None:
                _report_root(w, z, None, float(eq.bare[i]),
                             labels[i] if labels is not None else '')
    eq.rounds = scan.rounds
    return roots, zs, refusals


# ------------------------------------------- the reference's per-state seams

def _host_or_device_wc(Bp, eps, nocc, nu_points, wbp, wc, C_ov):
    """The state's contracted screening wc (nfreq, norb): given, contracted
    from W B_p (wbp), or built explicitly from C_ov (`wc_explicit`)."""
    if wc is None:
        if wbp is not None:
            Bh = Bp.detach().cpu().numpy() if isinstance(Bp, torch.Tensor) else np.asarray(Bp)
            wc = screening_contraction(Bh, wbp)
        else:
            require_three_index(C_ov, 'the imaginary-axis screening without wbp or wc')
            wc = wc_explicit(Bp, C_ov, ov_energies(eps, nocc), nu_points)
    return wc


def _one_state_equation(p, Bp, eps, nocc, nu_points, nu_weights, xc_correction, wbp, wc,
                        C_ov, eta, real_screening):
    eps = np.asarray(eps, float)
    wc = _host_or_device_wc(Bp, eps, nocc, nu_points, wbp, wc, C_ov)
    backend = (residue_backend(real_screening, C_ov, eps, nocc, eta)
               if real_screening is not None or C_ov is not None else None)
    quad = LorentzianQuadrature(nu_points, nu_weights)
    return ContourEquation(Bp, wc, eps, nocc, quad,
                           [float(eps[p]) + float(xc_correction)], backend)


def sigma_cd(p, omega, Bp, eps, nocc, nu_points, nu_weights, residues=None, wbp=None,
             eta=0.0, wc=None, C_ov=None, real_screening=None):
    """Sigma^c_pp(omega) by contour deformation (``contour_deformation.py:310-343``)
    from the state's slice Bp and its contracted screening (wc, or W Bp as
    wbp, or -- with neither -- built explicitly from C_ov); the residues at
    omega unless `residues` [(q, weight)] fixes them, their W from
    `real_screening` (a LaplaceRealScreening or ExplicitRealScreening) or,
    with C_ov and no backend, the explicit one."""
    eq = _one_state_equation(p, Bp, eps, nocc, nu_points, nu_weights, 0.0, wbp, wc, C_ov,
                             eta, real_screening)
    if eq.backend is not None:
        eq.backend._refuse(_residue_frequencies(eq, float(omega), residues))
    s, _, _ = eq.sigma([0], [float(omega)], want_slope=False, residues=residues)
    return float(s[0])


def _residue_frequencies(eq, omega, residues):
    if residues is None:
        r = residue_weights(eq.eps, eq.nocc, [omega])[0]
        return np.abs(eq.eps[r != 0] - omega)
    return np.array([abs(eq.eps[q] - omega) for q, _ in residues])


def sigma_cd_slope(p, omega, Bp, eps, nocc, nu_points, nu_weights, residues, wc, eta=0.0,
                   C_ov=None, real_screening=None):
    """dSigma^c_pp/domega in closed form at a frozen residue set
    (``contour_deformation.py:346-373``)."""
    eq = _one_state_equation(p, Bp, eps, nocc, nu_points, nu_weights, 0.0, None, wc, C_ov,
                             eta, real_screening)
    if residues and eq.backend is not None:
        eq.backend._refuse(_residue_frequencies(eq, float(omega), residues))
    _, ds, _ = eq.sigma([0], [float(omega)], want_slope=True, residues=residues or [])
    return float(ds[0])


def qp_energy_cd(p, Bp, eps, nocc, nu_points, nu_weights, xc_correction=0.0, tol=QP_ROOT_TOL,
                 max_iter=QP_ROOT_MAX_ITER, follow=None, wbp=None, wc=None, C_ov=None,
                 eta=0.0, real_screening=None, branch=None, rescan=True):
    """(eps^QP_p, Z_p, residues) of w = eps_p + xc_correction + Sigma^c(w) by
    contour deformation (``contour_deformation.py:376-436``): the lockstep
    scan about the bare level with the residues re-decided at every point,
    the residue set of the root returned. Screening and backend as
    `sigma_cd`. follow, branch, rescan: a walk's previous root (the root
    nearest it is kept, whatever its weight), the dict its branch goes to,
    and whether a weak followed root's window is searched for the largest
    weight beside it."""
    eq = _one_state_equation(p, Bp, eps, nocc, nu_points, nu_weights, xc_correction, wbp, wc,
                             C_ov, eta, real_screening)
    if follow is None and branch is None:
        roots, zs, refusals = solve_contour_roots(eq, [f'orbital {p}'], tol, max_iter)
        if refusals[0] is not None:
            raise refusals[0]
        w = float(roots[0])
        return w, float(zs[0]), residue_set(eps, nocc, w)
    w, z = _scan_one(_contour_equation_callable(eq), eq.bare[0], follow, tol, max_iter,
                     f'orbital {p}', branch, True, rescan)
    return w, z, residue_set(eps, nocc, w)


def residue_backend(real_screening, C_ov, eps, nocc, eta):
    """The backend the residue term uses: the one given, else the explicit one
    from C_ov (``contour_deformation.py:117-122``)."""
    if real_screening is not None:
        return real_screening
    require_three_index(C_ov, 'the residue term')
    return ExplicitRealScreening(C_ov, eps, nocc, eta)


def require_three_index(C_ov, what):
    """``contour_deformation.py:109-114``."""
    if C_ov is None:
        raise ResidueRefused(
            f'{what} needs C_ov = B[:, occ, virt] as (naux, nocc*nvirt) and it was not '
            f'supplied. A frontier state sweeps no residues and needs none once the '
            f'imaginary-axis screening comes in as wbp or wc.')


HARTREE_TO_EV = 27.211386245988  # MBPTcode constants.py:11 (CODATA 2018)


def _admission(eps, nocc, states, continuation, pairs=None):
    """(start points, [(admits, reach)]) of the states: each judged at eps_p
    moved 1 mHa toward the chemical potential by the pole model's compression
    condition, which 'sop' enforces before anything is built
    (``contour_deformation.py:690-703``)."""
    from . import sum_over_poles as sop
    starts = np.array([sop.qp_start(eps, int(p), nocc) for p in states])
    admission = [sop.compressible(float(w), eps, nocc, pair_energies=pairs) for w in starts]
    if continuation == 'sop':
        for p, start, (admits, reach) in zip(states, starts, admission):
            if not admits:
                raise ValueError(
                    f"continuation='sop' cannot serve orbital {int(p)}: its start point "
                    f'{start:.4f} Ha sweeps a pole {reach:.3f} particle-hole gaps away, and '
                    'the pole model converges only below one (beyond it single excitations '
                    "of W matter, not their envelope); use continuation='cd'.")
    return starts, admission


def _sop_roots(states, wcs, eps, nocc, nu, xc, n_poles, sop_stride, pairs):
    """Each state's root and Z on its pole model, fitted to its wc."""
    from . import sum_over_poles as sop
    roots, zs, poles_of = np.zeros(len(states)), np.zeros(len(states)), []
    for i, p in enumerate(states):
        wc = wcs[i].detach().cpu().numpy() if torch.is_tensor(wcs[i]) else np.asarray(wcs[i])
        poles, amp = sop.sop_from_wc(wc, nu, eps, nocc, n_poles=n_poles, stride=sop_stride,
                                     pair_energies=pairs, state=int(p))
        roots[i], zs[i] = sop.qp_energy_sop(int(p), amp, poles, eps, nocc,
                                            xc_correction=float(xc[i]))
        poles_of.append(poles)
    return roots, zs, poles_of


def _roots_on_contour(continuation, states, B, wcs, eps, nocc, nu, nu_w, xc_correction,
                      backend, w0, ntau, nfreq_cd, starts=None, admission=None, n_poles=None,
                      sop_stride=None, pairs=None):
    """Every state's root and Z on one contour grid, all states' scans in
    lockstep (or each on its pole model, 'sop'), with the per-state records
    (``contour_deformation.py:558-598``)."""
    explicit = continuation == 'cd'
    xc = np.broadcast_to(np.asarray(xc_correction, float).ravel()
                         if np.ndim(xc_correction) else float(xc_correction),
                         (len(states),))
    if starts is None:
        starts, admission = _admission(eps, nocc, states, continuation, pairs)
    if continuation == 'sop':
        from . import sum_over_poles as sop
        roots, zs, poles_of = _sop_roots(states, wcs, eps, nocc, nu, xc,
                                         n_poles or sop.SOP_N_POLES,
                                         sop.SOP_FIT_STRIDE if sop_stride is None else sop_stride,
                                         pairs)
        records = [{'state': int(p), 'qp_start': float(starts[i]), 'residues': 0,
                    'representation_error': None, 'sop_admits': bool(admission[i][0]),
                    'sop_reach': float(admission[i][1]), 'sop_poles': poles_of[i]}
                   for i, p in enumerate(states)]
        info = {'continuation': 'sop', 'ntau': int(ntau), 'nfreq_cd': int(nfreq_cd),
                'w0_cd': float(w0), 'residue_route_taken': 'sop', 'states': records}
        return roots, zs, info
    wc = torch.stack([to_device(w, B.device) for w in wcs])
    eq = ContourEquation(B, wc, eps, nocc, LorentzianQuadrature(nu, nu_w),
                         eps[states] + xc, backend)
    roots, zs, refusals = solve_contour_roots(eq, [f'orbital {int(p)}' for p in states])
    records = []
    for i, p in enumerate(states):
        if refusals[i] is not None:
            if explicit:
                raise refusals[i]
            raise ResidueRefused(
                f"continuation='laplace' cannot serve orbital {int(p)}: its contour sweeps "
                f'a residue the imaginary-time grid does not represent. {refusals[i]}'
            ) from refusals[i]
        res = residue_set(eps, nocc, roots[i])
        error = None
        if not explicit and res:
            error = float(backend.errors([abs(eps[q] - roots[i]) for q, _ in res]).max())
        records.append({'state': int(p), 'qp_start': float(starts[i]), 'residues': len(res),
                        'representation_error': error, 'sop_admits': bool(admission[i][0]),
                        'sop_reach': float(admission[i][1])})
    info = {'continuation': continuation, 'ntau': int(ntau), 'nfreq_cd': int(nfreq_cd),
            'w0_cd': float(w0), 'residue_route_taken': 'explicit' if explicit else 'laplace',
            'states': records, 'points_evaluated': int(eq.points),
            'evaluation_rounds': int(getattr(eq, 'rounds', 0)),
            'residue_solves': dict(getattr(backend, 'stats', {}))}
    return roots, zs, info


def contour_roots(X, D, eps, nocc, states, ntau=CD_NTAU, nfreq_cd=CD_NFREQ, w0_cd=None,
                  e_min_below_gap=None, xc_correction=0.0, mu=None, continuation='laplace',
                  precision='fp64', n_poles=None, sop_stride=None):
    """(roots in Hartree, Z, per-state records) of the states on one contour
    grid (``contour_deformation.py:558-598, 767-812``): one proj(tau) and one
    W per frequency serve every state's imaginary-axis term, each state's
    root by `qp_energy_cd`. The residues read W at real frequencies from the
    cosh transform of the same proj(tau) (continuation 'laplace', which
    refuses a state whose residues the time grid does not carry) or from the
    explicit particle-hole response of C_ov (continuation 'cd', any state);
    'sop' models W on the imaginary axis by n_poles fitted poles instead
    (`sum_over_poles`), Sigma closed form and no real-frequency screening,
    and refuses the states the compression condition excludes before
    anything is built. xc_correction: the static term, one per state or one
    for all. precision 'mixed' runs the screening contraction and the
    explicit response as split tensor-core products (the Dyson steps and the
    Laplace residues stay FP64)."""
    if continuation not in ('laplace', 'cd', 'sop'):
        raise ValueError(f"continuation={continuation!r}: choose 'cd', 'laplace' or 'sop'")
    eps = _eps_host(eps)
    states = np.atleast_1d(np.asarray(states, int))
    starts, admission = _admission(eps, nocc, states, continuation)
    explicit = (ExplicitRealScreening(three_index_ov(X, D, eps, nocc), eps, nocc,
                                      precision=precision)
                if continuation == 'cd' else None)
    nu, nu_w, grid, w0 = cd_frequency_grid(eps, nocc, ntau=ntau, nfreq_cd=nfreq_cd,
                                           w0_cd=w0_cd, e_min_below_gap=e_min_below_gap)
    proj = polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    B = three_index_slices(X, D, states)
    wcs = cd_screening_contraction_multi(proj, grid.cosft_wt, list(B), precision=precision)
    backend = (explicit if explicit is not None else None if continuation == 'sop'
               else LaplaceRealScreening(proj, grid, eps, nocc))
    del proj
    return _roots_on_contour(continuation, states, B, wcs, eps, nocc, nu, nu_w, xc_correction,
                             backend, w0, ntau, nfreq_cd, starts, admission, n_poles,
                             sop_stride)


def contour_roots_unrestricted(X_mos, D, spectra, noccs, spin, states, ntau=CD_NTAU,
                               nfreq_cd=CD_NFREQ, w0_cd=None, e_min_below_gap=None,
                               xc_correction=0.0, continuation='laplace', precision='fp64',
                               n_poles=None, sop_stride=None):
    """`contour_roots` for one spin channel of an unrestricted reference
    (``contour_deformation.py:686-812``): both spins' pair energies side by
    side set the contour grid, proj(tau) is the spin sum (half of each spin's
    restricted sweep at its own mid-gap), the channel's slices and contraction
    read it, and the residues come from its cosh transform on those pair
    energies ('laplace') or from both spins' C_ov side by side at 1/sqrt(2),
    so that the restricted factor 2 counts every pair once ('cd'), or the
    channel's pole model with its bounds and compression test on both spins'
    pair energies ('sop'). spin: 0 (alpha) or 1 (beta); states are the
    channel's orbitals."""
    if continuation not in ('laplace', 'cd', 'sop'):
        raise ValueError(f"continuation={continuation!r}: choose 'cd', 'laplace' or 'sop'")
    if len(X_mos) != 2 or len(spectra) != 2 or len(noccs) != 2 or spin not in (0, 1):
        raise ValueError('an unrestricted contour takes two spin channels and spin 0 or 1')
    from .space_time import spin_summed
    spectra = [_eps_host(e) for e in spectra]
    noccs = [int(n) for n in noccs]
    pairs = np.concatenate([ov_energies(e, n) for e, n in zip(spectra, noccs)])
    eps, nocc = spectra[spin], noccs[spin]
    states = np.atleast_1d(np.asarray(states, int))
    starts, admission = _admission(eps, nocc, states, continuation, pairs)
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
    backend = (explicit if explicit is not None else None if continuation == 'sop'
               else LaplaceRealScreening(proj, grid, eps, nocc, pair_energies=pairs))
    del proj
    return _roots_on_contour(continuation, states, B, wcs, eps, nocc, nu, nu_w, xc_correction,
                             backend, w0, ntau, nfreq_cd, starts, admission, n_poles,
                             sop_stride, pairs)


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
    pole model: numerics.qp.n_poles poles, every numerics.qp.sop_stride-th
    orbital's wc in the fit) refuses the states the compression condition
    excludes. precision: as `contour_roots`."""
    if continuation not in ('cd', 'laplace', 'sop'):
        raise ValueError(f"solve_qp_energy_contour runs continuation='cd', 'laplace' or "
                         f"'sop', not {continuation!r}")
    if factors is None:
        raise NotImplementedError('building the ISDF factors needs pyscf (integrals and the '
                                  'fit); pass factors=(X_mo, D)')
    eps = np.asarray(getattr(mf, 'mo_energy', mf), float)
    ntau, nfreq = CD_NTAU, CD_NFREQ
    n_poles = sop_stride = None
    if numerics is not None:
        q = numerics.quadrature
        ntau = getattr(q, 'ntau_cd', ntau)
        nfreq = getattr(q, 'nfreq_cd', nfreq)
        qp = getattr(numerics, 'qp', None)
        n_poles = getattr(qp, 'n_poles', None)
        sop_stride = getattr(qp, 'sop_stride', None)
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
            precision=precision, n_poles=n_poles, sop_stride=sop_stride)
        return roots * HARTREE_TO_EV, zs, info
    if eps_anchor is not None:
        xc = xc + (np.asarray(eps_anchor, float)[states] - eps[states])
    roots, zs, info = contour_roots(X, D, eps, nocc, states, ntau=ntau, nfreq_cd=nfreq,
                                    w0_cd=w0_cd, xc_correction=xc, continuation=continuation,
                                    precision=precision, n_poles=n_poles, sop_stride=sop_stride)
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


def _explicit_residue_backward(X, D, eps, nocc, pushes, X_bar, D_bar):
    """The explicit residues' share of (eps_bar, X_bar, D_bar): each residue
    at real frequency f puts c y y^T on chi0(f) = 2 C diag(fac) C^T, C[:, (i,a)]
    = D^T (x_i o x_a), so C_bar = y g^T with g = 4 c fac o (C^T y) -- rank one
    -- and the chain to (X, D) needs C^T y = X_o^T diag(D y) X_v alone:
    D_bar += u y^T with u = rowsum(X_o o (X_v G^T)), X_bar[:, occ] +=
    diag(D y) X_v G^T, X_bar[:, virt] += diag(D y) X_o G, and fac's slope in
    the pair energies gives eps (``gradients/gwbse/contour_deformation_adjoint.py:
    52-77, 149-166``, three_index_ov's reverse; C_bar never formed). X_bar and
    D_bar are added to in place; returns the eps adjoint (host)."""
    dev = X_bar.device
    Xd, Dd = to_device(X, dev), to_device(D, dev)
    Xo, Xv = Xd[:, :nocc], Xd[:, nocc:]
    dpair = (eps[nocc:][None, :] - eps[:nocc][:, None])
    eps_bar = np.zeros(len(eps))
    for f, y, c in pushes:
        Dy = Dd @ y
        t = (Xo * Dy[:, None]).T @ Xv                        # C^T y, (nocc, nvirt)
        fac, dfac, _ = frequency_factor(dpair, f, False, slopes=True)
        th = t.cpu().numpy()
        d_bar = 2.0 * c * th * th * dfac
        eps_bar[nocc:] += d_bar.sum(axis=0)
        eps_bar[:nocc] -= d_bar.sum(axis=1)
        G = torch.as_tensor(4.0 * c * fac, device=dev) * t
        XvG = Xv @ G.T                                       # (M, nocc)
        D_bar += torch.outer((Xo * XvG).sum(dim=1), y)
        X_bar[:, :nocc] += Dy[:, None] * XvG
        X_bar[:, nocc:] += Dy[:, None] * (Xo @ G)
    return eps_bar


EXPLICIT_RESIDUE_MAX_GB = 256.0   # MBPTcode src/Base/numerics/constants.py:1261


def _gradient_route(residue_route, scissor, p, eps, nocc, w0, sop_poles, naux):
    """(route, shift) of orbital p in the QP gradient
    (``gradients/gwbse/qp_space_time.py:162-217``, ``GW/qp_states.py:
    323-338``): 'sop' keeps the pole model for a state the compression test
    admits at its start (the frozen root, else eps_p moved toward the
    chemical potential) or that sop_poles froze onto it; a frozen scissor
    shift (a mapping per orbital, or one number for the states the test
    excludes) takes 'scissor'; any other falls back to 'explicit' where C_ov
    fits in EXPLICIT_RESIDUE_MAX_GB, else 'laplace'. Other routes as asked."""
    if residue_route != 'sop':
        return residue_route, None
    from . import sum_over_poles as sop
    root = _frozen_root(w0, p)
    start = sop.qp_start(eps, p, nocc) if root is None else root
    shift = None
    if scissor is not None and not isinstance(scissor, str):
        shift = (scissor.get(int(p)) if isinstance(scissor, dict) else float(scissor))
        shift = None if shift is None else float(shift)
    if isinstance(scissor, dict):
        route = 'scissor' if shift is not None else 'sop'
    elif shift is not None and not isinstance(scissor, str) and \
            not sop.compressible(start, eps, nocc)[0]:
        route = 'scissor'
    else:
        route = 'sop'
    if isinstance(sop_poles, dict) and sop_poles.get(int(p)) is not None:
        admitted = True
    elif isinstance(w0, dict) and w0.get(int(p)) is not None:
        admitted = False
    else:
        admitted = sop.compressible(start, eps, nocc)[0]
    if route == 'sop' and not admitted:
        nvir = len(eps) - nocc
        route = ('explicit' if naux * nocc * nvir * 8 / 1e9 <= EXPLICIT_RESIDUE_MAX_GB
                 else 'laplace')
    return route, shift


def _frozen_root(w0, p):
    """The root a reference geometry kept for orbital p: w0 a number or a
    mapping orbital -> root; None before one is kept
    (``gradients/gwbse/qp_space_time.py:102-114``)."""
    if isinstance(w0, dict):
        got = w0.get(int(p))
        return None if got is None else float(got)
    return None if w0 is None else float(w0)


def _followed_branch(follow, w0, p):
    """(w, labels) orbital p follows here: the branch `follow` (a mapping
    orbital -> (w, labels)) names, else the frozen root by energy, else None
    (``qp_space_time.py:137-150``)."""
    got = follow.get(int(p)) if isinstance(follow, dict) else None
    if got is not None:
        w, labels = got
        return float(w), (None if labels is None else tuple(labels))
    root = _frozen_root(w0, p)
    return None if root is None else (root, None)


def _rescans_beside(z0, p):
    """Whether a weak followed root of p has its window searched for the
    largest weight beside it: unless the reference root's Z (z0, a mapping
    orbital -> Z) was no quasiparticle's either (``qp_space_time.py:124-134``)."""
    z = z0.get(int(p)) if isinstance(z0, dict) else None
    return z is None or _valid(z, QP_WINDOW_Z_MIN)


def qp_gradient_space_time(X, D, eps, nocc, grid, nu_points, nu_weights, p, *,
                           residue_route='laplace', mu=None, xc_correction=0.0, w0=None,
                           tol=QP_ROOT_TOL, laplace_tol=LAPLACE_SCREENING_TOL, want_grad=True,
                           tile_gb=None, follow=None, route_out=None, n_poles=None,
                           sop_stride=None, scissor=None, sop_poles=None, comm=None, z0=None):
    """(eps^QP_p, Z, eps_bar, X_bar, D_bar), or (eps^QP_p, Z) with want_grad
    False: the contour-deformation QP energy of state p and its gradient in
    (eps, X, D) (``gradients/gwbse/qp_space_time.py:412-452``), residues by
    the cosh transform of proj(tau) on `grid` (residue_route 'laplace'; the
    contour's time grid, mu frozen) or from C_ov ('explicit': each residue's
    rank-one adjoint on chi0 taken back to (eps, X, D) through C_ov's
    definition without forming its adjoint). The root is differentiated implicitly, d eps^QP = Z [d eps_p +
    dSigma^c(w)|_w], the residue set frozen at the root: the integral term's
    adjoint goes to the slice, to W(i nu) (then W W_bar W onto chi0 and
    proj(tau)) and to eps through its weights; each residue's to the slice,
    to chi0 at its real frequency (folded onto proj(tau) by the cosh weights)
    and to eps through its frequency; then the chi0 sweep's and the slice's
    reverses. FP64 on the device; arrays come back as X is held.
    w0, follow, z0: a walk's frozen root (followed by energy), the branch
    the last accepted geometry kept ({p: (w, labels)}), and the reference
    roots' Z ({p: Z}, whether a weak followed root's window is rescanned);
    route_out receives 'residue_route', 'residues', 'weights', 'roots',
    'labels', 'branches' and 'sop_poles'. residue_route 'sop': the root on
    the state's pole model (n_poles fitted to wc at sop_stride, or the
    frozen poles sop_poles[p] of a reference geometry), differentiated at
    fixed poles, where the amplitudes A = F^+ wc are linear in wc: the
    adjoint on wc is Z (F^+)^T (1/D)^T and takes the integral term's chain
    (``gradients/gwbse/sum_over_poles_adjoint.py:24-47``); no residues."""
    if residue_route not in ('laplace', 'explicit', 'sop'):
        raise NotImplementedError(f'residue_route={residue_route!r}: the device route serves '
                                  "'laplace' (the cubic residues), 'explicit' (C_ov) and 'sop' "
                                  '(the pole model)')
    if comm is not None:
        raise NotImplementedError('rank splits are outside the one-GPU route')
    dev = require_device()
    eps_h = _eps_host(eps)
    p = int(p)
    if mu is None:
        mu = particle_hole_window(eps_h, nocc)[2]
    proj = polarizability_tau(X, D, eps_h, nocc, grid, mu=mu)
    wmi, _ = screening_minus_identity(proj, grid.cosft_wt)
    B = three_index_slices(X, D, [p])[0]
    wc = screening_contraction_device(wmi, [B])[0]
    followed, branch = _followed_branch(follow, w0, p), {}
    residue_route, shift = _gradient_route(residue_route, scissor, p, eps_h, nocc, w0,
                                           sop_poles, B.shape[0])
    if residue_route == 'scissor':
        # a frozen shift: the root moves with eps_p alone
        w, z = float(eps_h[p] + xc_correction + shift), 1.0
        if route_out is not None:
            route_out.update(residue_route='scissor', residues=[], weights={p: z},
                             roots={p: w}, labels={p: None}, branches={}, sop_poles={})
        if not want_grad:
            return w, z
        eps_bar = np.zeros(len(eps_h))
        eps_bar[p] = z
        if isinstance(X, torch.Tensor):
            return (w, z, torch.as_tensor(eps_bar, device=dev),
                    torch.zeros_like(to_device(X, dev)), torch.zeros_like(to_device(D, dev)))
        return w, z, eps_bar, np.zeros(np.shape(X)), np.zeros(np.shape(D))
    if residue_route == 'sop':
        from . import sum_over_poles as sop
        wc_h = wc.cpu().numpy()
        frozen = None if sop_poles is None else sop_poles.get(p)
        if frozen is None:
            poles, amp = sop.sop_from_wc(wc_h, nu_points, eps_h, nocc,
                                         n_poles=n_poles or sop.SOP_N_POLES,
                                         stride=(sop.SOP_FIT_STRIDE if sop_stride is None
                                                 else sop_stride), state=p)
        else:
            poles = np.asarray(frozen, float)
            amp = sop.pole_amplitudes(wc_h, poles, nu_points)
        w, z = sop.qp_energy_sop(p, amp, poles, eps_h, nocc, xc_correction=xc_correction,
                                 tol=tol, follow=followed, branch=branch)
        res = []
    else:
        lap = (LaplaceRealScreening(proj, grid, eps_h, nocc, tol=laplace_tol)
               if residue_route == 'laplace' else
               ExplicitRealScreening(three_index_ov(X, D, eps_h, nocc), eps_h, nocc))
        w, z, res = qp_energy_cd(p, B, eps_h, nocc, nu_points, nu_weights,
                                 xc_correction=xc_correction, tol=tol, wc=wc, real_screening=lap,
                                 follow=followed, branch=branch, rescan=_rescans_beside(z0, p))
    if route_out is not None:
        route_out.update(residue_route=residue_route, residues=res, weights={p: float(z)},
                         roots={p: float(w)}, labels={p: branch.get('labels')},
                         branches={p: branch} if followed is not None else {},
                         sop_poles={p: poles} if residue_route == 'sop' else {})
    if not want_grad:
        return w, z
    naux, norb = B.shape
    eps_bar = np.zeros(norb)
    eps_bar[p] += z
    if residue_route == 'sop':
        den = sop.denominators(w, poles, eps_h, nocc)              # (norb, M)
        eps_bar += z * np.sum(amp.T / (den * den), axis=1)
        wc_bar = torch.as_tensor(z * (sop.pole_pseudoinverse(nu_points, poles).T @ (1.0 / den).T),
                                 dtype=torch.float64, device=dev)
    else:
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
    check(lib().mbpt_dyson_backward(ptr(wmi), ptr(W_bar), naux, wmi.shape[0], MODES['fp64'],
                                    ptr(wsd), wsd.numel(), stream_ptr()),
          'mbpt_dyson_backward')
    cw_t = np.ascontiguousarray(np.asarray(grid.cosft_wt, float).T)   # (ntau, nfreq)
    proj_bar = torch.zeros_like(proj)
    for k0 in range(0, cw_t.shape[1], _MAX_J):
        transform(W_bar[k0:k0 + _MAX_J].contiguous(), np.ascontiguousarray(cw_t[:, k0:k0 + _MAX_J]),
                  out=proj_bar, accumulate=True)
    del W_bar
    explicit_push = []
    for q, wt in res:
        f = abs(eps_h[q] - w)
        b = B[:, q]
        y = lap.apply(f, b)
        B_bar[:, q] += (z * wt * 2.0) * (y - b)
        if residue_route == 'laplace':
            cf, _ = real_frequency_weights(grid, f)
            proj_bar += (torch.as_tensor(z * wt * cf, device=dev)[:, None, None]
                         * torch.outer(y, y)[None])
        else:
            explicit_push.append((f, y, z * wt))
        eps_bar[q] += z * wt * lap.slope(f, y) * np.sign(eps_h[q] - w)
    from .adjoint import chi0_backward
    e2, X_bar, D_bar = chi0_backward(proj_bar, X, D, eps_h, nocc, grid.tau_points, mu)
    if explicit_push:
        eps_bar += _explicit_residue_backward(X, D, eps_h, nocc, explicit_push, X_bar, D_bar)
    _slice_backward(X, D, p, B_bar, X_bar, D_bar)
    eps_bar = eps_bar + e2.cpu().numpy()
    if isinstance(X, torch.Tensor):
        return w, z, torch.as_tensor(eps_bar, device=dev), X_bar, D_bar
    return w, z, eps_bar, X_bar.cpu().numpy(), D_bar.cpu().numpy()
