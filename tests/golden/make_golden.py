"""Generate the golden fixtures of tests/golden/ by running MBPTcode itself.

Run in a container that holds the reference at /root/reference (pure Python;
the modules used here import without pyscf):

    python tests/golden/make_golden.py [/root/reference]

Each fixture stores the inputs (seeded) and the reference's outputs for them:

* grids.npz          tabulated tau/omega axes and the four transform matrices
                     (src/Base/utils/grids/grids.py, time_frequency.py);
* shared_kernel.npz  the random-factor system of the reference's
                     tests/test_space_time_shared_kernel.py (M=23, n=8, nocc=3,
                     naux=6, ntau=8, nfreq=5, seed 11, five row tiles):
                     proj(tau) and chi0(i w);
* route_<name>.npz   a synthetic ISDF system (mbptcode_b200.synthetic) through
                     the reference route: chi0, W - I, Wt(tau), the Sigma_c
                     diagonal from the AO build, QP roots and Z for every
                     state, E_c and its adjoint;
* static.npz         the static screening W(omega = 0) of the BSE kernel: the
                     auto-sized one-frequency grid, W of a restricted system
                     (auto and 12 points) and the spin-summed W of an
                     unrestricted one;
* unrestricted.npz   the unrestricted route (two spin channels, one W from the
                     spin-summed chi0): grids, W - I, each channel's Sigma_c
                     diagonal, QP roots and Z;
* sigma_adjoint.npz  the self-energy diagonal of three states and its adjoint
                     (eps_bar, X_bar, D_bar) for seeded adjoints on Re and
                     Im Sigma;
* contour.npz        the contour-deformation self-energy's pieces: the contour
                     grid, proj(tau) on it, the screening contraction of three
                     states, Sigma^c at points around each state's level
                     (residues through the Laplace backend) and the integral
                     weights (the CD module loads pyscf for its driver; a
                     stand-in that raises on use lets it import here);
* contour_explicit.npz  the explicit particle-hole backend of continuation
                     'cd': C_ov, W(freq) b and its slope below and above the
                     gap, the explicit imaginary-axis contraction, Sigma^c
                     with explicit residues and five states' roots and Z;
* contour_unrestricted.npz  the contour of an unrestricted reference: the grid
                     on both spins' pair energies, the spin-summed proj(tau),
                     each channel's contraction and its roots and Z with the
                     Laplace and the explicit residues;
* sigma_ao.npz       the full AO self-energy with an AO collocation that is not
                     the MO one, a subset of its time points, its MO diagonal,
                     and the chi0 sweep's reverse for a seeded proj_bar;
* evgw.npz           the reference's evGW loop (GW/evGW.py) through its
                     space-time driver on two synthetic systems (default
                     numerics) and a windowed, damped run: the spectra,
                     cycles and convergence histories;
* drop_in.npz        the seam calls MBPTcode's own G0W0 driver, dRPA energy
                     and adjoint make (every name plugin.install() rebinds,
                     recorded with its arguments and result), and the
                     drivers' outputs;
* isdf.npz           the separable-RI fit from supplied collocations, pair
                     coefficients and metric: the reference's fit_M_stable,
                     aux_metric_sqrt and D = M^T V^1/2;
* qp_kat.npz         the root finder on closed-form self-energies
                     (tests/test_qp_refine_root.py's two-pole Sigma and others);
* qp_follow.npz      the scan following a previous root (`follow`, `out`,
                     `rescan`, `positive_weight`) on 24 seeded pole-sum
                     self-energies: each model's poles and amplitudes, the
                     followed points, and the root, Z and branch record the
                     reference's `solve_qp_equation_scan` returns;
* contour_follow.npz `qp_energy_cd` following a previous root on the system of
                     contour.npz (Laplace residues): root, Z, branch record
* contour_grad_explicit.npz  the QP gradient on the explicit residue route
                     (residues from C_ov) for orbitals 1-4 of contour.npz's system
* sop.npz            the pole model on contour.npz's wc (fitted poles and
                     amplitudes, Sigma, slope, roots, followed roots), the
                     compression test, the driver's 'sop' roots, and the
                     pole-sum root finder on seeded signed and positive sums
* c1_<variant>.npz   the synthetic FP64 configuration at full size (n_orb = 400,
                     nocc = 40, N_mu = 2400, 16 points, seed 400): the Sigma_c
                     diagonal, every QP root and Z, E_c, and the adjoint
                     projected on 32 seeded directions. X and D (46 MB) are not
                     stored: the tests regenerate them from the seed and check
                     the regeneration against the stored eps and checksums.

    python tests/golden/make_golden.py [/root/reference] [--only c1|static|unrestricted|sigma_adjoint|contour|contour_explicit|contour_unrestricted|sigma_ao|evgw|drop_in|isdf|follow|sop|grad_explicit]
"""
import os
import sys
import warnings

import numpy as np

ARGS = [a for a in sys.argv[1:] if not a.startswith('--')]
ONLY = sys.argv[sys.argv.index('--only') + 1] if '--only' in sys.argv else None
if ONLY:
    ARGS = [a for a in ARGS if a != ONLY]
REF = ARGS[0] if ARGS else '/root/reference'
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REF)
sys.path.insert(0, os.path.abspath(os.path.join(HERE, '..', '..')))

from src.Base.utils.grids.grids import (gauss_legendre_grid,            # noqa: E402
                                        minimax_frequency_grid, minimax_time_grid)
from src.Base.utils.grids.time_frequency import (TimeFrequencyGrid,     # noqa: E402
                                                 sigma_fit_ranges,
                                                 minimax_transform_weights,
                                                 COSINE_TW, COSINE_WT, SINE_TW)
from src.Base.utils.grids.analytic_continuation import (PadeFit,        # noqa: E402
                                                        thiele_coefficients)
from src.Base.orbital_spaces import particle_hole_window                # noqa: E402
from src.SingleReference.LinearResponse.space_time import (             # noqa: E402
    chi0_imaginary_frequency, dyson_screening, minimax_points_for_bse,
    polarizability_projected_sweep, rpa_correlation_energy_space_time,
    spin_summed, static_screening_grid, static_screening_matrix,
    static_screening_matrix_unrestricted)
from src.SingleReference.GW.imaginary_time import (                     # noqa: E402
    minimax_points_for_gw, screening_frequency_grid, _transform_screened,
    self_energy_matrix_imaginary_time, sigma_ao_to_mo_diagonal,
    minimax_points_for_gw_unrestricted, unrestricted_fit_ranges,
    unrestricted_screening_frequency_grid)
from src.Base.orbital_spaces import transition_range                    # noqa: E402
from src.Solvers.qp_equation import solve_qp_equation_pole_strength     # noqa: E402
from src.gradients.rpa.space_time_adjoint import (                      # noqa: E402
    rpa_energy_and_adjoint, selfenergy_diag_backward)
from src.SingleReference.GW.imaginary_time import selfenergy_diag        # noqa: E402
from src.Base.utils.grids.time_frequency import sigma_transforms        # noqa: E402

from mbptcode_b200.synthetic import synthetic_system                    # noqa: E402

sys.path.insert(0, HERE)
from c1_common import C1, c1_directions                                  # noqa: E402


def grids_fixture():
    out = {}
    cases = [(8, 1.0, 12.0), (12, 0.35, 6.5), (16, 0.3, 30.0), (18, 0.2, 40.0),
             (20, 0.3, 30.0), (24, 0.1, 20.0), (30, 1.0, 100.0), (34, 1.0, 100.0)]
    out['cases'] = np.array(cases)
    for i, (n, a, b) in enumerate(cases):
        n = int(n)
        out[f'tau_{i}'], out[f'tauw_{i}'] = minimax_time_grid(n, a, b)
        out[f'om_{i}'], out[f'omw_{i}'] = minimax_frequency_grid(n, a, b)
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            g = TimeFrequencyGrid.minimax(n, a, b)
        for k in ('cosft_wt', 'cosft_tw', 'sinft_wt', 'sinft_tw'):
            out[f'{k}_{i}'] = getattr(g, k)
    out['gl16'], out['gl16w'] = gauss_legendre_grid(16, 1.0)
    np.savez_compressed(os.path.join(HERE, 'grids.npz'), **out)


def shared_kernel_fixture():
    M, NORB, NOCC, NAUX, NTAU, NFREQ = 23, 8, 3, 6, 8, 5
    tile_gb = 5 * 3 * M * 8 / 1e9
    rng = np.random.default_rng(11)
    eps = np.sort(rng.normal(size=NORB))
    eps[NOCC:] += 2.0
    X = 0.25 * rng.normal(size=(M, NORB))
    D = 0.25 * rng.normal(size=(M, NAUX))
    gap = eps[NOCC] - eps[NOCC - 1]
    e_max = eps[-1] - eps[0]
    nu, wt = gauss_legendre_grid(NFREQ, w0=gap)
    grid = TimeFrequencyGrid.minimax_split(NTAU, gap, e_max, nu, wt,
                                           with_sine=False, with_inverse=False)
    proj = polarizability_projected_sweep(X, D, eps, NOCC, grid.tau_points,
                                          tile_memory_gb=tile_gb)
    chi0 = chi0_imaginary_frequency(X, D, eps, NOCC, grid, tile_memory_gb=tile_gb)
    np.savez_compressed(os.path.join(HERE, 'shared_kernel.npz'), X=X, D=D,
                        eps=eps, nocc=NOCC, tau=grid.tau_points,
                        cosft_wt=grid.cosft_wt, omega=nu, omega_w=wt,
                        proj=proj, chi0=chi0)


def route_fixture(name, n_orb, nocc, M, seed, variant, ntau, full=False):
    X, D, eps = synthetic_system(n_orb, nocc, M, seed, variant)
    e_min, e_max, mu = particle_hole_window(eps, nocc)
    ntau_auto, _ = minimax_points_for_gw(eps, nocc, mu=mu)
    freq, fw = screening_frequency_grid(ntau, eps, nocc, mu=mu)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        grid = TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, freq, fw)
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    tau_sigma = 0.5 * minimax_time_grid(ntau, *rS)[0]
    pade = gauss_legendre_grid(16, w0=1.0)[0]
    chi0 = chi0_imaginary_frequency(X, D, eps, nocc, grid, mu=mu)
    W = np.stack([dyson_screening(c, correlation=True) for c in chi0])
    Ctw = minimax_transform_weights(COSINE_WT, tau_sigma, freq, *rW, warn=False)[0]
    C = minimax_transform_weights(COSINE_TW, tau_sigma, pade, *rS, warn=False)[0]
    S = minimax_transform_weights(SINE_TW, tau_sigma, pade, *rS, warn=False)[0]
    Wt = _transform_screened(Ctw, W + np.eye(W.shape[-1]))
    sig_ao = self_energy_matrix_imaginary_time(
        X, D, W + np.eye(W.shape[-1]), np.eye(n_orb), eps, nocc, tau_sigma,
        freq, pade, mu=mu)
    states = np.arange(n_orb)
    sigma = sigma_ao_to_mo_diagonal(sig_ao, np.eye(n_orb), states=states).T
    roots, zs = np.empty(n_orb), np.empty(n_orb)
    for i, p in enumerate(states):
        sign = -1.0 if p < nocc else 1.0
        z_fit = mu + 1j * sign * pade
        s_p = np.conj(sigma[i]) if p < nocc else sigma[i]
        fit = PadeFit(z_fit, s_p, greedy=True)

        def residual(w, fit=fit, p=p):
            return w - eps[p] - fit(np.array([w], dtype=complex))[0].real
        got = solve_qp_equation_pole_strength(residual, eps[p],
                                              return_diagnostics=True)
        roots[i] = got[0]
        dz = [z for w, z in got[1] if w == got[0]]
        zs[i] = dz[0] if dz else np.nan
    e_c = rpa_correlation_energy_space_time(X, D, eps, nocc, grid, mu=mu)
    e_c2, eps_bar, X_bar, D_bar, _ = rpa_energy_and_adjoint(X, D, eps, nocc,
                                                            grid, mu=mu)
    big = dict(chi0=chi0, W_minus_I=W, Wt=Wt) if full else {}
    np.savez_compressed(
        os.path.join(HERE, f'route_{name}.npz'), **big, X=X, D=D, eps=eps, nocc=nocc,
        ntau=ntau, ntau_auto=ntau_auto, mu=mu, tau=grid.tau_points,
        omega=freq, omega_w=fw, cosft_wt=grid.cosft_wt, tau_sigma=tau_sigma,
        Ctw=Ctw, C=C, S=S, pade=pade, sigma=sigma, roots=roots, z=zs, e_c=e_c, e_c_adj=e_c2,
        eps_bar=eps_bar, X_bar=X_bar, D_bar=D_bar)


def c1_fixture(variant):
    n_orb, nocc, M, ntau, seed = (C1[k] for k in ('n_orb', 'nocc', 'M', 'ntau', 'seed'))
    X, D, eps = synthetic_system(n_orb, nocc, M, seed, variant)
    e_min, e_max, mu = particle_hole_window(eps, nocc)
    freq, fw = screening_frequency_grid(ntau, eps, nocc, mu=mu)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        grid = TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, freq, fw)
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    tau_sigma = 0.5 * minimax_time_grid(ntau, *rS)[0]
    pade = gauss_legendre_grid(16, w0=1.0)[0]
    chi0 = chi0_imaginary_frequency(X, D, eps, nocc, grid, mu=mu)
    W = np.stack([dyson_screening(c, correlation=True) for c in chi0])
    del chi0
    sig_ao = self_energy_matrix_imaginary_time(
        X, D, W + np.eye(W.shape[-1]), np.eye(n_orb), eps, nocc, tau_sigma,
        freq, pade, mu=mu)
    del W
    states = np.arange(n_orb)
    sigma = sigma_ao_to_mo_diagonal(sig_ao, np.eye(n_orb), states=states).T
    roots, zs = np.empty(n_orb), np.empty(n_orb)
    for i, p in enumerate(states):
        sign = -1.0 if p < nocc else 1.0
        s_p = np.conj(sigma[i]) if p < nocc else sigma[i]
        fit = PadeFit(mu + 1j * sign * pade, s_p, greedy=True)

        def residual(w, fit=fit, p=p):
            return w - eps[p] - fit(np.array([w], dtype=complex))[0].real
        got = solve_qp_equation_pole_strength(residual, eps[p], return_diagnostics=True)
        roots[i] = got[0]
        dz = [z for w, z in got[1] if w == got[0]]
        zs[i] = dz[0] if dz else np.nan
    e_c, eps_bar, X_bar, D_bar, _ = rpa_energy_and_adjoint(X, D, eps, nocc, grid, mu=mu)
    proj = np.array([float(eps_bar @ de + (X_bar * dX).sum() + (D_bar * dD).sum())
                     for de, dX, dD in c1_directions(n_orb, M, seed + 1)])
    np.savez_compressed(
        os.path.join(HERE, f'c1_{variant}.npz'), eps=eps, nocc=nocc, ntau=ntau, mu=mu,
        seed=seed, M=M, X_sum=X.sum(), X_abs_sum=np.abs(X).sum(), D_sum=D.sum(),
        D_diag=np.diag(D).copy(), sigma=sigma, roots=roots, z=zs, e_c=e_c,
        adjoint_projections=proj)


def static_fixture():
    """The static screening W(omega = 0) of the BSE kernel: the auto-sized
    one-frequency grid and W of a restricted system, and the spin-summed W of
    an unrestricted one (alpha: the restricted system; beta: its own
    collocation and spectrum from another seed, one electron fewer)."""
    X, D, eps = synthetic_system(24, 4, 64, 7, 'calibrated')
    ntau, resid = minimax_points_for_bse(eps, 4)
    grid = static_screening_grid(eps, 4)
    W = static_screening_matrix(X, D, eps, 4, grid)
    grid12 = static_screening_grid(eps, 4, ntau=12)
    W12 = static_screening_matrix(X, D, eps, 4, grid12)
    Xb, _, eps_b = synthetic_system(24, 3, 64, 8, 'calibrated')
    Wu = static_screening_matrix_unrestricted([X, Xb], D, [eps, eps_b], [4, 3])
    np.savez_compressed(
        os.path.join(HERE, 'static.npz'), X=X, D=D, eps=eps, nocc=4, ntau=ntau,
        resid=resid, tau=grid.tau_points, cosft_wt=grid.cosft_wt, W=W, tau12=grid12.tau_points,
        cosft_wt12=grid12.cosft_wt, W12=W12, Xb=Xb, eps_b=eps_b, nocc_b=3, W_u=Wu)


def _qp_roots(sigma, eps, nocc, mu, pade, states):
    """Roots and Z of every state, as GW/qp_solve.py:529-558 per state."""
    roots, zs = np.empty(len(states)), np.empty(len(states))
    for i, p in enumerate(states):
        sign = -1.0 if p < nocc else 1.0
        s_p = np.conj(sigma[i]) if p < nocc else sigma[i]
        fit = PadeFit(mu + 1j * sign * pade, s_p, greedy=True)

        def residual(w, fit=fit, p=p):
            return w - eps[p] - fit(np.array([w], dtype=complex))[0].real
        got = solve_qp_equation_pole_strength(residual, eps[p], return_diagnostics=True)
        roots[i] = got[0]
        dz = [z for w, z in got[1] if w == got[0]]
        zs[i] = dz[0] if dz else np.nan
    return roots, zs


def unrestricted_fixture(ntau=12):
    """The unrestricted route of GW/space_time.py:866-1009 composed from the
    reference's kernels (the driver module itself needs pyscf): both spins'
    chi0 by `spin_summed`, one W, then each channel's self-energy on the
    two-spin fit ranges and its QP roots through its own mid-gap. Spin alpha:
    5 of 24 orbitals occupied; spin beta: its own collocation and spectrum
    (another seed), 4 occupied."""
    X_a, D, eps_a = synthetic_system(24, 5, 72, 11, 'calibrated')
    X_b, _, eps_b = synthetic_system(24, 4, 72, 12, 'calibrated')
    X_mos, spectra, noccs = [X_a, X_b], [eps_a, eps_b], [5, 4]
    e_min, e_max = transition_range(spectra, noccs)
    ntau_auto, _ = minimax_points_for_gw_unrestricted(spectra, noccs)
    freq, fw = unrestricted_screening_frequency_grid(ntau, spectra, noccs)
    ranges = unrestricted_fit_ranges(spectra, noccs)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        grid = TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, freq, fw)
    tau_sigma = 0.5 * minimax_time_grid(ntau, *ranges[1])[0]
    pade = gauss_legendre_grid(16, w0=1.0)[0]
    chi0 = spin_summed(chi0_imaginary_frequency, X_mos, D, spectra, noccs, grid)
    W = np.stack([dyson_screening(c) for c in chi0])
    out = dict(X_a=X_a, X_b=X_b, D=D, eps_a=eps_a, eps_b=eps_b, nocc_a=5, nocc_b=4, ntau=ntau,
               ntau_auto=ntau_auto, tau=grid.tau_points, omega=freq, cosft_wt=grid.cosft_wt,
               tau_sigma=tau_sigma, rW=ranges[0], rS=ranges[1], W_minus_I=W - np.eye(72))
    for s, (X, e, n) in enumerate(zip(X_mos, spectra, noccs)):
        mu = particle_hole_window(e, n)[2]
        sig_ao = self_energy_matrix_imaginary_time(X, D, W, np.eye(24), e, n, tau_sigma, freq,
                                                   pade, mu=mu, ranges=ranges)
        states = np.arange(24)
        sigma = sigma_ao_to_mo_diagonal(sig_ao, np.eye(24), states=states).T
        roots, zs = _qp_roots(sigma, e, n, mu, pade, states)
        out.update({f'sigma_{s}': sigma, f'roots_{s}': roots, f'z_{s}': zs, f'mu_{s}': mu})
    np.savez_compressed(os.path.join(HERE, 'unrestricted.npz'), **out)


def sigma_adjoint_fixture(ntau=12, nfreq=10):
    """The self-energy diagonal and its adjoint (GW/imaginary_time.py:731-768,
    gradients/rpa/space_time_adjoint.py:795-875) on a small synthetic
    system, set up as the reference's tests/test_kernel_lockstep.py sets them
    up: Gauss-Legendre frequencies on the gap, the minimax tau axis over
    (gap / 2, span), `sigma_transforms` on those axes; three states around
    the gap and seeded adjoints on Re and Im Sigma."""
    X, D, eps = synthetic_system(20, 4, 48, 21, 'calibrated')
    nocc = 4
    gap = eps[nocc] - eps[nocc - 1]
    nu, wt = gauss_legendre_grid(nfreq, w0=gap)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        grid = TimeFrequencyGrid.minimax_split(ntau, 0.5 * gap, eps[-1] - eps[0], nu, wt,
                                               with_sine=False, with_inverse=False)
        mu = 0.5 * (eps[nocc - 1] + eps[nocc])
        transforms = sigma_transforms(eps, nocc, grid.tau_points, grid.omega_points,
                                      grid.omega_points, mu=mu)
    states = np.array([nocc - 1, nocc, nocc + 2])
    a_re, a_im = np.random.default_rng(4).normal(size=(2, len(states), nfreq))
    sigma, cache = selfenergy_diag(X, D, eps, nocc, grid, states, transforms, mu)
    eps_bar, X_bar, D_bar = selfenergy_diag_backward(a_re, a_im, X, D, eps, nocc, grid, states,
                                                     transforms, mu, cache)
    np.savez_compressed(
        os.path.join(HERE, 'sigma_adjoint.npz'), X=X, D=D, eps=eps, nocc=nocc, mu=mu,
        states=states, tau=grid.tau_points, cosft_wt=grid.cosft_wt, omega=nu, omega_w=wt,
        Ctw=transforms[0], C=transforms[1], S=transforms[2], a_re=a_re, a_im=a_im,
        sigma=sigma, eps_bar=eps_bar, X_bar=X_bar, D_bar=D_bar)


_STAND_IN = []


def _install_stand_ins():
    """MBPTcode's drivers import pyscf (and, through the CC package that
    evGW's DIIS lives in, opt_einsum) at module load for what this fixture
    never runs: integrals, SCF, coupled cluster. Both are absent here, so a
    stand-in package whose every attribute raises when called lets the
    modules load. One call is answered: pyscf.df.addons.make_auxmol returns
    an inert placeholder, because the space-time driver builds the auxiliary
    molecule of the solvent gauge transform unconditionally
    (GW/reaction_field.py:98) and, in the gas phase, the transform returns
    None without reading it (GW/reaction_field.py:67-68)."""
    if _STAND_IN:
        return
    import importlib.abc
    import importlib.machinery
    import types

    class _Inert:
        def __init__(self, name):
            self._n = name

        def __getattr__(self, name):
            return _Inert(self._n + '.' + name)

        def __call__(self, *a, **k):
            if self._n == 'pyscf.df.addons.make_auxmol':
                return _Inert('auxmol placeholder')
            raise RuntimeError(f'{self._n}: pyscf is not available here')

        def __mro_entries__(self, bases):
            return (object,)

        def __instancecheck__(self, obj):
            return False

    class _Package(types.ModuleType):
        def __init__(self, name):
            super().__init__(name)
            self.__path__ = []

        def __getattr__(self, name):
            if name.startswith('__'):
                raise AttributeError(name)
            return _Inert(self.__name__ + '.' + name)

    class _Finder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
        def find_spec(self, fullname, path, target=None):
            if fullname.split('.')[0] in ('pyscf', 'opt_einsum'):
                return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
            return None

        def create_module(self, spec):
            return _Package(spec.name)

        def exec_module(self, module):
            pass

    sys.meta_path.insert(0, _Finder())
    _STAND_IN.append(True)


def _import_contour_deformation():
    """The contour-deformation modules, loaded with the stand-ins."""
    _install_stand_ins()
    import src.SingleReference.GW.contour_deformation as cd
    import src.SingleReference.GW.real_screening as rs
    return cd, rs


class _Molecule:
    """The fields of a pyscf Mole the space-time drivers read for a
    closed-shell gas-phase reference with pre-built factors."""

    def __init__(self, nocc):
        self.nelectron = 2 * nocc
        self.spin = 0
        self.basis = 'cc-pvdz'


class _MeanField:
    """The fields of a pyscf RHF object the drivers read when the factors
    come pre-built: the spectrum, occupations, MO coefficients (identity: the
    AO collocation is the MO one) and the AO overlap (identity)."""

    def __init__(self, eps, nocc):
        self.mo_energy = np.asarray(eps, float)
        n = self.mo_energy.size
        self.mo_occ = np.where(np.arange(n) < nocc, 2.0, 0.0)
        self.mo_coeff = np.eye(n)
        self.mol = _Molecule(nocc)
        self._nocc = nocc

    def get_ovlp(self):
        return np.eye(self.mo_energy.size)

    def copy(self):
        return _MeanField(self.mo_energy, self._nocc)


def evgw_fixture():
    """The reference's own evGW loop (GW/evGW.py:78-229) on synthetic
    factors through calc_qp_energy(mode='space-time') and its space-time
    driver, with the stand-ins for pyscf: two systems, default numerics
    (auto-sized grids, DIIS 8 from the second cycle) and a windowed run
    (update a frontier window, linear mixing with damping 0.3)."""
    _install_stand_ins()
    import dataclasses
    from src.SingleReference.GW import evGW
    from src.Base.numerics.numerics import numerics_or_default
    out = {}
    systems = {'a': (24, 4, 96, 5), 'b': (32, 5, 128, 13)}
    for key, (n, nocc, M, seed) in systems.items():
        X, D, eps = synthetic_system(n, nocc, M, seed=seed, variant='calibrated')
        mf = _MeanField(eps, nocc)
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            e, info = evGW.evgw_eigenvalues(mf, mf.mol, mode='space-time', factors=(X, D),
                                            xc_diagonal=np.zeros(n))
        out.update({f'{key}_X': X, f'{key}_D': D, f'{key}_eps0': eps,
                    f'{key}_size': np.array([n, nocc, M, seed]), f'{key}_eps': e,
                    f'{key}_cycles': info['cycles'], f'{key}_history': np.array(info['history']),
                    f'{key}_converged': info['converged']})
    # windowed, damped: orbitals 2..7 of system a move, linear mixing
    n, nocc, M, seed = systems['a']
    X, D, eps = out['a_X'], out['a_D'], out['a_eps0']
    base = numerics_or_default(None)
    num = dataclasses.replace(base, evgw=dataclasses.replace(base.evgw, diis_size=0,
                                                             damping=0.3))
    mf = _MeanField(eps, nocc)
    update = np.arange(2, 8)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        e, info = evGW.evgw_eigenvalues(mf, mf.mol, mode='space-time', factors=(X, D),
                                        xc_diagonal=np.zeros(n), numerics=num, update=update)
    out.update({'w_update': update, 'w_damping': 0.3, 'w_eps': e, 'w_cycles': info['cycles'],
                'w_history': np.array(info['history']), 'w_frozen': info['frozen']})
    np.savez_compressed(os.path.join(HERE, 'evgw.npz'), **out)


GRID_FIELDS = ('tau_points', 'tau_weights', 'omega_points', 'omega_weights', 'cosft_wt')


def _encode(value, key, arrays, seen):
    """A JSON description of one call argument; arrays are copied into
    `arrays` (each distinct array once, found again by its bytes through
    `seen`), a TimeFrequencyGrid as its fields."""
    import hashlib
    if isinstance(value, np.ndarray):
        h = hashlib.sha1(value.tobytes() + str((value.dtype, value.shape)).encode()).hexdigest()
        if h not in seen:
            seen[h] = key
            arrays[key] = np.array(value)
        return {'array': seen[h]}
    if hasattr(value, 'tau_points') and hasattr(value, 'cosft_wt'):
        for f in GRID_FIELDS:
            arrays[f'{key}_{f}'] = np.array(getattr(value, f))
        return {'grid': key}
    if isinstance(value, (np.integer,)):
        return {'value': int(value)}
    if isinstance(value, (np.floating,)):
        return {'value': float(value)}
    if isinstance(value, (list, tuple)) and all(np.isscalar(v) for v in value):
        return {'value': [v.item() if hasattr(v, 'item') else v for v in value]}
    if value is None or isinstance(value, (bool, int, float, str)):
        return {'value': value}
    if isinstance(value, dict) and not value:
        return {'value': {}}
    return {'opaque': type(value).__name__}


def drop_in_fixture():
    """The seam calls the reference's own drivers make, and what each seam
    returned: MBPTcode's G0W0 driver (GW/space_time.py:631-863, through the
    stand-ins for pyscf with pre-built factors), its dRPA energy
    (LinearResponse/space_time.py:1100-1183) and adjoint
    (gradients/rpa/space_time_adjoint.py:473-563) run with every name that
    `mbptcode_b200.plugin.install()` rebinds wrapped by a recorder that keeps
    the arguments and the result of each call (the first few calls per
    name) and forwards to the reference's own function. A GPU test replays
    the recorded calls through the device seams."""
    import json
    _install_stand_ins()
    import importlib
    from mbptcode_b200 import plugin
    from src.SingleReference.GW import space_time as gst
    from src.SingleReference.LinearResponse import space_time as lst
    from src.gradients.rpa import space_time_adjoint as adj
    n, nocc, M, seed = 24, 4, 64, 7
    X, D, eps = synthetic_system(n, nocc, M, seed=seed, variant='calibrated')
    arrays = {'X': X, 'D': D, 'eps': eps}
    calls, counts, saved, seen = [], {}, [], {}
    keep = {'solve_qp_from_imaginary_axis': 6, 'dielectric_log_determinant': 4}
    for modname, names in plugin.replacements().items():
        try:
            mod = importlib.import_module(modname)
        except Exception:                    # noqa: BLE001 -- modules outside the route
            continue
        for name in names:
            if not hasattr(mod, name):
                continue
            original = getattr(mod, name)

            def recorder(*a, _name=name, _mod=modname, _f=original, **k):
                i = counts.get(_name, 0)
                counts[_name] = i + 1
                if i >= keep.get(_name, 2):
                    return _f(*a, **k)
                c = len(calls)
                desc = {'module': _mod, 'name': _name,
                        'args': [_encode(v, f'c{c}_a{j}', arrays, seen) for j, v in enumerate(a)],
                        'kwargs': {kk: _encode(v, f'c{c}_k_{kk}', arrays, seen)
                                   for kk, v in k.items()}}
                calls.append(desc)
                out = _f(*a, **k)
                res = out if isinstance(out, tuple) else (out,)
                desc['result'] = [_encode(np.asarray(r) if np.ndim(r) or isinstance(
                    r, (np.ndarray, float, complex)) else r, f'c{c}_r{j}', arrays, seen)
                    for j, r in enumerate(res)]
                desc['result_tuple'] = isinstance(out, tuple)
                return out
            saved.append((mod, name, original))
            setattr(mod, name, recorder)
    try:
        mf = _MeanField(eps, nocc)
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            roots = gst.solve_qp_energy_space_time(mf, mf.mol, nocc, np.arange(n),
                                                   factors=(X, D), xc_diagonal=np.zeros(n))
            e_min, e_max, mu = particle_hole_window(eps, nocc)
            ntau = 12
            freq, fw = screening_frequency_grid(ntau, eps, nocc, mu=mu)
            grid = TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, freq, fw)
            e_c = lst.rpa_correlation_energy_space_time(X, D, eps, nocc, grid)
            e_a, eb, xb, db, _ = adj.rpa_energy_and_adjoint(X, D, eps, nocc, grid)
    finally:
        for mod, name, original in saved:
            setattr(mod, name, original)
    arrays.update(driver_roots=np.asarray(roots), e_c=np.float64(e_c), eps_bar=eb, X_bar=xb,
                  D_bar=db)
    arrays['calls'] = np.array(json.dumps(calls))
    np.savez_compressed(os.path.join(HERE, 'drop_in.npz'), **arrays)
    print('recorded', {k: v for k, v in counts.items()})


def isdf_fixture():
    """The device half of the separable-RI factors against the reference's
    own fit (Base/factorization/separable_ri.py, loaded with the stand-ins):
    a seeded AO collocation on nk points, the second-factor columns and
    angular weights of the product pairs, the auxiliary collocation, the
    pairs' fitting coefficients F and a Coulomb metric V. The reference's
    explicit estimator `fit_M_stable` on D = [pair columns | auxiliary
    collocation], F = [F_pairs | I] (``build_D_F``'s layout), the metric root
    `aux_metric_sqrt` (with a near-null direction it drops) and D = M^T V^1/2."""
    _install_stand_ins()
    from src.Base.factorization import separable_ri as sr
    rng = np.random.default_rng(31)
    nk, nao, naux = 96, 20, 40
    second = np.array([0, 2, 3, 5, 7, 11, 13, 17])
    w = rng.uniform(0.5, 1.5, len(second))
    pts = rng.uniform(-2, 2, (nk, 3))
    centres = rng.uniform(-2, 2, (nao, 3))
    ao = np.exp(-0.7 * ((pts[:, None, :] - centres[None]) ** 2).sum(-1))
    ao *= rng.uniform(0.5, 2.0, nao)[None, :]
    aux_c = rng.uniform(-2, 2, (naux, 3))
    aux = np.exp(-0.4 * ((pts[:, None, :] - aux_c[None]) ** 2).sum(-1))
    pairs = (ao[:, :, None] * (ao[:, second] * w[None, :])[:, None, :]).reshape(nk, -1)
    F_pairs = rng.standard_normal((naux, pairs.shape[1])) / np.sqrt(pairs.shape[1])
    D = np.hstack([pairs, aux])
    F = np.hstack([F_pairs, np.eye(naux)])
    M = sr.fit_M_stable(D, F)
    Q, _ = np.linalg.qr(rng.standard_normal((naux, naux)))
    lam = np.exp(rng.uniform(np.log(1e-2), np.log(10.0), naux))
    lam[3] = 1e-14 * lam.max()              # a direction in the numerical null space
    V = (Q * lam) @ Q.T
    V = 0.5 * (V + V.T)
    root = sr.aux_metric_sqrt(V=V)
    C = np.linalg.qr(rng.standard_normal((nao, nao)))[0]
    np.savez_compressed(os.path.join(HERE, 'isdf.npz'), ao=ao, second=second, w=w, aux=aux,
                        F_pairs=F_pairs, FD=F @ D.T, M=M, V=V, root=root, D_factor=M.T @ root,
                        mo_coeff=C, X_mo=ao @ C)


def contour_fixture():
    """The contour-deformation self-energy's pieces (GW/contour_deformation.py,
    GW/real_screening.py) on a small synthetic system: the contour grid
    (64 Gauss-Legendre frequencies on half the gap, 24 time points reaching
    half a gap below it), proj(tau) on it, the screening contraction wc of
    three states around the gap, Sigma^c at points on both sides of each
    state's level and on it (residues through the Laplace backend), each
    state's quasiparticle root and Z (`qp_energy_cd`), the gradient of each
    root in (eps, X, D) (gradients/gwbse/qp_space_time.py:412-452, residues
    by the cosh transform), and the integral weights at a set of de
    values."""
    cd, rs = _import_contour_deformation()
    from src.gradients.rpa.space_time_adjoint import polarizability_tau
    from src.SingleReference.LinearResponse.space_time import three_index_slice
    X, D, eps = synthetic_system(16, 3, 48, 31, 'calibrated')
    nocc = 3
    mu = particle_hole_window(eps, nocc)[2]
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, w0 = cd.cd_frequency_grid(eps, nocc)
    proj = polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    states = np.array([nocc - 1, nocc, nocc + 1])
    Bps = [three_index_slice(X, D, int(p)) for p in states]
    wcs = cd.cd_screening_contraction_multi(proj, grid.cosft_wt, Bps)
    lap = rs.LaplaceRealScreening(proj, grid, eps, nocc)
    shifts = np.array([-0.06, -0.02, 0.0, 0.02, 0.06])
    sig = np.zeros((len(states), len(shifts)))
    for i, p in enumerate(states):
        for j, dw in enumerate(shifts):
            sig[i, j] = cd.sigma_cd(int(p), eps[p] + dw, Bps[i], eps, nocc, nu, nu_w,
                                    wc=wcs[i], real_screening=lap)
    roots = np.zeros((len(states), 2))
    for i, p in enumerate(states):
        w, z, _ = cd.qp_energy_cd(int(p), Bps[i], eps, nocc, nu, nu_w, wc=wcs[i],
                                  real_screening=rs.LaplaceRealScreening(proj, grid, eps, nocc))
        roots[i] = w, z
    from src.gradients.gwbse.qp_space_time import qp_gradient_space_time
    grads = [qp_gradient_space_time(X, D, eps, nocc, grid, nu, nu_w, int(p),
                                    residue_route='laplace', mu=mu) for p in states]
    de = np.array([-0.3, -1e-3, 0.0, 1e-12, 2e-3, 0.05, 0.7])
    c, dc = cd.cd_integral_weights(de, nu, nu_w)
    np.savez_compressed(
        os.path.join(HERE, 'contour.npz'), X=X, D=D, eps=eps, nocc=nocc, mu=mu, nu=nu,
        nu_w=nu_w, w0=w0, tau=grid.tau_points, tau_w=grid.tau_weights, cosft_wt=grid.cosft_wt,
        proj=proj, states=states, B=np.stack(Bps), wc=np.stack(wcs), shifts=shifts, sigma=sig,
        roots=roots, de=de, c=c, dc=dc,
        grad_roots=np.array([[gr[0], gr[1]] for gr in grads]),
        eps_bar=np.stack([gr[2] for gr in grads]), X_bar=np.stack([gr[3] for gr in grads]),
        D_bar=np.stack([gr[4] for gr in grads]))


def contour_explicit_fixture():
    """The contour deformation's explicit particle-hole backend (continuation
    'cd'; GW/real_screening.py:57-91, 171-181; GW/contour_deformation.py:240-245)
    on the contour fixture's system: C_ov (LinearResponse/space_time.py:833-851),
    W(freq) b and its slope at real frequencies below and above the gap (with
    and without broadening), the explicit imaginary-axis contraction wc of
    three states, Sigma^c with explicit residues around their levels, and the
    quasiparticle roots and Z of five states from the deepest to the highest
    (the cubic wc with explicit residues; one state with the explicit wc too)."""
    cd, rs = _import_contour_deformation()
    from src.gradients.rpa.space_time_adjoint import polarizability_tau
    from src.SingleReference.LinearResponse.space_time import (three_index_ov,
                                                               three_index_slice)
    from src.Base.orbital_spaces import ov_energies
    X, D, eps = synthetic_system(16, 3, 48, 31, 'calibrated')
    nocc = 3
    mu = particle_hole_window(eps, nocc)[2]
    gap = particle_hole_window(eps, nocc)[0]
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, w0 = cd.cd_frequency_grid(eps, nocc)
    C_ov = three_index_ov(X, D, eps, nocc)
    d = ov_energies(eps, nocc)
    rng = np.random.default_rng(41)
    b = rng.standard_normal(C_ov.shape[0])
    freqs = np.array([0.2, 0.8, 1.3, 2.5]) * gap
    etas = np.array([0.0, 0.01])
    apply_ = np.zeros((len(etas), len(freqs), len(b)))
    slope = np.zeros((len(etas), len(freqs)))
    for a, eta in enumerate(etas):
        ers = rs.ExplicitRealScreening(C_ov, eps, nocc, eta=float(eta))
        for j, f in enumerate(freqs):
            apply_[a, j] = ers.apply(float(f), b)
            slope[a, j] = ers.slope(float(f), apply_[a, j])
    proj = polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    states = np.array([0, nocc - 1, nocc, nocc + 1, len(eps) - 1])
    Bps = [three_index_slice(X, D, int(p)) for p in states]
    wcs = cd.cd_screening_contraction_multi(proj, grid.cosft_wt, Bps)
    near = [1, 2, 3]                      # the three states around the gap
    wcx = np.stack([cd.wc_explicit(Bps[i], C_ov, d, nu) for i in near])
    shifts = np.array([-0.06, 0.0, 0.06])
    sig = np.zeros((len(near), len(shifts)))
    for r, i in enumerate(near):
        p = int(states[i])
        for j, dw in enumerate(shifts):
            sig[r, j] = cd.sigma_cd(p, eps[p] + dw, Bps[i], eps, nocc, nu, nu_w, wc=wcs[i],
                                    C_ov=C_ov)
    roots = np.zeros((len(states), 2))
    for i, p in enumerate(states):
        w, z, _ = cd.qp_energy_cd(int(p), Bps[i], eps, nocc, nu, nu_w, wc=wcs[i], C_ov=C_ov)
        roots[i] = w, z
    w, z, _ = cd.qp_energy_cd(int(states[2]), Bps[2], eps, nocc, nu, nu_w, C_ov=C_ov)
    np.savez_compressed(
        os.path.join(HERE, 'contour_explicit.npz'), X=X, D=D, eps=eps, nocc=nocc, mu=mu, nu=nu,
        nu_w=nu_w, C_ov=C_ov, b=b, freqs=freqs, etas=etas, apply=apply_, slope=slope,
        states=states, wc=np.stack(wcs), near=np.array(near), wc_explicit=wcx, shifts=shifts,
        sigma=sig, roots=roots, root_explicit_wc=np.array([w, z]))


def contour_unrestricted_fixture():
    """The contour deformation of an unrestricted reference, composed from the
    reference's pieces as GW/contour_deformation.py:686-812 composes them (the
    driver itself needs pyscf): both spins' pair energies side by side set the
    contour grid (cd_grid_range / cd_frequency_grid with pair_energies), the
    spin-summed proj(tau), each channel's slices and screening contraction,
    and each channel's roots and Z with the Laplace residues (pair energies
    of both spins) and with the explicit ones (both spins' C_ov side by side
    at 1/sqrt(2)). Spin alpha: 3 of 16 orbitals occupied; spin beta: its own
    collocation and spectrum (another seed), 2 occupied."""
    cd, rs = _import_contour_deformation()
    from src.SingleReference.LinearResponse.space_time import (three_index_ov,
                                                               three_index_slice)
    from src.Base.orbital_spaces import ov_energies
    X_a, D, eps_a = synthetic_system(16, 3, 48, 31, 'calibrated')
    X_b, _, eps_b = synthetic_system(16, 2, 48, 33, 'calibrated')
    X_mos, spectra, noccs = [X_a, X_b], [eps_a, eps_b], [3, 2]
    pairs = np.concatenate([ov_energies(e, n) for e, n in zip(spectra, noccs)])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, w0 = cd.cd_frequency_grid(eps_a, 3, pair_energies=pairs)
    proj = spin_summed(polarizability_projected_sweep, X_mos, D, spectra, noccs,
                       grid.tau_points)
    C_ov = np.hstack([three_index_ov(X, D, e, n) for X, e, n in zip(X_mos, spectra, noccs)])
    out = dict(X_a=X_a, X_b=X_b, D=D, eps_a=eps_a, eps_b=eps_b, nocc_a=3, nocc_b=2, nu=nu,
               nu_w=nu_w, w0=w0, tau=grid.tau_points, tau_w=grid.tau_weights,
               cosft_wt=grid.cosft_wt, proj=proj, pairs=pairs)
    for s, (X, e, n) in enumerate(zip(X_mos, spectra, noccs)):
        states = np.array([n - 1, n, n + 1])
        Bps = [three_index_slice(X, D, int(p)) for p in states]
        wcs = cd.cd_screening_contraction_multi(proj, grid.cosft_wt, Bps)
        lap, exp_ = np.full((3, 2), np.nan), np.zeros((3, 2))
        for i, p in enumerate(states):
            try:
                w, z, _ = cd.qp_energy_cd(int(p), Bps[i], e, n, nu, nu_w, wc=wcs[i],
                                          real_screening=rs.LaplaceRealScreening(
                                              proj, grid, e, n, pair_energies=pairs))
                lap[i] = w, z
            except ValueError:
                pass
            w, z, _ = cd.qp_energy_cd(int(p), Bps[i], e, n, nu, nu_w, wc=wcs[i],
                                      real_screening=rs.ExplicitRealScreening(
                                          C_ov / np.sqrt(2.0), e, n, pair_energies=pairs))
            exp_[i] = w, z
        out.update({f'states_{s}': states, f'wc_{s}': np.stack(wcs), f'roots_laplace_{s}': lap,
                    f'roots_cd_{s}': exp_})
    np.savez_compressed(os.path.join(HERE, 'contour_unrestricted.npz'), **out)


def sigma_ao_fixture():
    """The full AO self-energy of GW/imaginary_time.py:403-533 with an AO
    collocation that is not the MO one (X_ao = X_mo C^T, C a seeded orthogonal
    mo_coeff), its MO diagonal (:581-587), and proj_bar's reverse sweep
    (gradients/rpa/space_time_adjoint.py:136-164) for a seeded proj_bar."""
    from src.gradients.rpa.space_time_adjoint import polarizability_backward
    X, D, eps = synthetic_system(20, 4, 48, 17, 'calibrated')
    nocc, ntau = 4, 12
    rng = np.random.default_rng(17)
    Cmo = np.linalg.qr(rng.standard_normal((20, 20)))[0]
    X_ao = X @ Cmo.T
    e_min, e_max, mu = particle_hole_window(eps, nocc)
    freq, fw = screening_frequency_grid(ntau, eps, nocc, mu=mu)
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        grid = TimeFrequencyGrid.minimax_split(ntau, e_min, e_max, freq, fw)
    rW, rS = sigma_fit_ranges(eps, nocc, mu=mu)
    tau_sigma = 0.5 * minimax_time_grid(ntau, *rS)[0]
    pade = gauss_legendre_grid(16, w0=1.0)[0]
    chi0 = chi0_imaginary_frequency(X, D, eps, nocc, grid, mu=mu)
    W = np.stack([dyson_screening(c) for c in chi0])
    sig = self_energy_matrix_imaginary_time(X_ao, D, W, Cmo, eps, nocc, tau_sigma, freq, pade,
                                            mu=mu)
    sig_sub = self_energy_matrix_imaginary_time(X_ao, D, W, Cmo, eps, nocc, tau_sigma, freq,
                                                pade, mu=mu, tau_indices=[1, 4, 7])
    states = np.array([nocc - 1, nocc, nocc + 3])
    diag = sigma_ao_to_mo_diagonal(sig, Cmo, states=states)
    proj_bar = rng.standard_normal((ntau, 48, 48))
    eb, xb, db = polarizability_backward(proj_bar, X, D, eps, nocc, grid, mu=mu)
    np.savez_compressed(
        os.path.join(HERE, 'sigma_ao.npz'), X=X, X_ao=X_ao, D=D, eps=eps, nocc=nocc, mo=Cmo,
        mu=mu, ntau=ntau, omega=freq, tau_sigma=tau_sigma, pade=pade, W=W, sigma=sig,
        sigma_sub=sig_sub, states=states, diag=diag, proj_bar=proj_bar, eps_bar=eb, X_bar=xb,
        D_bar=db)


def qp_fixture():
    cases = {  # poles placed off the scan grids, so no division hits one
        'two_pole': (lambda w: 0.05 / (w + 0.8) + 0.01 / (w - 0.9), -0.2),
        'one_pole': (lambda w: 0.02 / (w + 0.5), 0.3),
        'satellite': (lambda w: 0.3 / (w + 0.4537) + 0.02 / (w + 1.1129), -0.6),
        'deep': (lambda w: 0.4 / (w - 0.2113) + 0.1 / (w + 3.0171), -2.0),
    }
    out = {}
    for k, (sig, a) in cases.items():
        f = lambda w, sig=sig, a=a: w - a - sig(w)
        got = solve_qp_equation_pole_strength(f, a, return_diagnostics=True,
                                              full_output=True)
        out[k] = np.array([got[0], float(got[2])])
    # Thiele coefficients of a random complex sample (16 points)
    rng = np.random.default_rng(5)
    z = 0.1 + 1j * np.sort(rng.uniform(0.01, 10.0, 16))
    f = rng.normal(size=16) + 1j * rng.normal(size=16)
    out['thiele_z'], out['thiele_f'] = z, f
    out['thiele_a'] = thiele_coefficients(z, f)
    fit = PadeFit(z, f, greedy=True)
    out['greedy_z'] = fit.z
    out['greedy_eval'] = fit(np.linspace(-1, 1, 7) + 0j)
    np.savez_compressed(os.path.join(HERE, 'qp_kat.npz'), **out)


def follow_fixture(nmodels=24, seed=31):
    """Root following on the scan (``Solvers/qp_equation.py:1396-1420``,
    `find_qp_root` with `follow`): the reference's `solve_qp_equation_scan`
    on seeded pole-sum self-energies Sigma(w) = sum_k A_k / (w - p_k), each
    with its closed-form slope, unfollowed and following points beside each
    root, between roots and outside every window, rescan on and off,
    positive_weight on (positive amplitudes) and off (some negative), with
    the branch record the `out` dict receives."""
    from src.Solvers.qp_equation import solve_qp_equation_scan
    rng = np.random.default_rng(seed)
    models, cases = [], []

    def model(a, pol, amp):
        def f(w):
            return w - a - float(np.sum(amp / (w - pol)))

        def fp(w):
            return 1.0 + float(np.sum(amp / (w - pol) ** 2))
        return f, fp
    for m in range(nmodels):
        npol = int(rng.integers(3, 7))
        pol = np.sort(rng.uniform(-2.0, 2.0, npol))
        amp = np.exp(rng.uniform(np.log(1e-6), np.log(0.3), npol))
        positive = m % 4 != 3
        if not positive:
            amp[int(rng.integers(npol))] *= -1.0
        a = float(rng.uniform(-0.6, 0.6))
        models.append((a, pol, amp, positive))
        f, fp = model(a, pol, amp)
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            w0, _ = solve_qp_equation_scan(f, fp, a, positive_weight=positive)
        grid = np.linspace(a - 0.5, a + 0.5, 2001)
        vals = np.array([f(x) for x in grid])
        roots = [0.5 * (grid[i] + grid[i + 1]) for i in range(len(grid) - 1)
                 if vals[i] < 0.0 < vals[i + 1]]
        targets = [None] + [r + d for r in roots[:4] for d in (0.0, 3e-3)]
        targets += [float(rng.uniform(a - 0.4, a + 0.4)), a + 3.0]
        for t in targets:
            for rescan in ((True, False) if t is not None else (True,)):
                out = {}
                with warnings.catch_warnings():
                    warnings.simplefilter('ignore')
                    w, z = solve_qp_equation_scan(f, fp, a, follow=t, out=out,
                                                  positive_weight=positive, rescan=rescan)
                lg = out.get('largest')
                cases.append([m, np.nan if t is None else t, float(rescan), w, z,
                              np.nan if lg is None or not len(lg) else lg[0],
                              np.nan if lg is None or not len(lg) else lg[1],
                              {None: -1.0, False: 0.0, True: 1.0}[out.get('followed')],
                              float(bool(out.get('flipped'))), float(bool(out.get('no_root'))),
                              float(bool(out.get('z_outside')))])
    npol_max = max(len(mm[1]) for mm in models)
    pols = np.full((nmodels, npol_max), np.nan)
    amps = np.zeros((nmodels, npol_max))
    for i, (_, pol, amp, _) in enumerate(models):
        pols[i, :len(pol)], amps[i, :len(amp)] = pol, amp
    np.savez_compressed(os.path.join(HERE, 'qp_follow.npz'),
                        a=np.array([mm[0] for mm in models]), poles=pols, amps=amps,
                        positive=np.array([mm[3] for mm in models]),
                        cases=np.array(cases, float),
                        columns=np.array(['model', 'follow', 'rescan', 'w', 'z', 'largest_w',
                                          'largest_z', 'followed', 'flipped', 'no_root',
                                          'z_outside']))


def contour_follow_fixture():
    """`qp_energy_cd` following a previous root (``contour_deformation.py:
    376-436`` with `follow`, `branch`, `rescan`) on the system of
    `contour_fixture`, residues through the Laplace backend: per state, the
    followed points the root itself, 2e-3 above it, 0.02 below it and 0.3
    above its level, the rescan on and off; the root, Z and the branch
    record."""
    cd, rs = _import_contour_deformation()
    from src.gradients.rpa.space_time_adjoint import polarizability_tau
    from src.SingleReference.LinearResponse.space_time import three_index_slice
    g = np.load(os.path.join(HERE, 'contour.npz'))
    X, D, eps, nocc, mu = g['X'], g['D'], g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = cd.cd_frequency_grid(eps, nocc)
    proj = polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    states = g['states']
    Bps = [three_index_slice(X, D, int(p)) for p in states]
    wcs = cd.cd_screening_contraction_multi(proj, grid.cosft_wt, Bps)
    cases = []
    for i, p in enumerate(states):
        root = float(g['roots'][i, 0])
        for t in (root, root + 2e-3, root - 0.02, float(eps[p]) + 0.3):
            for rescan in (True, False):
                out = {}
                with warnings.catch_warnings():
                    warnings.simplefilter('ignore')
                    w, z, res = cd.qp_energy_cd(
                        int(p), Bps[i], eps, nocc, nu, nu_w, wc=wcs[i],
                        real_screening=rs.LaplaceRealScreening(proj, grid, eps, nocc),
                        follow=t, branch=out, rescan=rescan)
                lg = out.get('largest')
                cases.append([i, t, float(rescan), w, z,
                              np.nan if lg is None or not len(lg) else lg[0],
                              np.nan if lg is None or not len(lg) else lg[1],
                              {None: -1.0, False: 0.0, True: 1.0}[out.get('followed')],
                              float(bool(out.get('flipped'))), len(res)])
    np.savez_compressed(os.path.join(HERE, 'contour_follow.npz'), cases=np.array(cases, float),
                        columns=np.array(['state', 'follow', 'rescan', 'w', 'z', 'largest_w',
                                          'largest_z', 'followed', 'flipped', 'residues']))


def sop_fixture(nsums=40, seed=37):
    """The pole model (GW/sum_over_poles.py) on the contour system's wc (from
    contour.npz): per state the fitted poles and amplitudes (12 poles at the
    default stride, 8 poles at stride 1, and 12 log-spaced unfitted),
    Sigma and its slope at five points, the root and Z, the root followed
    from 2e-3 away and from the neighbouring interval, with their branch
    records, and the compression test at the start points; the reference
    driver's per-state 'sop' roots (`_contour_roots`); and the pole-sum root
    finder (`solve_qp_equation_poles`) on seeded sums of positive and of
    mixed-sign weights, unfollowed and following labelled branches."""
    cd, _ = _import_contour_deformation()
    from src.SingleReference.GW import sum_over_poles as sp
    from src.Solvers.qp_equation import solve_qp_equation_poles, qp_start
    g = np.load(os.path.join(HERE, 'contour.npz'))
    eps, nocc, nu, nu_w = g['eps'], int(g['nocc']), g['nu'], g['nu_w']
    states, wcs = g['states'], g['wc']
    out = {}
    shifts = np.array([-0.05, -0.01, 0.0, 0.01, 0.05])
    for tag, kw in (('fit12', dict()), ('fit8s1', dict(n_poles=8, stride=1)),
                    ('log12', dict(relocate=False))):
        poles_l, amps_l, sig, slope, roots, fol = [], [], [], [], [], []
        for i, p in enumerate(states):
            with warnings.catch_warnings():
                warnings.simplefilter('ignore')
                poles, amp = sp.sop_from_wc(wcs[i], nu, eps, nocc, **kw)
                poles_l.append(poles)
                amps_l.append(amp)
                sig.append([sp.sigma_sop(eps[p] + d, amp, poles, eps, nocc, check=False)
                            for d in shifts])
                slope.append([sp.sigma_sop_slope(eps[p] + d, amp, poles, eps, nocc)
                              for d in shifts])
                br = {}
                w, z = sp.qp_energy_sop(int(p), amp, poles, eps, nocc, branch=br)
                roots.append([w, z])
                lab = br['labels']
                for follow in ((w + 2e-3, lab), (w + 2e-3, None), (w, (lab[0], None)),
                               (w - 0.3, None)):
                    b2 = {}
                    w2, z2 = sp.qp_energy_sop(int(p), amp, poles, eps, nocc,
                                              follow=follow, branch=b2)
                    lg = b2.get('largest')
                    fol.append([i, follow[0], -2 if follow[1] is None else
                                (-1 if follow[1][1] is None else 0), w2, z2,
                                np.nan if lg is None else lg[0],
                                {None: -1.0, False: 0.0, True: 1.0}[b2.get('followed')],
                                float(bool(b2.get('flipped')))])
        npl = max(len(q) for q in poles_l)
        P = np.full((len(states), npl), np.nan)
        A = np.full((len(states), npl, len(eps)), np.nan)
        for i in range(len(states)):
            P[i, :len(poles_l[i])] = poles_l[i]
            A[i, :len(poles_l[i])] = amps_l[i]
        out.update({f'{tag}_poles': P, f'{tag}_amps': A, f'{tag}_sigma': np.array(sig),
                    f'{tag}_slope': np.array(slope), f'{tag}_roots': np.array(roots),
                    f'{tag}_follow': np.array(fol, float)})
    starts = np.array([qp_start(eps, int(p), nocc) for p in states])
    adm = [sp.compressible(float(w), eps, nocc) for w in starts]
    out['starts'] = starts
    out['admits'] = np.array([a[0] for a in adm])
    out['reach'] = np.array([a[1] for a in adm])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        r, zz, rec = cd._contour_roots('sop', states, starts, adm, list(g['B']), list(wcs),
                                       eps, nocc, nu, nu_w, 0.0, sp.SOP_N_POLES,
                                       sp.SOP_FIT_STRIDE, None)
    out['driver_roots'] = np.asarray(r, float)
    out['driver_z'] = np.asarray(zz, float)
    # the QP gradient on the pole model's route (poles fitted here, then held)
    from src.gradients.gwbse.qp_space_time import qp_gradient_space_time
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        grid = cd.cd_frequency_grid(eps, nocc)[2]
        grads = []
        for p in states:
            rec = {}
            grads.append(qp_gradient_space_time(g['X'], g['D'], eps, nocc, grid, nu, nu_w,
                                                int(p), residue_route='sop',
                                                mu=float(g['mu']), route_out=rec))
    out['grad_roots'] = np.array([[gr[0], gr[1]] for gr in grads])
    out['grad_eps_bar'] = np.stack([gr[2] for gr in grads])
    out['grad_X_bar'] = np.stack([gr[3] for gr in grads])
    out['grad_D_bar'] = np.stack([gr[4] for gr in grads])
    rng = np.random.default_rng(seed)
    sums, cases = [], []
    for k in range(nsums):
        n = int(rng.integers(4, 30))
        pol = rng.uniform(-2.0, 2.0, n)
        num = np.exp(rng.uniform(np.log(1e-5), np.log(0.2), n))
        if k % 2:
            neg = rng.random(n) < 0.3
            num[neg] *= -rng.uniform(0.05, 1.0, int(neg.sum()))
        if k % 5 == 4:
            pol[1] = pol[0]                       # coinciding poles
        a = float(rng.uniform(-0.5, 0.5))
        sums.append((a, pol, num))
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            b = {}
            w, z = solve_qp_equation_poles(num, pol, a, out=b)
            lab = b.get('labels')
            cases.append([k, np.nan, -2, w, z, np.nan, -1.0, 0.0,
                          np.nan if lab is None or lab[0] is None else lab[0],
                          np.nan if lab is None or lab[1] is None else lab[1]])
            for t, labels in ((a + 0.05, None), (float(rng.uniform(-2, 2)), None),
                              (w + 1e-3, lab)):
                if labels is not None and not np.isfinite(w):
                    continue
                b2 = {}
                w2, z2 = solve_qp_equation_poles(num, pol, a, follow=(t, labels), out=b2)
                lg = b2.get('largest')
                l2 = b2.get('labels')
                cases.append([k, t, -2 if labels is None else 0, w2, z2,
                              np.nan if lg is None else lg[0],
                              {None: -1.0, False: 0.0, True: 1.0}[b2.get('followed')],
                              float(bool(b2.get('flipped'))),
                              np.nan if l2 is None or l2[0] is None else l2[0],
                              np.nan if l2 is None or l2[1] is None else l2[1]])
    nmax = max(len(q[1]) for q in sums)
    SP = np.full((nsums, nmax), np.nan)
    SN = np.zeros((nsums, nmax))
    for k, (_, pol, num) in enumerate(sums):
        SP[k, :len(pol)], SN[k, :len(num)] = pol, num
    out.update(sum_a=np.array([q[0] for q in sums]), sum_poles=SP, sum_nums=SN,
               sum_cases=np.array(cases, float), shifts=shifts)
    np.savez_compressed(os.path.join(HERE, 'sop.npz'), **out)


def contour_grad_explicit_fixture():
    """The QP gradient on the explicit residue route (residue_route 'explicit':
    residues from C_ov, their adjoint chained onto (C_ov, d) and back to
    (eps, X, D) by three_index_ov's reverse) on the contour system, for
    orbitals 1 to 4 (orbital 1 sweeps residues above the gap)."""
    cd, _ = _import_contour_deformation()
    from src.gradients.gwbse.qp_space_time import qp_gradient_space_time
    g = np.load(os.path.join(HERE, 'contour.npz'))
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = cd.cd_frequency_grid(eps, nocc)
        states = np.array([1, 2, 3, 4])
        grads, nres = [], []
        for p in states:
            rec = {}
            grads.append(qp_gradient_space_time(g['X'], g['D'], eps, nocc, grid, nu, nu_w,
                                                int(p), residue_route='explicit', mu=mu,
                                                route_out=rec))
            nres.append(len(rec['residues']))
    # the pole-model route's decisions: orbital 9 (reach 1.45 gaps) falls back
    # to the explicit residues; a frozen scissor mapping, or a scalar where the
    # compression test fails, shifts it; orbital 2 keeps the pole model
    route_cases = [(9, None), (9, {9: 0.05}), (9, 0.07), (2, 0.07)]
    route_out = []
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        for p, sc in route_cases:
            rec = {}
            gr = qp_gradient_space_time(g['X'], g['D'], eps, nocc, grid, nu, nu_w, p,
                                        residue_route='sop', mu=mu, scissor=sc, route_out=rec)
            route_out.append((rec['residue_route'], gr))
    extra = {}
    for j, (route, gr) in enumerate(route_out):
        extra[f'route{j}_name'] = np.array(route)
        extra[f'route{j}_root'] = np.array([gr[0], gr[1]])
        extra[f'route{j}_eps_bar'] = np.asarray(gr[2])
        extra[f'route{j}_D_bar'] = np.asarray(gr[4])
    np.savez_compressed(os.path.join(HERE, 'contour_grad_explicit.npz'), states=states,
                        **extra, residues=np.array(nres),
                        roots=np.array([[gr[0], gr[1]] for gr in grads]),
                        eps_bar=np.stack([gr[2] for gr in grads]),
                        X_bar=np.stack([gr[3] for gr in grads]),
                        D_bar=np.stack([gr[4] for gr in grads]))


if __name__ == '__main__':
    if ONLY == 'c1':
        c1_fixture('literal')
        c1_fixture('calibrated')
        print('C1 fixtures written to', HERE)
        sys.exit(0)
    if ONLY == 'static':
        static_fixture()
        print('static screening fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'unrestricted':
        unrestricted_fixture()
        print('unrestricted fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'sigma_adjoint':
        sigma_adjoint_fixture()
        print('self-energy adjoint fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'sigma_ao':
        sigma_ao_fixture()
        print('AO self-energy fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'isdf':
        isdf_fixture()
        print('ISDF fit fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'drop_in':
        drop_in_fixture()
        print('drop-in call fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'evgw':
        evgw_fixture()
        print('evGW fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'contour':
        contour_fixture()
        print('contour-deformation fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'contour_explicit':
        contour_explicit_fixture()
        print('explicit contour backend fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'contour_unrestricted':
        contour_unrestricted_fixture()
        print('unrestricted contour fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'grad_explicit':
        contour_grad_explicit_fixture()
        print('explicit-route gradient fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'sop':
        sop_fixture()
        print('pole-model fixture written to', HERE)
        sys.exit(0)
    if ONLY == 'follow':
        follow_fixture()
        contour_follow_fixture()
        print('root-following fixtures written to', HERE)
        sys.exit(0)
    if ONLY:
        sys.exit(f'--only {ONLY}: choose c1, static, unrestricted, sigma_adjoint, contour, '
                 'contour_explicit, contour_unrestricted, sigma_ao, evgw, drop_in, isdf, '
                 'follow, sop or grad_explicit')
    grids_fixture()
    shared_kernel_fixture()
    route_fixture('calibrated', 24, 4, 64, 7, 'calibrated', 12, full=True)
    route_fixture('literal16', 20, 3, 48, 3, 'literal', 16)
    route_fixture('calibrated16', 28, 5, 72, 9, 'calibrated', 16)
    qp_fixture()
    static_fixture()
    unrestricted_fixture()
    sigma_adjoint_fixture()
    contour_fixture()
    contour_explicit_fixture()
    contour_unrestricted_fixture()
    sigma_ao_fixture()
    evgw_fixture()
    drop_in_fixture()
    isdf_fixture()
    print('fixtures written to', HERE)
