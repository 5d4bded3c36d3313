"""The CPU oracle and the host-side grid builder, pinned to golden vectors
that MBPTcode itself produced (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from mbptcode_b200 import grids
from oracle import st_oracle as orc


def test_grids_match_reference_bitwise(golden):
    g = golden('grids')
    for i, (n, a, b) in enumerate(g['cases']):
        n = int(n)
        tau, tw = grids.minimax_time_grid(n, a, b)
        om, ow = grids.minimax_frequency_grid(n, a, b)
        assert np.array_equal(tau, g[f'tau_{i}']) and np.array_equal(tw, g[f'tauw_{i}'])
        assert np.array_equal(om, g[f'om_{i}']) and np.array_equal(ow, g[f'omw_{i}'])
        with _quiet():
            tf = grids.TimeFrequencyGrid.minimax(n, a, b)
        for k in ('cosft_wt', 'cosft_tw', 'sinft_wt', 'sinft_tw'):
            assert np.array_equal(getattr(tf, k), g[f'{k}_{i}']), (n, k)
    x, w = grids.gauss_legendre_grid(16, 1.0)
    assert np.array_equal(x, g['gl16']) and np.array_equal(w, g['gl16w'])


class _quiet:
    def __enter__(self):
        import warnings
        self._c = warnings.catch_warnings()
        self._c.__enter__()
        warnings.simplefilter('ignore')

    def __exit__(self, *a):
        self._c.__exit__(*a)


# Laplace-identity known answers of the reference's tests/test_minimax_tau_grid.py
IN_TABLE = [(6, 1.0, 3.0, 1e-6), (8, 1.0, 12.0, 1e-5), (14, 0.3, 30.0, 1e-6),
            (20, 0.3, 30.0, 1e-9), (30, 1.0, 4000.0, 1e-8)]
STRETCHED = [(22, 1.0, 100.0, 1e-9), (24, 1.0, 100.0, 1e-9), (28, 1.0, 100.0, 1e-9),
             (30, 1.0, 100.0, 1e-9), (34, 1.0, 100.0, 1e-9), (34, 0.3, 30.0, 1e-9),
             (30, 2.0, 60.0, 1e-9)]


@pytest.mark.parametrize('n,a,b,tol', IN_TABLE + STRETCHED)
def test_laplace_identity_known_answers(n, a, b, tol):
    tau, w = grids.minimax_time_grid(n, a, b)
    x = np.geomspace(a, b, 2001)
    assert float(np.abs(1.0 - x * (np.exp(-np.outer(x, tau)) @ w)).max()) < tol


def test_refusals():
    with pytest.raises(ValueError):
        grids.minimax_time_grid(7, 1.0, 10.0)
    with pytest.raises(ValueError):
        grids.minimax_time_grid(16, 0.0, 10.0)
    with pytest.raises(ValueError):
        grids.minimax_frequency_grid(16, 1.0, 0.5)


def test_shared_kernel_system(golden):
    g = golden('shared_kernel')
    nocc = int(g['nocc'])
    # five row tiles with a short last one, as in the reference's test
    tile_gb = 5 * 3 * 23 * 8 / 1e9
    proj = orc.polarizability_projected_sweep(g['X'], g['D'], g['eps'], nocc,
                                              g['tau'], tile_gb=tile_gb)
    assert np.allclose(proj, g['proj'], rtol=1e-13, atol=1e-13 * np.abs(g['proj']).max())
    chi0 = np.tensordot(g['cosft_wt'], proj, axes=(1, 0))
    scale = np.abs(g['chi0']).max()
    assert np.abs(chi0 - g['chi0']).max() <= 1e-13 * scale


@pytest.mark.parametrize('name', ['calibrated', 'literal16', 'calibrated16'])
def test_route_matches_reference(golden, name):
    g = golden('route_' + name)
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    with _quiet():
        axes = grids.space_time_axes(eps, nocc, ntau=int(g['ntau']))
    assert np.array_equal(axes.grid.tau_points, g['tau'])
    assert np.array_equal(axes.grid.cosft_wt, g['cosft_wt'])
    assert np.array_equal(axes.tau_sigma, g['tau_sigma'])
    for k in ('Ctw', 'C', 'S'):
        assert np.array_equal(getattr(axes, k), g[k]), k
    out = orc.gw_space_time(X, D, eps, nocc, np.arange(len(eps)), axes)
    if 'chi0' in g:
        s = np.abs(g['chi0']).max()
        assert np.abs(out['chi0'] - g['chi0']).max() <= 1e-12 * s
        s = np.abs(g['W_minus_I']).max()
        assert np.abs(out['W_minus_I'] - g['W_minus_I']).max() <= 1e-11 * s
        s = np.abs(g['Wt']).max()
        assert np.abs(out['Wt'] - g['Wt']).max() <= 1e-11 * s
    s = np.abs(g['sigma']).max()
    assert np.abs(out['sigma'] - g['sigma']).max() <= 1e-10 * s
    # QP roots: the scan's bisection tolerance is 1e-8 Ha
    ok = np.isfinite(g['roots'])
    assert np.array_equal(ok, np.isfinite(out['roots']))
    assert np.abs(out['roots'][ok] - g['roots'][ok]).max() < 2e-8
    e_c = orc.rpa_correlation_energy(X, D, eps, nocc, axes.grid)
    assert abs(e_c - float(g['e_c'])) <= 1e-12 * abs(float(g['e_c'])) + 1e-15
    e2, eb, xb, db = orc.rpa_energy_and_adjoint(X, D, eps, nocc, axes.grid)
    for a, b in ((eb, g['eps_bar']), (xb, g['X_bar']), (db, g['D_bar'])):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max() + 1e-18


def test_qp_known_answers(golden):
    g = golden('qp_kat')
    cases = {
        'two_pole': (lambda w: 0.05 / (w + 0.8) + 0.01 / (w - 0.9), -0.2),
        'one_pole': (lambda w: 0.02 / (w + 0.5), 0.3),
        'satellite': (lambda w: 0.3 / (w + 0.4537) + 0.02 / (w + 1.1129), -0.6),
        'deep': (lambda w: 0.4 / (w - 0.2113) + 0.1 / (w + 3.0171), -2.0),
    }
    for k, (sig, a) in cases.items():
        root, z, qp = orc.solve_qp_equation_pole_strength(lambda w: w - a - sig(w), a)
        assert root == g[k][0] and float(qp) == g[k][1], k
    a = orc.thiele_coefficients(g['thiele_z'], g['thiele_f'])
    assert np.allclose(a, g['thiele_a'], rtol=1e-12)
    fit = orc.PadeFit(g['thiele_z'], g['thiele_f'])
    assert np.array_equal(fit.z, g['greedy_z'])
    assert np.allclose(fit(np.linspace(-1, 1, 7) + 0j), g['greedy_eval'], rtol=1e-10)


def test_static_screening_grid_and_oracle(golden):
    """The static screening W(omega = 0): the auto-sized one-frequency grid is
    the reference's bit for bit, and the oracle's W (restricted, and the
    spin-summed unrestricted form) matches the reference's."""
    g = golden('static')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    n, resid = grids.minimax_points_for_bse(eps, nocc)
    assert n == int(g['ntau']) and resid == float(g['resid'])
    grid = grids.static_screening_grid(eps, nocc)
    assert np.array_equal(grid.tau_points, g['tau'])
    assert np.array_equal(grid.cosft_wt, g['cosft_wt'])
    assert np.array_equal(grid.omega_points, [0.0]) and grid.cosft_tw is None
    g12 = grids.static_screening_grid(eps, nocc, ntau=12)
    assert np.array_equal(g12.tau_points, g['tau12'])
    assert np.array_equal(g12.cosft_wt, g['cosft_wt12'])
    W = orc.static_screening_matrix(X, D, eps, nocc, grid)
    assert np.abs(W - g['W']).max() <= 1e-12
    W12 = orc.static_screening_matrix(X, D, eps, nocc, g12)
    assert np.abs(W12 - g['W12']).max() <= 1e-12
    spectra, noccs = [eps, g['eps_b']], [nocc, int(g['nocc_b'])]
    e_min, e_max = grids.transition_range(spectra, noccs)
    nu = max(grids.minimax_points_for_bse(e, k)[0] for e, k in zip(spectra, noccs))
    with _quiet():
        gu = grids.TimeFrequencyGrid.minimax_split(nu, e_min, e_max, [0.0], [1.0],
                                                   with_sine=False, with_inverse=False)
    Wu = orc.static_screening_matrix_unrestricted([X, g['Xb']], D, spectra, noccs, gu)
    assert np.abs(Wu - g['W_u']).max() <= 1e-12


def test_unrestricted_axes_and_oracle(golden):
    """The unrestricted route: the two-spin axes (chi0's time grid over both
    spins' transitions, W's frequencies and the self-energy's fit ranges
    over both channels) are the reference's bit for bit, and the oracle's
    W - I, Sigma_c diagonals and QP roots of both channels match it."""
    g = golden('unrestricted')
    spectra, noccs = [g['eps_a'], g['eps_b']], [int(g['nocc_a']), int(g['nocc_b'])]
    assert grids.minimax_points_for_gw_unrestricted(spectra, noccs)[0] == int(g['ntau_auto'])
    rW, rS = grids.unrestricted_fit_ranges(spectra, noccs)
    assert rW == tuple(g['rW']) and rS == tuple(g['rS'])
    with _quiet():
        axes = grids.space_time_axes_unrestricted(spectra, noccs, ntau=int(g['ntau']))
    assert np.array_equal(axes.grid.omega_points, g['omega'])
    assert np.array_equal(axes.grid.tau_points, g['tau'])
    assert np.array_equal(axes.grid.cosft_wt, g['cosft_wt'])
    assert np.array_equal(axes.tau_sigma, g['tau_sigma'])
    assert axes.mu == (g['mu_0'], g['mu_1'])
    states = [np.arange(24)] * 2
    out = orc.gw_space_time_unrestricted([g['X_a'], g['X_b']], g['D'], spectra, noccs, states,
                                         axes)
    W = g['W_minus_I']
    assert np.abs(out['W_minus_I'] - W).max() <= 1e-12 * np.abs(W).max()
    for s in range(2):
        sig = g[f'sigma_{s}']
        assert np.abs(out['sigma'][s] - sig).max() <= 1e-10 * np.abs(sig).max()
        assert np.abs(out['roots'][s] - g[f'roots_{s}']).max() < 2e-6


def _sigma_adjoint_case(g):
    nu, wt = g['omega'], g['omega_w']
    eps, nocc = g['eps'], int(g['nocc'])
    gap = eps[nocc] - eps[nocc - 1]
    with _quiet():
        grid = grids.TimeFrequencyGrid.minimax_split(len(g['tau']), 0.5 * gap,
                                                     eps[-1] - eps[0], nu, wt,
                                                     with_sine=False, with_inverse=False)
        tr = grids.sigma_transforms(eps, nocc, grid.tau_points, nu, nu, mu=float(g['mu']))
    return grid, tr


def test_sigma_adjoint_oracle_and_grid_space_form(golden):
    """The self-energy diagonal and its adjoint: the axes and transforms are
    the reference's bit for bit, the oracle (three-index form, as the
    reference writes it) reproduces the reference's Sigma and
    (eps_bar, X_bar, D_bar), and so does the grid-space form that
    mbpt_sigma_backward evaluates on the device (restated here in NumPy:
    Zt = D Wt D^T, the Hadamard reverse, Wt_bar = D^T Zt_bar D)."""
    g = golden('sigma_adjoint')
    X, D, eps, nocc, mu = g['X'], g['D'], g['eps'], int(g['nocc']), float(g['mu'])
    grid, tr = _sigma_adjoint_case(g)
    assert np.array_equal(grid.tau_points, g['tau'])
    assert np.array_equal(grid.cosft_wt, g['cosft_wt'])
    for a, k in zip(tr, ('Ctw', 'C', 'S')):
        assert np.array_equal(a, g[k]), k
    states = g['states']
    sigma, cache = orc.selfenergy_diag(X, D, eps, nocc, grid, states, tr, mu)
    assert np.abs(sigma - g['sigma']).max() <= 1e-12 * np.abs(g['sigma']).max()
    out = orc.selfenergy_diag_backward(g['a_re'], g['a_im'], X, D, eps, nocc, grid, states,
                                       tr, mu, cache)
    for a, k in zip(out, ('eps_bar', 'X_bar', 'D_bar')):
        assert np.abs(a - g[k]).max() <= 1e-10 * np.abs(g[k]).max(), k
    # the grid-space reverse of the self-energy sweep, step for step as on the device
    proj, Wt, _ = cache
    ac, bs = g['a_re'] @ tr[1], g['a_im'] @ tr[2]
    sl, sg = -0.5 * (ac - bs).T, -0.5 * (ac + bs).T
    Xo, Xv = X[:, :nocc], X[:, nocc:]
    eb, xb, db, wtb = np.zeros_like(eps), np.zeros_like(X), np.zeros_like(D), np.zeros_like(Wt)
    Xs = X[:, states]
    for k, tau in enumerate(grid.tau_points):
        w, u = np.exp((eps[:nocc] - mu) * tau), np.exp(-(eps[nocc:] - mu) * tau)
        Go, Gv = (Xo * w) @ Xo.T, (Xv * u) @ Xv.T
        U = D @ Wt[k]
        Zt = U @ D.T
        Xl, Xg = Xs * sl[k], Xs * sg[k]
        Al, Ag = Xl @ Xs.T, Xg @ Xs.T
        Zb, Gob, Gvb, L, H = Go * Al - Gv * Ag, Zt * Al, -Zt * Ag, Go * Zt, Gv * Zt
        np.add.at(xb.T, states, 2.0 * (L @ Xl - H @ Xg).T)
        GoX, GvX = Gob @ Xo, Gvb @ Xv
        xb[:, :nocc] += 2.0 * GoX * w
        xb[:, nocc:] += 2.0 * GvX * u
        eb[:nocc] += tau * w * np.einsum('ri,ri->i', Xo, GoX)
        eb[nocc:] -= tau * u * np.einsum('ra,ra->a', Xv, GvX)
        T = Zb @ D
        wtb[k] = D.T @ T
        db += 2.0 * T @ Wt[k]
    pb = orc.screened_interaction_tau_backward(wtb, proj, grid, tr[0])
    e2, x2, d2 = orc.polarizability_backward(pb, X, D, eps, nocc, grid.tau_points, mu)
    for a, k in zip((eb + e2, xb + x2, db + d2), ('eps_bar', 'X_bar', 'D_bar')):
        assert np.abs(a - g[k]).max() <= 1e-10 * np.abs(g[k]).max(), k


def test_contour_deformation_pieces(golden):
    """The contour-deformation self-energy's host pieces and the oracle
    against the reference (GW/contour_deformation.py, GW/real_screening.py):
    the contour grid bit for bit, the integral weights, the screening
    contraction of three states and Sigma^c around each state's level."""
    from mbptcode_b200 import contour
    g = golden('contour')
    eps, nocc = g['eps'], int(g['nocc'])
    with _quiet():
        nu, nu_w, grid, w0 = contour.cd_frequency_grid(eps, nocc)
    assert np.array_equal(nu, g['nu']) and np.array_equal(nu_w, g['nu_w']) and w0 == g['w0']
    assert np.array_equal(grid.tau_points, g['tau']) and np.array_equal(grid.tau_weights, g['tau_w'])
    assert np.array_equal(grid.cosft_wt, g['cosft_wt'])
    c, dc = contour.cd_integral_weights(g['de'], nu, nu_w)
    assert np.allclose(c, g['c'], rtol=1e-13, atol=0) and np.allclose(dc, g['dc'], rtol=1e-13, atol=0)
    assert np.allclose(orc.cd_integral_weights(g['de'], nu, nu_w), g['c'], rtol=1e-13, atol=0)
    wcs = orc.cd_screening_contraction(g['proj'], g['cosft_wt'], list(g['B']))
    assert np.abs(np.stack(wcs) - g['wc']).max() <= 1e-12 * np.abs(g['wc']).max()
    for i, p in enumerate(g['states']):
        for j, dw in enumerate(g['shifts']):
            s = orc.sigma_cd(int(p), eps[p] + dw, g['B'][i], eps, nocc, nu, nu_w, g['wc'][i],
                             g['proj'], g['tau'], g['tau_w'])
            assert abs(s - g['sigma'][i, j]) <= 1e-11 * abs(g['sigma'][i, j]), (p, dw)
    assert contour.residue_set(eps, nocc, eps[nocc]) == orc.residue_set(eps, nocc, eps[nocc])



def test_contour_root_finder_on_the_oracle(golden):
    """The contour deformation's scan root finder (restated in
    mbptcode_b200.contour from Solvers/qp_equation.py) driven by the oracle's
    Sigma^c and closed-form slope gives the reference's `qp_energy_cd` roots
    and Z for three states around the gap."""
    from mbptcode_b200 import contour
    g = golden('contour')
    eps, nocc = g['eps'], int(g['nocc'])
    args = (g['proj'], g['tau'], g['tau_w'])
    for i, p in enumerate(g['states']):
        p = int(p)
        B, wc = g['B'][i], g['wc'][i]

        def residual(w, p=p, B=B, wc=wc):
            return w - eps[p] - orc.sigma_cd(p, w, B, eps, nocc, g['nu'], g['nu_w'], wc, *args)

        def fprime(w, p=p, B=B, wc=wc):
            return 1.0 - orc.sigma_cd_slope(p, w, B, eps, nocc, g['nu'], g['nu_w'], wc, *args)
        w, z = contour.solve_qp_equation_scan(residual, fprime, float(eps[p]),
                                              refusals=(orc.LaplaceRefused,),
                                              positive_weight=True)
        assert abs(w - g['roots'][i, 0]) < 1e-10 and abs(z - g['roots'][i, 1]) < 1e-9, p


def test_contour_explicit_backend_oracle(golden):
    """The oracle's explicit particle-hole backend (continuation 'cd') against
    the reference: C_ov, W(freq) b and its slope below and above the gap with
    and without broadening, the explicit imaginary-axis contraction, Sigma^c
    with explicit residues, and five states' roots and Z through the scan
    root finder of mbptcode_b200.contour."""
    from mbptcode_b200 import contour
    g = golden('contour_explicit')
    eps, nocc, X, D = g['eps'], int(g['nocc']), g['X'], g['D']
    C = orc.three_index_ov(X, D, eps, nocc)
    assert np.abs(C - g['C_ov']).max() <= 1e-13 * np.abs(g['C_ov']).max()
    d = orc.ov_energies(eps, nocc)
    for a, eta in enumerate(g['etas']):
        for j, f in enumerate(g['freqs']):
            y = orc.explicit_screening_apply(C, d, f, g['b'], eta)
            ref = g['apply'][a, j]
            assert np.abs(y - ref).max() <= 1e-11 * np.abs(ref).max(), (eta, f)
            s = orc.explicit_screening_slope(C, d, f, y, eta)
            assert abs(s - g['slope'][a, j]) <= 1e-10 * abs(g['slope'][a, j]), (eta, f)
    B = [orc.three_index_slice(X, D, int(p)) for p in g['states']]
    for r, i in enumerate(g['near']):
        wcx = orc.wc_explicit(B[i], C, d, g['nu'])
        assert np.abs(wcx - g['wc_explicit'][r]).max() <= 1e-11 * np.abs(wcx).max()
        p = int(g['states'][i])
        for j, dw in enumerate(g['shifts']):
            s = orc.sigma_cd_explicit(p, eps[p] + dw, B[i], eps, nocc, g['nu'], g['nu_w'],
                                      g['wc'][i], C)
            assert abs(s - g['sigma'][r, j]) <= 1e-11 * abs(g['sigma'][r, j]), (p, dw)
    for i, p in enumerate(g['states']):
        p = int(p)

        def residual(w, p=p, i=i):
            return w - eps[p] - orc.sigma_cd_explicit(p, w, B[i], eps, nocc, g['nu'],
                                                      g['nu_w'], g['wc'][i], C)

        def fprime(w, p=p, i=i):
            return 1.0 - orc.sigma_cd_slope_explicit(p, w, B[i], eps, nocc, g['nu'],
                                                     g['nu_w'], g['wc'][i], C)
        w, z = contour.solve_qp_equation_scan(residual, fprime, float(eps[p]),
                                              positive_weight=True)
        assert abs(w - g['roots'][i, 0]) < 1e-10 and abs(z - g['roots'][i, 1]) < 1e-9, p


def test_contour_unrestricted_oracle(golden):
    """The contour of an unrestricted reference against the reference's
    composition: the grid on both spins' pair energies (host code, bit for
    bit), the oracle's spin-summed proj(tau) and each channel's contraction,
    and each channel's roots and Z through the scan root finder with the
    Laplace residues (on both spins' pair energies) and the explicit ones
    (both spins' C_ov side by side at 1/sqrt(2))."""
    from mbptcode_b200 import contour
    g = golden('contour_unrestricted')
    X_mos, D = [g['X_a'], g['X_b']], g['D']
    spectra, noccs = [g['eps_a'], g['eps_b']], [int(g['nocc_a']), int(g['nocc_b'])]
    pairs = np.concatenate([orc.ov_energies(e, n) for e, n in zip(spectra, noccs)])
    assert np.array_equal(pairs, g['pairs'])
    with _quiet():
        nu, nu_w, grid, w0 = contour.cd_frequency_grid(spectra[0], noccs[0], pair_energies=pairs)
    assert np.array_equal(nu, g['nu']) and np.array_equal(nu_w, g['nu_w']) and w0 == g['w0']
    assert np.array_equal(grid.tau_points, g['tau']) and np.array_equal(grid.cosft_wt,
                                                                       g['cosft_wt'])
    proj = 0.5 * sum(orc.polarizability_projected_sweep(X, D, e, n, g['tau'])
                     for X, e, n in zip(X_mos, spectra, noccs))
    assert np.abs(proj - g['proj']).max() <= 1e-12 * np.abs(g['proj']).max()
    C = np.hstack([orc.three_index_ov(X, D, e, n)
                   for X, e, n in zip(X_mos, spectra, noccs)]) / np.sqrt(2.0)
    for s, (X, e, n) in enumerate(zip(X_mos, spectra, noccs)):
        B = [orc.three_index_slice(X, D, int(p)) for p in g[f'states_{s}']]
        wcs = orc.cd_screening_contraction(g['proj'], g['cosft_wt'], B)
        assert np.abs(np.stack(wcs) - g[f'wc_{s}']).max() <= 1e-12 * np.abs(g[f'wc_{s}']).max()
        for i, p in enumerate(g[f'states_{s}']):
            p, wc = int(p), g[f'wc_{s}'][i]
            lap = dict(pair_energies=pairs)
            roots = {}
            for name, sig, slope, extra in (
                    ('laplace', orc.sigma_cd, orc.sigma_cd_slope,
                     (g['proj'], g['tau'], g['tau_w'])),
                    ('cd', orc.sigma_cd_explicit, orc.sigma_cd_slope_explicit, (C,))):
                def residual(w, p=p, i=i, sig=sig, extra=extra):
                    return w - e[p] - sig(p, w, B[i], e, n, nu, nu_w, wc, *extra, **lap)

                def fprime(w, p=p, i=i, slope=slope, extra=extra):
                    return 1.0 - slope(p, w, B[i], e, n, nu, nu_w, wc, *extra, **lap)
                roots[name] = contour.solve_qp_equation_scan(residual, fprime, float(e[p]),
                                                             refusals=(orc.LaplaceRefused,),
                                                             positive_weight=True)
            for name in ('laplace', 'cd'):
                want = g[f'roots_{name}_{s}'][i]
                w, z = roots[name]
                assert abs(w - want[0]) < 1e-10 and abs(z - want[1]) < 1e-9, (s, p, name)


def test_ao_self_energy_oracle(golden):
    """The oracle's full AO self-energy (an AO collocation that is not the MO
    one) and the chi0 sweep's reverse against the reference's."""
    g = golden('sigma_ao')
    args = (g['X_ao'], g['D'], g['W'], g['mo'], g['eps'], int(g['nocc']), g['tau_sigma'],
            g['omega'], g['pade'], float(g['mu']))
    sig = orc.self_energy_matrix(*args)
    assert np.abs(sig - g['sigma']).max() <= 1e-10 * np.abs(g['sigma']).max()
    sub = orc.self_energy_matrix(*args, tau_indices=[1, 4, 7])
    assert np.abs(sub - g['sigma_sub']).max() <= 1e-10 * np.abs(g['sigma_sub']).max()


def test_contour_qp_gradient_oracle(golden):
    """The oracle's gradient of a contour-deformation QP energy (Laplace
    residues) against the reference's qp_gradient_space_time for three
    states around the gap."""
    g = golden('contour')
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    for i, p in enumerate(g['states']):
        w, z = g['grad_roots'][i]
        eb, xb, db = orc.qp_gradient_laplace(g['X'], g['D'], eps, nocc, g['tau'], g['tau_w'],
                                             g['cosft_wt'], g['nu'], g['nu_w'], int(p), mu, w, z)
        for a, k in ((eb, 'eps_bar'), (xb, 'X_bar'), (db, 'D_bar')):
            ref = g[k][i]
            assert np.abs(a - ref).max() <= 1e-9 * np.abs(ref).max(), (int(p), k)


def test_isdf_fit_oracle(golden):
    """The separable-RI fit restated in the oracle against the reference's
    own estimator, metric root and D = M^T V^1/2 (tests/golden/isdf.npz)."""
    g = golden('isdf')
    M = orc.isdf_fit_products(g['ao'], g['second'], g['w'], g['aux'], g['FD'])
    assert np.abs(M - g['M']).max() <= 1e-9 * np.abs(g['M']).max()
    root = orc.aux_metric_root(g['V'])
    assert np.abs(root - g['root']).max() <= 1e-12 * np.abs(g['root']).max()
    assert np.abs(M.T @ root - g['D_factor']).max() <= 1e-9 * np.abs(g['D_factor']).max()
