"""Device parity: libmbpt_b200 against the CPU oracle and the reference's
golden vectors, through the C ABI (via the package's ctypes binding).

Tolerances: FP64 mode agrees with the FP64 oracle to ~1e-10 relative (the
same arithmetic in another summation order), and so does 'fp64_int8' (the
products emulated on the int8 tensor cores with 8 seven-bit digits, ~5e-15
of the operands' scale per product); mixed mode (split-BF16 3-term
products, FP32 accumulation) to 2e-5 relative on chi0-sized quantities."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from mbptcode_b200 import grids                       # noqa: E402
from mbptcode_b200 import space_time as st            # noqa: E402
from mbptcode_b200 import gw                           # noqa: E402
from mbptcode_b200 import _lib                         # noqa: E402
from mbptcode_b200.synthetic import synthetic_system   # noqa: E402
from oracle import st_oracle as orc                    # noqa: E402

FP64_REL = 1e-10
MIXED_REL = 2e-5


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope='module')
def dev():
    return _lib.require_device()


@pytest.mark.parametrize('kind,tol', [('bf16', 3e-5), ('tf32', 2e-6)])
@pytest.mark.parametrize('m,n,k', [(300, 260, 200), (128, 128, 64), (1000, 700, 1100),
                                   (17, 5, 3)])
def test_split_gemm_matches_fp64(dev, m, n, k, kind, tol):
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((n, k))
    Ad = torch.as_tensor(A, device=dev)
    Bd = torch.as_tensor(B, device=dev)
    C = torch.empty((m, n), dtype=torch.float32, device=dev)
    lib = _lib.lib()
    size = (lib.mbpt_gemm_split_workspace_bytes if kind == 'bf16'
            else lib.mbpt_gemm_split_tf32_workspace_bytes)(m, n, k)
    fn = lib.mbpt_gemm_split if kind == 'bf16' else lib.mbpt_gemm_split_tf32
    ws = torch.empty(size, dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(fn(_lib.ptr(Ad), _lib.ptr(Bd), m, n, k, 1.0, _lib.ptr(C), n, _lib.ptr(ws),
                  ws.numel(), _lib.ptr(err), _lib.stream_ptr()), 'gemm')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A @ B.T
    # per-entry error against the scale of the products that were summed:
    # 2^-18 per BF16x3 product, 2^-22 per TF32x3 product, FP32 accumulation
    scale = np.sqrt(k) * np.abs(A).max() * np.abs(B).max()
    assert np.abs(C.cpu().numpy() - ref).max() <= tol * scale


@pytest.mark.parametrize('precision,tol', [('fp64', FP64_REL), ('mixed', MIXED_REL),
                                           ('fp64_int8', FP64_REL)])
def test_chi0_matches_reference_golden(golden, precision, tol):
    g = golden('route_calibrated')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    axes = grids.space_time_axes(eps, nocc, ntau=int(g['ntau']))
    chi0 = st.chi0_imaginary_frequency(X, D, eps, nocc, axes.grid, precision=precision)
    assert rel(chi0, g['chi0']) < tol


@pytest.mark.parametrize('precision,tol', [('fp64', FP64_REL), ('mixed', MIXED_REL),
                                           ('fp64_int8', FP64_REL)])
def test_shared_kernel_system(golden, precision, tol):
    g = golden('shared_kernel')
    proj = st.polarizability_projected_sweep(g['X'], g['D'], g['eps'], int(g['nocc']),
                                             g['tau'], precision=precision)
    assert rel(proj, g['proj']) < tol


def test_dyson_and_transform_match_oracle(golden):
    g = golden('route_calibrated')
    W = st.dyson_screening(g['chi0'], correlation=True)
    assert rel(W, g['W_minus_I']) < 1e-11
    Wt = gw.w_tau_from_frequencies(torch.as_tensor(g['W_minus_I'], device='cuda'), g['Ctw'])
    assert rel(Wt.cpu().numpy(), g['Wt']) < 1e-12


@pytest.mark.parametrize('n', [96, 300, 1000])
def test_dyson_inverse_both_modes(n, monkeypatch):
    """W - I from the Cholesky factor (shared-memory diagonal blocks, the
    recursive triangular inverse, L^-T L^-1) against torch's FP64 inverse:
    FP64 mode to rounding; mixed mode to 5e-6 absolute. 1 - chi0 >= I puts
    every eigenvalue of W in (0, 1], so each entry of L^-T L^-1 is a sum
    bounded by 1, which TF32 pairs (2^-22 per factor) and FP32 accumulation
    (drained every 64 terms) reproduce to a few 2^-22. The mixed L^-T L^-1
    runs on CTA pairs with triangular K spans per pair (1, 3 and 8 row
    tiles); one CTA per tile (MBPT_ENGINE_PAIRS=0) agrees within 1e-9."""
    g = torch.Generator(device='cpu').manual_seed(n)
    A = torch.randn(n, n // 2 + 7, generator=g, dtype=torch.float64)
    chi0 = -(A @ A.T) / n * 3.0
    chi0 = torch.stack([chi0, 0.25 * chi0]).cuda()
    eye = torch.eye(n, dtype=torch.float64, device='cuda')
    ref = torch.linalg.inv(eye - chi0)
    ref.diagonal(dim1=-2, dim2=-1).sub_(1.0)
    out = {}
    for prec in ('fp64', 'mixed'):
        c = chi0.clone()
        logdet, trace, info, _ = st.dyson_batch(c, want_w=True, precision=prec)
        assert not np.any(info)
        out[prec] = (c, logdet)
    monkeypatch.setenv('MBPT_ENGINE_PAIRS', '0')
    c = chi0.clone()
    st.dyson_batch(c, want_w=True, precision='mixed')
    monkeypatch.delenv('MBPT_ENGINE_PAIRS')
    assert float((c - out['mixed'][0]).abs().max()) < 1e-9
    assert float((out['fp64'][0] - ref).abs().max()) < 1e-12
    err_mixed = float((out['mixed'][0] - ref).abs().max())
    print(f'n={n}: mixed max |W - W_ref| {err_mixed:.3e}')
    assert err_mixed < 5e-6
    # the factorisation and log-determinant are FP64 in both modes
    assert torch.equal(out['fp64'][1], out['mixed'][1])
    want = torch.linalg.slogdet(eye - chi0)[1]
    assert float((out['fp64'][1] - want).abs().max()) < 1e-10 * n


def frontier(nocc, n, width=4):
    return np.arange(max(0, nocc - width), min(n, nocc + width))


@pytest.mark.parametrize('name', ['calibrated', 'literal16', 'calibrated16'])
def test_route_fp64_matches_reference_golden(golden, name):
    g = golden('route_' + name)
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    res = gw.gw_sweep(X, D, eps, nocc, ntau=int(g['ntau']), precision='fp64')
    sigma = res['sigma'].cpu().numpy()
    assert rel(sigma, g['sigma']) < 1e-9
    roots = res['roots'].cpu().numpy()
    ok = np.isfinite(g['roots'])
    assert np.array_equal(ok, np.isfinite(roots))
    # frontier roots to the scan's bisection tolerance; states far from the
    # gap sit where the 16-node Pade continuation amplifies the last bits of
    # Sigma (1e-12 relative) into roots that move by up to ~1e-6 Ha
    f = frontier(nocc, len(eps))
    assert np.abs(roots[f] - g['roots'][f]).max() < 5e-8
    assert np.abs(roots[ok] - g['roots'][ok]).max() < 2e-6


def test_route_mixed_within_qp_tolerance(golden):
    g = golden('route_calibrated')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    res = gw.gw_sweep(X, D, eps, nocc, ntau=int(g['ntau']), precision='mixed')
    roots = res['roots'].cpu().numpy()
    f = frontier(nocc, len(eps))
    # the 10 meV bar of the precision configuration, in Hartree, on the
    # HOMO/LUMO region the bar is stated for
    assert np.abs(roots[f] - g['roots'][f]).max() < 10e-3 / 27.211386


def test_mixed_refuses_ill_conditioned_transforms(golden):
    # at 16 points the unregularised tau -> omega weights reach ~1e9, and a
    # 1e-5 relative product error no longer survives the cancellation
    g = golden('route_calibrated16')
    with pytest.raises(ValueError, match='mixed precision'):
        gw.gw_sweep(g['X'], g['D'], g['eps'], int(g['nocc']), ntau=16, precision='mixed')


@pytest.mark.parametrize('precision,tol,names', [
    ('fp64', 1e-11, ('calibrated', 'calibrated16', 'literal16')),
    ('mixed', 2e-5, ('calibrated',)),
    ('fp64_int8', 1e-11, ('calibrated',)),
    # the int8 emulation's per-product error changes erratically from one tau
    # point to the next, and the 16-point transforms (weights 2.4e8, 8.9e8)
    # amplify it to ~1e-9 relative; the adjoints pick native FP64 there
    ('fp64_int8', 1e-8, ('calibrated16', 'literal16'))])
def test_rpa_energy_matches_reference_golden(golden, precision, tol, names):
    for name in names:
        g = golden('route_' + name)
        axes = grids.space_time_axes(g['eps'], int(g['nocc']), ntau=int(g['ntau']))
        e = st.rpa_correlation_energy_space_time(g['X'], g['D'], g['eps'], int(g['nocc']),
                                                 axes.grid, precision=precision)
        ref = float(g['e_c'])
        # absolute floor: the 16-point weights turn FP64 rounding into ~1e-13 Ha
        assert abs(e - ref) <= tol * abs(ref) + 1e-12, (name, e, ref)


def test_odd_sizes_against_oracle():
    # M not a multiple of 128, naux != M, nocc/nvirt not multiples of 64
    rng = np.random.default_rng(4)
    M, n, nocc, naux = 301, 37, 5, 173
    X = rng.standard_normal((M, n)) * 0.08
    D = rng.standard_normal((M, naux)) * 0.08
    eps = np.sort(np.concatenate([rng.uniform(-1.2, -0.4, nocc),
                                  rng.uniform(0.1, 3.0, n - nocc)]))
    axes = grids.space_time_axes(eps, nocc, ntau=12)
    ref = orc.chi0_imaginary_frequency(X, D, eps, nocc, axes.grid)
    for precision, tol in (('fp64', FP64_REL), ('mixed', MIXED_REL), ('fp64_int8', FP64_REL)):
        got = st.chi0_imaginary_frequency(X, D, eps, nocc, axes.grid, precision=precision)
        assert rel(got, ref) < tol, precision
    W = np.stack([orc.dyson_screening(c, True) for c in ref])
    Wt = np.tensordot(axes.Ctw, W, axes=(1, 0))
    states = [0, 3, 4, 5, 9, 36]
    br = orc.sigma_branch_sums(X, D, Wt, eps, nocc, axes.tau_sigma, axes.mu, states)
    for precision, tol in (('fp64', 1e-10), ('mixed', 5e-5), ('fp64_int8', 1e-10)):
        got = gw.sigma_branch_sums(X, D, torch.as_tensor(Wt, device='cuda'), eps, nocc,
                                   axes.tau_sigma, states, axes.mu, precision=precision)
        assert rel(got.cpu().numpy(), br) < tol, precision


def test_qp_kernel_on_oracle_sigma(golden):
    # the device Pade + root search on the reference's own Sigma_c diagonal
    g = golden('route_calibrated16')
    eps, nocc = g['eps'], int(g['nocc'])
    sig = torch.as_tensor(g['sigma'], device='cuda')
    roots, z, flags, evals = gw.qp_solve(sig, g['pade'], eps, np.arange(len(eps)), nocc,
                                         float(g['mu']))
    roots = roots.cpu().numpy()
    ok = np.isfinite(g['roots'])
    assert np.abs(roots[ok] - g['roots'][ok]).max() < 5e-8


def test_synthetic_literal_is_weak_and_calibrated_is_not():
    for variant in ('literal', 'calibrated'):
        X, D, eps = synthetic_system(60, 6, 240, seed=2, variant=variant)
        axes = grids.space_time_axes(eps, 6, ntau=16)
        e = st.rpa_correlation_energy_space_time(X, D, eps, 6, axes.grid)
        e_ref = orc.rpa_correlation_energy(X, D, eps, 6, axes.grid)
        assert abs(e - e_ref) <= 1e-10 * abs(e_ref) + 1e-12
        if variant == 'literal':
            assert abs(e_ref) < 1e-8      # nearly non-interacting
        else:
            assert abs(e_ref) > 1e-2


def test_planted_nonpositive_dielectric_is_flagged():
    # the reference's planted-input test (tests/test_rpa_log_determinant.py):
    # one eigenvalue of chi0 at 1.5 makes det(1 - chi0) negative; the
    # Cholesky fails, the LU fallback gives log|det| and the inverse, and the
    # frequency is flagged
    rng = np.random.default_rng(1)
    n = 40
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = -rng.uniform(0.1, 2.0, n)
    lam[0] = 1.5
    c = (Q * lam) @ Q.T
    flags = {}
    with pytest.warns(st.NonPositiveDielectric):
        ld = st.dielectric_log_determinant(np.eye(n) - c, 3, flags)
    sign, ref = np.linalg.slogdet(np.eye(n) - c)
    assert sign < 0 and abs(ld - ref) < 1e-10
    assert flags['nonpositive_det'] == [3]
    W = st.dyson_screening(c, correlation=True)
    assert rel(W, np.linalg.inv(np.eye(n) - c) - np.eye(n)) < 1e-10



def test_deferred_dyson_reports_on_the_device_and_the_sweep_repeats():
    """The Dyson step without a host wait: the info words come back on the
    device (the non-positive-definite frequency flagged, the others' log-
    determinants and W - I equal to the synchronous step's), and a sweep that
    meets such a frequency is repeated with the LU fallback, giving the same
    result as the synchronous sweep."""
    rng = np.random.default_rng(7)
    n = 300
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    mats = []
    for f in range(4):
        lam = -rng.uniform(0.05, 3.0, n)
        if f == 1:
            lam[5] = 1.4
        mats.append((Q * lam) @ Q.T)
    c_sync = torch.as_tensor(np.stack(mats), device='cuda')
    c_def = c_sync.clone()
    ld_s, _, info_s, _ = st.dyson_batch(c_sync, want_w=True, precision='fp64')
    ld_d, _, info_d, sign_d = st.dyson_batch(c_def, want_w=True, precision='fp64',
                                             deferred=True)
    assert isinstance(info_d, torch.Tensor) and sign_d is None
    info_d = info_d.cpu().numpy()
    assert list(info_d != 0) == [False, True, False, False]
    ok = [0, 2, 3]
    assert np.abs(ld_d.cpu().numpy()[ok] - ld_s.cpu().numpy()[ok]).max() < 1e-12
    assert rel(c_def[ok].cpu().numpy(), c_sync[ok].cpu().numpy()) < 1e-13
    # a sweep whose deferred step reports a failed frequency (on the imaginary
    # axis 1 - chi0 >= I for any physical system, so the report is planted by
    # a wrapper around the step) is repeated with the synchronous step
    from mbptcode_b200.synthetic import synthetic_system
    X, D, eps = synthetic_system(40, 5, 200, seed=1, variant='calibrated')
    axes = grids.space_time_axes(eps, 5, ntau=12)
    real, calls = gw.dyson_batch, []

    def planted(chi0, *args, deferred=False, **kw):
        calls.append(deferred)
        out = real(chi0, *args, deferred=deferred, **kw)
        if deferred:
            out[2][0] = 3
        return out
    gw.dyson_batch = planted
    try:
        a = gw.gw_sweep(X, D, eps, 5, axes=axes, precision='fp64')
    finally:
        gw.dyson_batch = real
    b = gw.gw_sweep(X, D, eps, 5, axes=axes, precision='fp64', _deferred=False)
    assert calls == [True, False]
    assert not a['dyson_info'].any()
    ra, rb = a['roots'].cpu().numpy(), b['roots'].cpu().numpy()
    assert np.array_equal(np.isnan(ra), np.isnan(rb))
    fin = np.isfinite(ra)
    assert np.abs(ra[fin] - rb[fin]).max() < 1e-12
    assert abs(float(a['e_c']) - float(b['e_c'])) <= 1e-12 * abs(float(b['e_c']))


@pytest.mark.parametrize('prec', ['fp64', 'mixed'])
def test_dyson_batch_with_failed_frequency_inside(prec):
    """Four frequencies, the second not positive definite: the batched
    Cholesky of all four flags it (its other factors are unaffected), the
    inverses of the others run on the side stream, the failed one takes the
    LU fallback after the streams drain, restored from the triangle the
    factorisation left untouched; every output must match the dense FP64
    answer and only the failed frequency is flagged."""
    rng = np.random.default_rng(7)
    n = 300
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    mats = []
    for f in range(4):
        lam = -rng.uniform(0.05, 3.0, n)
        if f == 1:
            lam[5] = 1.4
        mats.append((Q * lam) @ Q.T)
    chi0 = torch.as_tensor(np.stack(mats), device='cuda')
    logdet, trace, info, sign = st.dyson_batch(chi0, want_w=True, precision=prec)
    assert list(info != 0) == [False, True, False, False]
    assert list(sign) == [1, -1, 1, 1]
    tol = 1e-10 if prec == 'fp64' else 5e-6
    for f, c in enumerate(mats):
        one_minus = np.eye(n) - c
        s_ref, ld_ref = np.linalg.slogdet(one_minus)
        assert abs(float(logdet[f]) - ld_ref) < 1e-9 * n
        assert abs(float(trace[f]) - np.trace(c)) < 1e-9 * n
        W_ref = np.linalg.inv(one_minus) - np.eye(n)
        # the LU frequency is FP64 in both modes
        err = np.abs(chi0[f].cpu().numpy() - W_ref).max()
        assert err < (1e-10 if f == 1 else tol) * max(1.0, np.abs(W_ref).max()), (f, err)


@pytest.mark.parametrize('prec', ['fp64', 'mixed'])
def test_sigma_branch_sums_identity_w(prec):
    """Wt omitted stands for W = I at every tau: the same branch sums as an
    explicit identity stack (the exchange diagonal's path, which skips the
    D W product and the W conversion)."""
    n, nocc, M = 60, 8, 256
    X, D, eps = synthetic_system(n, nocc, M, seed=31, variant='calibrated')
    mu = st.particle_hole_window(eps, nocc)[2]
    taus = [0.0, 0.7]
    states = np.arange(n)
    eye = np.broadcast_to(np.eye(M), (2, M, M)).copy()
    a = gw.sigma_branch_sums(X, D, None, eps, nocc, taus, states, mu, precision=prec)
    b = gw.sigma_branch_sums(X, D, eye, eps, nocc, taus, states, mu, precision=prec)
    tol = 1e-12 if prec == 'fp64' else MIXED_REL
    assert rel(a.cpu().numpy(), b.cpu().numpy()) < tol


def test_bounded_wait_gives_up_and_context_survives(dev):
    """Failure detection without a fault: a barrier that nothing completes
    makes the engine's wait routine give up after its limit (20 ms here) and
    report MBPT_ERR_TIMEOUT through the error word; the kernel returns, and
    the same context then runs a tensor-core product correctly."""
    lib = _lib.lib()
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.mbpt_wait_selftest(0, 20000, _lib.ptr(err), _lib.stream_ptr()), 'selftest')
    torch.cuda.synchronize()
    assert int(err.item()) == _lib.ERR_TIMEOUT
    err.zero_()
    _lib.check(lib.mbpt_wait_selftest(1, 20000, _lib.ptr(err), _lib.stream_ptr()), 'selftest')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert lib.mbpt_wait_selftest(0, 0, _lib.ptr(err), _lib.stream_ptr()) == _lib.ERR_SHAPE
    # the context still works
    rng = np.random.default_rng(3)
    A, B = rng.standard_normal((200, 96)), rng.standard_normal((150, 96))
    C = torch.empty((200, 150), dtype=torch.float32, device=dev)
    ws = torch.empty(lib.mbpt_gemm_split_workspace_bytes(200, 150, 96), dtype=torch.uint8,
                     device=dev)
    Ad, Bd = torch.as_tensor(A, device=dev), torch.as_tensor(B, device=dev)  # kept alive
    _lib.check(lib.mbpt_gemm_split(_lib.ptr(Ad), _lib.ptr(Bd), 200, 150, 96, 1.0,
                                   _lib.ptr(C), 150, _lib.ptr(ws), ws.numel(), _lib.ptr(err),
                                   _lib.stream_ptr()), 'gemm')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert np.abs(C.cpu().numpy() - A @ B.T).max() < 3e-5 * np.sqrt(96) * 16


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-11), ('mixed', 5e-5)])
def test_static_screening_matches_reference_golden(golden, precision, tol):
    """W(omega = 0) = [1 - chi0(0)]^-1 of the BSE kernel on the auto-sized
    one-frequency grid and on 12 points, restricted and spin-summed
    unrestricted, against the reference's W (entries bounded by 1, so the
    bars are absolute: FP64 to rounding, mixed within the split products'
    error on chi0)."""
    g = golden('static')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    W = st.static_screening_matrix(X, D, eps, nocc, precision=precision)
    assert isinstance(W, np.ndarray) and W.shape == g['W'].shape
    assert np.abs(W - g['W']).max() < tol
    W12 = st.static_screening_matrix(X, D, eps, nocc, grids.static_screening_grid(eps, nocc, 12),
                                     precision=precision)
    assert np.abs(W12 - g['W12']).max() < tol
    Wb = st.static_screening_matrix(None, D, eps, nocc, precision=precision,
                                    branches=(X[:, :nocc], X[:, nocc:]))
    assert np.array_equal(Wb, W)
    Wu = st.static_screening_matrix_unrestricted([X, g['Xb']], D, [eps, g['eps_b']],
                                                 [nocc, int(g['nocc_b'])], precision=precision)
    assert np.abs(Wu - g['W_u']).max() < tol
    if precision == 'fp64':
        grid = grids.static_screening_grid(eps, nocc)
        chi0 = st.spin_summed(st.chi0_imaginary_frequency, [X, X], D, [eps, eps],
                              [nocc, nocc], grid)
        assert rel(chi0, orc.chi0_imaginary_frequency(X, D, eps, nocc, grid)) < FP64_REL


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_unrestricted_route_matches_reference_golden(golden, precision):
    """Two spin channels, one W from the spin-summed chi0, each channel's
    Sigma_c diagonal and QP roots against the reference's composition: FP64
    to rounding (frontier roots to the scan's tolerance), mixed within the
    QP bar (10 meV) on the frontier states."""
    g = golden('unrestricted')
    X_mos = [g['X_a'], g['X_b']]
    spectra, noccs = [g['eps_a'], g['eps_b']], [int(g['nocc_a']), int(g['nocc_b'])]
    res = gw.gw_sweep_unrestricted(X_mos, g['D'], spectra, noccs, ntau=int(g['ntau']),
                                   precision=precision)
    assert res['axes'].ntau == int(g['ntau'])
    for s in range(2):
        sigma = res['channels'][s]['sigma'].cpu().numpy()
        roots = res['channels'][s]['roots'].cpu().numpy()
        ref = g[f'roots_{s}']
        f = frontier(noccs[s], len(spectra[s]))
        if precision == 'fp64':
            assert rel(sigma, g[f'sigma_{s}']) < 1e-9
            assert np.abs(roots[f] - ref[f]).max() < 5e-8
            assert np.abs(roots - ref).max() < 2e-6
        else:
            assert rel(sigma, g[f'sigma_{s}']) < 1e-4
            assert np.abs(roots[f] - ref[f]).max() * 27.211386 < 10e-3


def test_unrestricted_closed_shell_equals_restricted(golden):
    """A closed shell run unrestricted reads every grid the restricted route
    reads and halves twice its own chi0: the roots are the restricted ones."""
    g = golden('route_calibrated')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    r = gw.gw_sweep(X, D, eps, nocc, ntau=int(g['ntau']), precision='fp64')
    u = gw.gw_sweep_unrestricted([X, X], D, [eps, eps], [nocc, nocc], ntau=int(g['ntau']),
                                 precision='fp64')
    for s in range(2):
        assert torch.equal(u['channels'][s]['roots'], r['roots'])
    assert float(u['e_c']) == float(r['e_c'])


def test_unrestricted_driver_channel(golden):
    """solve_qp_energy_space_time on an unrestricted mean field: the channel's
    collocation is X_ao C_s (here C_s = I, X_ao the alpha collocation for both
    spins with the beta spectrum), nocc = (nalpha, nbeta)."""
    g = golden('unrestricted')
    X, D = g['X_a'], g['D']
    eps2 = np.stack([g['eps_a'], g['eps_a']])

    class MF:
        mo_energy = eps2
        mo_coeff = [np.eye(24), np.eye(24)]
    n = int(g['nocc_a'])
    got = gw.solve_qp_energy_space_time(MF, None, (n, n), np.arange(n - 2, n + 2),
                                        factors=(X, D, X), spin_channel='beta')
    ref = gw.gw_sweep_unrestricted([X, X], D, [g['eps_a']] * 2, [n, n],
                                   states=[None, np.arange(n - 2, n + 2)], channels=(1,))
    assert np.array_equal(got, ref['channels'][1]['roots'].cpu().numpy())
    with pytest.raises(ValueError):
        gw.solve_qp_energy_space_time(MF, None, (n, n), 0, factors=(X, D))


@pytest.mark.parametrize('precision', ['fp64', 'mixed'])
def test_frequency_blocked_screening(golden, precision):
    """freq_block: chi0 held for 5 of the 12 frequencies at a time (blocks of
    5, 5, 2; the tau sweep recomputed per block) gives the unblocked sweep's
    W(tau), E_c and roots up to the order of the W(tau) sums, and, in FP64,
    the reference's Sigma_c diagonal."""
    g = golden('route_calibrated')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    axes = grids.space_time_axes(eps, nocc, ntau=int(g['ntau']))
    full = gw.gw_sweep(X, D, eps, nocc, axes=axes, precision=precision, keep=True)
    blk = gw.gw_sweep(X, D, eps, nocc, axes=axes, precision=precision, keep=True, freq_block=5)
    assert rel(blk['Wt'].cpu().numpy(), full['Wt'].cpu().numpy()) < 1e-12
    assert abs(float(blk['e_c']) - float(full['e_c'])) <= 1e-12 * abs(float(full['e_c']))
    assert np.array_equal(blk['dyson_info'], full['dyson_info'])
    r_b, r_f = blk['roots'].cpu().numpy(), full['roots'].cpu().numpy()
    f = frontier(nocc, len(eps))
    assert np.abs(r_b[f] - r_f[f]).max() < 1e-9
    if precision == 'fp64':
        assert rel(blk['sigma'].cpu().numpy(), g['sigma']) < 1e-9


def test_driver_freq_block_and_scratch_dir(golden):
    g = golden('route_calibrated')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    states = np.arange(nocc - 2, nocc + 2)

    class Quad:
        ntau_st, npade, w0_gl = int(g['ntau']), 16, 1.0

    class Num:
        quadrature = Quad
    a = gw.solve_qp_energy_space_time(eps, None, nocc, states, numerics=Num, factors=(X, D))
    b = gw.solve_qp_energy_space_time(eps, None, nocc, states, numerics=Num, factors=(X, D),
                                      freq_block=4)
    assert np.abs(a - b).max() < 1e-9
    with pytest.raises(NotImplementedError):
        gw.solve_qp_energy_space_time(eps, None, nocc, states, numerics=Num, factors=(X, D),
                                      freq_block=4, scratch_dir='/tmp/x')


@pytest.mark.parametrize('n', [96, 1000, 1200])
def test_dyson_batched_cholesky(n):
    """Five frequencies take the batched left-looking Cholesky (128-column
    steps: one batched DGEMM update, the diagonal blocks factorised and
    inverted in shared memory, one batched DGEMM panel; n = 1000 and 1200
    end on a partial block): log-determinants against slogdet, W - I against
    the FP64 inverse, FP64 mode to rounding and mixed mode to 5e-6."""
    g = torch.Generator(device='cpu').manual_seed(n + 5)
    A = torch.randn(5, n, n // 2 + 3, generator=g, dtype=torch.float64)
    scale = torch.tensor([3.0, 0.5, 1.0, 2.0, 0.1], dtype=torch.float64)[:, None, None]
    chi0 = (-(A @ A.transpose(1, 2)) / n * scale).cuda()
    eye = torch.eye(n, dtype=torch.float64, device='cuda')
    ref = torch.linalg.inv(eye - chi0) - eye
    want = torch.linalg.slogdet(eye - chi0)[1]
    for prec, tol in (('fp64', 1e-12), ('mixed', 5e-6)):
        c = chi0.clone()
        logdet, trace, info, _ = st.dyson_batch(c, want_w=True, precision=prec)
        assert not np.any(info)
        assert float((logdet - want).abs().max()) < 1e-10 * n
        assert float((trace - chi0.diagonal(dim1=-2, dim2=-1).sum(-1)).abs().max()) < 1e-9 * n
        assert float((c - ref).abs().max()) < tol, prec


def test_contour_deformation_device_matches_reference_golden(golden):
    """The contour-deformation self-energy on the device against the
    reference (GW/contour_deformation.py, GW/real_screening.py): proj(tau) on
    the contour's time grid, the three-index slices of three states, their
    screening contraction over 64 frequencies (one Dyson step per frequency
    for all states), and Sigma^c at five points around each state's level with
    the residues' W from the cosh transform of proj(tau); FP64 throughout."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    X, D, eps, nocc, mu = g['X'], g['D'], g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = contour.cd_frequency_grid(eps, nocc)
    proj = contour.polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    assert rel(proj.cpu().numpy(), g['proj']) < FP64_REL
    B = contour.three_index_slices(X, D, g['states'])
    assert rel(B.cpu().numpy(), g['B']) < FP64_REL
    wcs = contour.cd_screening_contraction_multi(proj, grid.cosft_wt, list(B))
    assert rel(torch.stack(wcs).cpu().numpy(), g['wc']) < 1e-10
    wc_np = contour.cd_screening_contraction_multi(g['proj'], grid.cosft_wt, list(g['B']))
    assert isinstance(wc_np[0], np.ndarray) and rel(np.stack(wc_np), g['wc']) < 1e-10
    # the contraction's products as split-BF16 tensor-core products (FP32
    # out, 2^-16-level relative error per product term): wc to 1e-4 of its
    # scale, Sigma^c to 1e-5 Ha
    wc_mx = contour.cd_screening_contraction_multi(proj, grid.cosft_wt, list(B),
                                                   precision='mixed')
    assert rel(torch.stack(wc_mx).cpu().numpy(), g['wc']) < 1e-4
    lap_mx = contour.LaplaceRealScreening(proj, grid, eps, nocc)
    for i, p in enumerate(g['states']):
        s = contour.sigma_cd(int(p), eps[p], B[i], eps, nocc, nu, nu_w, wc=wc_mx[i],
                             real_screening=lap_mx)
        assert abs(s - g['sigma'][i, 2]) < 1e-5, p
    lap = contour.LaplaceRealScreening(proj, grid, eps, nocc)
    for i, p in enumerate(g['states']):
        for j, dw in enumerate(g['shifts']):
            s = contour.sigma_cd(int(p), eps[p] + dw, B[i], eps, nocc, nu, nu_w, wc=wcs[i],
                                 real_screening=lap)
            assert abs(s - g['sigma'][i, j]) <= 1e-9 * abs(g['sigma'][i, j]), (p, dw)
    # a residue frequency at the gap is refused, as the reference refuses it
    gap = eps[nocc] - eps[nocc - 1]
    with pytest.raises(contour.ResidueRefused):
        lap.apply(gap, B[0][:, 0])
    # the quasiparticle roots and Z of the three states (`qp_energy_cd`: the
    # scan with Newton on the closed-form slope, the device's Sigma^c)
    for i, p in enumerate(g['states']):
        w, z, res = contour.qp_energy_cd(int(p), B[i], eps, nocc, nu, nu_w, wc=wcs[i],
                                         real_screening=lap)
        assert abs(w - g['roots'][i, 0]) < 1e-9 and abs(z - g['roots'][i, 1]) < 1e-8, p
        assert res == contour.residue_set(eps, nocc, w)
    # the drop-in driver on the same factors (default contour grid): eV roots
    ev, zs, info = contour.solve_qp_energy_contour(eps, None, nocc, g['states'],
                                                   continuation='laplace', factors=(X, D))
    assert np.abs(ev / contour.HARTREE_TO_EV - g['roots'][:, 0]).max() < 1e-9
    assert np.abs(zs - g['roots'][:, 1]).max() < 1e-8
    assert info['continuation'] == 'laplace' and len(info['states']) == 3
    # the pole model through the same driver: the reference driver's 'sop' roots
    ev, zs, info = contour.solve_qp_energy_contour(eps, None, nocc, g['states'],
                                                   continuation='sop', factors=(X, D))
    assert np.abs(ev / contour.HARTREE_TO_EV - golden('sop')['driver_roots']).max() < 1e-8
    assert info['continuation'] == 'sop'


def test_contour_explicit_backend_matches_reference_golden(golden):
    """Continuation 'cd' against the reference: C_ov from the occupied
    states' slices, the explicit response (mbpt_chi0_aux) against its NumPy
    composition, W(freq) b and its slope below and above the particle-hole
    gap with and without broadening (the Dyson step's LU above the gap), the
    explicit imaginary-axis contraction, Sigma^c with explicit residues, the
    roots and Z of five states from the deepest to the highest (one with the
    explicit contraction too), and the drop-in driver's default
    continuation."""
    from mbptcode_b200 import contour, gw, space_time
    g = golden('contour_explicit')
    eps, nocc, X, D = g['eps'], int(g['nocc']), g['X'], g['D']
    nu, nu_w = g['nu'], g['nu_w']
    C = contour.three_index_ov(X, D, eps, nocc)
    assert np.abs(C.cpu().numpy() - g['C_ov']).max() <= 1e-12 * np.abs(g['C_ov']).max()
    d = contour.ov_energies(eps, nocc)
    # the response alone, one block and two accumulated blocks (host in, host out)
    f = space_time.frequency_factor(d, float(g['freqs'][2]), False)
    ref = 2.0 * (g['C_ov'] * f) @ g['C_ov'].T
    chi = space_time.chi0_aux([(g['C_ov'], f)], 2.0)
    assert np.abs(chi - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.array_equal(chi, chi.T)
    chi2 = space_time.chi0_aux([(g['C_ov'][:, :20], f[:20]), (g['C_ov'][:, 20:], f[20:])], 2.0)
    assert np.abs(chi2 - ref).max() <= 1e-13 * np.abs(ref).max()
    # mixed: one split BF16x3 tensor-core product (FP32 accumulation)
    chim = space_time.chi0_aux([(g['C_ov'], f)], 2.0, precision='mixed')
    err_m = np.abs(chim - ref).max() / np.abs(ref).max()
    assert err_m <= 5e-5, err_m
    for a, eta in enumerate(g['etas']):
        ers = contour.ExplicitRealScreening(C, eps, nocc, eta=float(eta))
        for j, fr in enumerate(g['freqs']):
            y = ers.apply(float(fr), g['b'])
            want = g['apply'][a, j]
            assert np.abs(y - want).max() <= 1e-10 * np.abs(want).max(), (eta, fr)
            s = ers.slope(float(fr), y)
            assert abs(s - g['slope'][a, j]) <= 1e-9 * abs(g['slope'][a, j]), (eta, fr)
    B = contour.three_index_slices(X, D, g['states'])
    for r, i in enumerate(g['near']):
        wcx = contour.wc_explicit(B[i], C, d, nu)
        assert np.abs(wcx - g['wc_explicit'][r]).max() <= 1e-10 * np.abs(wcx).max()
        p = int(g['states'][i])
        for j, dw in enumerate(g['shifts']):
            s = contour.sigma_cd(p, eps[p] + dw, B[i], eps, nocc, nu, nu_w, wc=g['wc'][i],
                                 C_ov=C)
            assert abs(s - g['sigma'][r, j]) <= 1e-9 * abs(g['sigma'][r, j]), (p, dw)
    for i, p in enumerate(g['states']):
        w, z, res = contour.qp_energy_cd(int(p), B[i], eps, nocc, nu, nu_w, wc=g['wc'][i],
                                         C_ov=C)
        assert abs(w - g['roots'][i, 0]) < 1e-9 and abs(z - g['roots'][i, 1]) < 1e-8, p
        assert res == contour.residue_set(eps, nocc, w)
    w, z, _ = contour.qp_energy_cd(int(g['states'][2]), B[2], eps, nocc, nu, nu_w, C_ov=C)
    assert abs(w - g['root_explicit_wc'][0]) < 1e-9 and abs(z - g['root_explicit_wc'][1]) < 1e-8
    # the drop-in driver: 'cd' is its default, as in the reference
    ev, zs, info = contour.solve_qp_energy_contour(eps, None, nocc, g['states'], factors=(X, D))
    assert np.abs(ev / contour.HARTREE_TO_EV - g['roots'][:, 0]).max() < 1e-9
    assert np.abs(zs - g['roots'][:, 1]).max() < 1e-8
    assert info['continuation'] == 'cd' and info['residue_route_taken'] == 'explicit'
    # the mixed route: the screening contraction and the explicit response as
    # split products, the Dyson steps FP64 -- within 1e-5 Ha (0.27 meV) of the
    # reference's roots
    r_m, z_m, _ = contour.contour_roots(X, D, eps, nocc, g['states'], continuation='cd',
                                        precision='mixed')
    dr = np.abs(r_m - g['roots'][:, 0]).max()
    assert dr < 1e-5 and np.abs(z_m - g['roots'][:, 1]).max() < 1e-4, (dr, z_m)
    # and through calc_qp_energy(mode='space-time', continuation='cd')
    from types import SimpleNamespace
    occ = np.zeros(len(eps))
    occ[:nocc] = 2.0
    e, z = gw.calc_qp_energy(SimpleNamespace(mo_energy=eps, mo_occ=occ), mode='space-time',
                             continuation='cd', state=[int(p) for p in g['states']],
                             factors=(X, D), return_z=True)
    assert np.abs(np.asarray(z) - g['roots'][:, 1]).max() < 1e-8
    assert np.abs(np.asarray(e) / contour.HARTREE_TO_EV - g['roots'][:, 0]).max() < 1e-9


def test_contour_unrestricted_matches_reference_golden(golden):
    """The contour of an unrestricted reference on the device: each channel's
    roots and Z with the Laplace residues (both spins' pair energies) and the
    explicit ones (both spins' C_ov at 1/sqrt(2)) against the reference's
    composition, directly and through the drop-in driver and calc_qp_energy
    with an unrestricted mean field (X_ao = [X_alpha | X_beta], mo_coeff
    selecting each half)."""
    from types import SimpleNamespace
    from mbptcode_b200 import contour, gw
    g = golden('contour_unrestricted')
    X_mos, D = [g['X_a'], g['X_b']], g['D']
    spectra, noccs = [g['eps_a'], g['eps_b']], [int(g['nocc_a']), int(g['nocc_b'])]
    for s in (0, 1):
        for cont in ('laplace', 'cd'):
            r, z, info = contour.contour_roots_unrestricted(X_mos, D, spectra, noccs, s,
                                                            g[f'states_{s}'], continuation=cont)
            want = g[f'roots_{cont}_{s}']
            assert np.abs(r - want[:, 0]).max() < 1e-9 and np.abs(z - want[:, 1]).max() < 1e-8, \
                (s, cont, r - want[:, 0])
            assert info['continuation'] == cont
    norb = len(spectra[0])
    X_ao = np.hstack(X_mos)
    mo = np.zeros((2, 2 * norb, norb))
    mo[0, :norb] = np.eye(norb)
    mo[1, norb:] = np.eye(norb)
    occ = np.zeros((2, norb))
    occ[0, :noccs[0]] = 1.0
    occ[1, :noccs[1]] = 1.0
    mf = SimpleNamespace(mo_energy=np.stack(spectra), mo_occ=occ, mo_coeff=mo)
    ev, zs, info = contour.solve_qp_energy_contour(mf, None, tuple(noccs), g['states_1'],
                                                   spin_channel='beta',
                                                   factors=(X_mos[0], D, X_ao))
    assert np.abs(ev / contour.HARTREE_TO_EV - g['roots_cd_1'][:, 0]).max() < 1e-9
    assert info['residue_route_taken'] == 'explicit'
    e, z = gw.calc_qp_energy(mf, mode='space-time', continuation='laplace', spin_channel='alpha',
                             state=[int(p) for p in g['states_0']], factors=(X_mos[0], D, X_ao),
                             return_z=True)
    assert np.abs(np.asarray(e) / contour.HARTREE_TO_EV - g['roots_laplace_0'][:, 0]).max() < 1e-9
    assert np.abs(np.asarray(z) - g['roots_laplace_0'][:, 1]).max() < 1e-8


def test_ao_self_energy_and_mirrors_match_reference_golden(golden):
    """self_energy_matrix_imaginary_time (full AO matrix, an AO collocation
    that is not the MO one; all time points and a subset), its MO diagonal,
    screened_interaction_tau from proj(tau) and polarizability_backward,
    under the reference's names and signatures, against the reference."""
    g = golden('sigma_ao')
    X, X_ao, D, eps, nocc, mo = g['X'], g['X_ao'], g['D'], g['eps'], int(g['nocc']), g['mo']
    mu = float(g['mu'])
    args = (X_ao, D, g['W'], mo, eps, nocc, g['tau_sigma'], g['omega'], g['pade'])
    sig = gw.self_energy_matrix_imaginary_time(*args, mu=mu)
    assert isinstance(sig, np.ndarray) and sig.dtype == complex
    assert rel(sig, g['sigma']) < 1e-10
    sub = gw.self_energy_matrix_imaginary_time(*args, mu=mu, tau_indices=[1, 4, 7])
    assert rel(sub, g['sigma_sub']) < 1e-10
    diag = gw.sigma_ao_to_mo_diagonal(sig, mo, states=g['states'])
    assert rel(diag, g['diag']) < 1e-10
    # the same matrix with the products on the int8 emulation (FP64 level)
    # and on the engine's split BF16 products (mixed: ~1e-5 relative)
    for precision, tol in (('fp64_int8', 1e-10), ('mixed', 5e-5)):
        s_p = gw.self_energy_matrix_imaginary_time(*args, mu=mu, precision=precision)
        assert rel(s_p, g['sigma']) < tol, precision
    axes_grid = grids.TimeFrequencyGrid.minimax_split(
        int(g['ntau']), *grids.particle_hole_window(eps, nocc)[:2], g['omega'],
        grids.screening_frequency_grid(int(g['ntau']), eps, nocc, mu=mu)[1],
        with_sine=False, with_inverse=False)
    proj = orc.polarizability_projected_sweep(X, D, eps, nocc, axes_grid.tau_points, mu)
    rW, _ = grids.sigma_fit_ranges(eps, nocc, mu=mu)
    Ctw = grids.minimax_transform_weights(grids.COSINE_WT, g['tau_sigma'], g['omega'], *rW,
                                          warn=False)[0]
    Wt = gw.screened_interaction_tau(proj, axes_grid, Ctw)
    assert rel(Wt, orc.screened_interaction_tau(proj, axes_grid, Ctw)) < 1e-11
    from mbptcode_b200 import adjoint
    out = adjoint.polarizability_backward(g['proj_bar'], X, D, eps, nocc, axes_grid, mu=mu)
    for a, k in zip(out, ('eps_bar', 'X_bar', 'D_bar')):
        assert rel(a, g[k]) < 1e-10, k


def test_per_state_qp_solve_matches_reference_golden(golden):
    """solve_qp_from_imaginary_axis under the reference's signature (sample
    points mu -/+ i omega, the lower branch conjugated), one state at a time
    on the device, against the reference's roots and Z of every state."""
    g = golden('route_calibrated')
    eps, nocc = g['eps'], int(g['nocc'])
    mu = float(grids.particle_hole_window(eps, nocc)[2])
    for p in range(len(eps)):
        z_fit, _ = gw.imaginary_axis_sample_points(g["pade"], nocc, p, mu)
        s_p = np.conj(g['sigma'][p]) if p < nocc else g['sigma'][p]
        root, z = gw.solve_qp_from_imaginary_axis(eps, p, 0.0, z_fit, s_p, with_z=True)
        if np.isfinite(g['roots'][p]):
            tol = 5e-8 if abs(p - nocc) <= 4 else 2e-6
            assert abs(root - g['roots'][p]) < tol, p
    with pytest.raises(NotImplementedError):
        gw.solve_qp_from_imaginary_axis(eps, 0, 0.0, z_fit, s_p, max_order=8)


def test_calc_qp_energy_dispatch(golden):
    """calc_qp_energy, mode='space-time', on pre-built factors: 'homo' and a
    list of states by the Pade route against the reference's roots (eV), the
    contour ('laplace') with Z against the reference's qp_energy_cd, and the
    reference's refusals."""
    from types import SimpleNamespace
    g = golden('route_calibrated')
    X, D, eps, nocc = g['X'], g['D'], g['eps'], int(g['nocc'])
    occ = np.zeros(len(eps))
    occ[:nocc] = 2.0
    mf = SimpleNamespace(mo_energy=eps, mo_occ=occ)

    class Quad:
        ntau_st, npade, w0_gl = int(g['ntau']), 16, 1.0

    class Num:
        quadrature = Quad
    ev = gw.HARTREE_TO_EV
    homo = gw.calc_qp_energy(mf, mode='space-time', factors=(X, D), numerics=Num)
    assert abs(homo / ev - g['roots'][nocc - 1]) < 5e-8
    both = gw.calc_qp_energy(mf, mode='space-time', state=[nocc - 1, nocc], factors=(X, D),
                             numerics=Num)
    assert np.abs(np.array(both) / ev - g['roots'][nocc - 1:nocc + 1]).max() < 5e-8
    c = golden('contour')
    occ_c = np.zeros(len(c['eps']))
    occ_c[:int(c['nocc'])] = 2.0
    mf_c = SimpleNamespace(mo_energy=c['eps'], mo_occ=occ_c)
    e, z = gw.calc_qp_energy(mf_c, mode='space-time', continuation='laplace',
                             state=[int(p) for p in c['states']], factors=(c['X'], c['D']),
                             return_z=True)
    assert np.abs(np.array(e) / ev - c['roots'][:, 0]).max() < 1e-9
    assert np.abs(np.array(z) - c['roots'][:, 1]).max() < 1e-8
    from mbptcode_b200 import evgw
    e_ev = gw.calc_qp_energy(mf, mode='space-time', self_consistency='evGW',
                             state=[nocc - 1, nocc], factors=(X, D))
    e_direct, _ = evgw.evgw_device(X, D, eps, nocc)
    assert np.abs(np.array(e_ev) / ev - e_direct[nocc - 1:nocc + 1]).max() < 1e-12
    with pytest.raises(NotImplementedError):
        gw.calc_qp_energy(mf, mode='casida', factors=(X, D))
    with pytest.raises(ValueError):
        gw.calc_qp_energy(mf, mode='space-time', selfenergy='GWGammaInf', factors=(X, D))
    with pytest.raises(ValueError):
        gw.calc_qp_energy(mf, mode='space-time', eta=0.01, factors=(X, D))
    with pytest.raises(ValueError):
        gw.calc_qp_energy(mf, mode='space-time', return_z=True, factors=(X, D), numerics=Num)


def test_contour_qp_gradient_matches_reference_golden(golden):
    """The gradient of a contour-deformation QP energy in (eps, X, D) on the
    device (Laplace residues) against the reference's qp_gradient_space_time
    for three states around the gap: FP64 to 1e-9 of each adjoint's scale."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = contour.cd_frequency_grid(eps, nocc)
    for i, p in enumerate(g['states']):
        w, z, eb, xb, db = contour.qp_gradient_space_time(g['X'], g['D'], eps, nocc, grid, nu,
                                                          nu_w, int(p), mu=mu)
        assert abs(w - g['grad_roots'][i, 0]) < 1e-9 and abs(z - g['grad_roots'][i, 1]) < 1e-8
        for a, k in ((eb, 'eps_bar'), (xb, 'X_bar'), (db, 'D_bar')):
            ref = g[k][i]
            assert np.abs(a - ref).max() <= 1e-8 * np.abs(ref).max(), (int(p), k)
    # a walk's next geometry (here the same one): the root frozen as w0 and its
    # branch followed from 1e-3 away; the quasiparticle branch continues, so
    # the root, Z and gradient are the unfollowed ones
    i, p = 1, int(g['states'][1])
    root, zr = float(g['grad_roots'][i, 0]), float(g['grad_roots'][i, 1])
    rec = {}
    w, z, eb, xb, db = contour.qp_gradient_space_time(
        g['X'], g['D'], eps, nocc, grid, nu, nu_w, p, mu=mu, w0={p: root},
        follow={p: (root + 1e-3, None)}, z0={p: zr}, route_out=rec)
    assert abs(w - root) < 1e-9 and abs(z - zr) < 1e-8
    assert rec['branches'][p]['followed'] and not rec['branches'][p]['flipped']
    assert rec['roots'][p] == w and rec['weights'][p] == z
    assert np.abs(db - g['D_bar'][i]).max() <= 1e-8 * np.abs(g['D_bar'][i]).max()


@pytest.mark.parametrize('prec', ['fp64', 'mixed'])
def test_dyson_batched_groups_with_failed_frequency(prec):
    """17 frequencies: the batched Cholesky in four stream groups (4-5
    frequencies each), frequency 11 (third group) not positive definite.
    It alone is flagged and takes the LU fallback; every other output matches
    the dense FP64 answer."""
    rng = np.random.default_rng(11)
    n, nfreq = 200, 17
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    mats = []
    for f in range(nfreq):
        lam = -rng.uniform(0.05, 3.0, n)
        if f == 11:
            lam[3] = 1.7
        mats.append((Q * lam) @ Q.T)
    chi0 = torch.as_tensor(np.stack(mats), device='cuda')
    logdet, trace, info, sign = st.dyson_batch(chi0, want_w=True, precision=prec)
    assert [int(f) for f in np.nonzero(info)[0]] == [11]
    assert sign[11] == -1 and np.all(np.delete(sign, 11) == 1)
    tol = 1e-10 if prec == 'fp64' else 5e-6
    for f, c in enumerate(mats):
        one_minus = np.eye(n) - c
        assert abs(float(logdet[f]) - np.linalg.slogdet(one_minus)[1]) < 1e-9 * n
        W_ref = np.linalg.inv(one_minus) - np.eye(n)
        err = np.abs(chi0[f].cpu().numpy() - W_ref).max()
        assert err < (1e-10 if f == 11 else tol) * max(1.0, np.abs(W_ref).max()), (f, err)


def test_ao_self_energy_mixed_on_partial_tiles():
    """The mixed AO self-energy (U = D W, the G o Zt tile pass, X_ao^T H X_ao
    on the engine) against the FP64 one where no size is a multiple of 128:
    M = 1100, nao = 300, naux = 900, 40 of 260 orbitals occupied, 6 time
    points; both branches within 5e-5 of their scale."""
    from mbptcode_b200._lib import MODES, WORKSPACE, check, lib, ptr, stream_ptr
    from mbptcode_b200.space_time import _Err
    rng = np.random.default_rng(3)
    M, nao, norb, nocc, naux, nt = 1100, 300, 260, 40, 900, 6
    Xa = torch.as_tensor(rng.standard_normal((M, nao)) * 0.05, device='cuda')
    C = torch.as_tensor(np.linalg.qr(rng.standard_normal((nao, norb)))[0], device='cuda')
    Dd = torch.as_tensor(rng.standard_normal((M, naux)) * 0.05, device='cuda')
    A = rng.standard_normal((nt, naux, naux)) * 0.02
    Wt = torch.as_tensor(A + A.transpose(0, 2, 1), device='cuda')
    e = torch.as_tensor(np.sort(np.concatenate([rng.uniform(-1, -0.3, nocc),
                                                rng.uniform(0.1, 2, norb - nocc)])),
                        device='cuda')
    tau = np.linspace(0.2, 3.0, nt)
    out = {}
    for p in ('fp64', 'mixed'):
        m = MODES[p]
        br = torch.empty((2, nt, nao, nao), dtype=torch.float64, device='cuda')
        ws = WORKSPACE.get(lib().mbpt_sigma_ao_workspace_bytes(M, nao, norb, nocc, naux, m),
                           'cuda')
        err = _Err('cuda')
        check(lib().mbpt_sigma_ao(ptr(Xa), M, nao, ptr(C), norb, nocc, ptr(e), -0.1, ptr(Dd),
                                  naux, ptr(Wt), tau.ctypes.data, nt, m, ptr(br), ptr(ws),
                                  ws.numel(), ptr(err.t), stream_ptr()), 'mbpt_sigma_ao')
        err.check('mbpt_sigma_ao')
        out[p] = br.cpu().numpy()
    for b in range(2):
        assert rel(out['mixed'][b], out['fp64'][b]) < 5e-5, b


def test_contour_root_following_matches_reference_golden(golden):
    """`qp_energy_cd` with a followed root (`follow`, `branch`, `rescan`) on
    the contour system, residues by the cosh transform of proj(tau): root,
    Z and branch record against the reference's (`contour_follow.npz`)."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    cf = golden('contour_follow')
    col = {c: i for i, c in enumerate(cf['columns'])}
    X, D, eps, nocc, mu = g['X'], g['D'], g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = contour.cd_frequency_grid(eps, nocc)
    proj = contour.polarizability_tau(X, D, eps, nocc, grid, mu=mu)
    B = contour.three_index_slices(X, D, g['states'])
    wcs = contour.cd_screening_contraction_multi(proj, grid.cosft_wt, list(B))
    for row in cf['cases']:
        i = int(row[col['state']])
        p = int(g['states'][i])
        out = {}
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            w, z, res = contour.qp_energy_cd(
                p, B[i], eps, nocc, nu, nu_w, wc=wcs[i],
                real_screening=contour.LaplaceRealScreening(proj, grid, eps, nocc),
                follow=float(row[col['follow']]), branch=out, rescan=bool(row[col['rescan']]))
        assert abs(w - row[col['w']]) < 1e-9 and abs(z - row[col['z']]) < 1e-8, (p, row)
        assert {None: -1.0, False: 0.0, True: 1.0}[out['followed']] == row[col['followed']]
        assert float(out['flipped']) == row[col['flipped']]
        assert len(res) == int(row[col['residues']])
        assert abs(out['largest'][0] - row[col['largest_w']]) < 1e-9


def test_contour_pole_model_route_matches_reference_golden(golden):
    """continuation='sop' from the factors on the device (proj(tau), the
    slices, W on the contour's frequencies and the screening contraction),
    each state's pole model fitted to its wc and solved in closed form,
    against the reference driver's roots and Z (`sop.npz`); a state the
    compression test excludes (orbital 9, reach 1.45 gaps) is refused by
    name before anything is built."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    s = golden('sop')
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        roots, zs, info = contour.contour_roots(g['X'], g['D'], eps, nocc, g['states'],
                                                mu=mu, continuation='sop')
    assert np.abs(roots - s['driver_roots']).max() < 1e-8
    assert np.abs(zs - s['driver_z']).max() < 1e-7
    assert info['residue_route_taken'] == 'sop'
    assert [r['sop_admits'] for r in info['states']] == list(s['admits'])
    with pytest.raises(ValueError, match="continuation='sop' cannot serve orbital 9"):
        contour.contour_roots(g['X'], g['D'], eps, nocc, [9], mu=mu, continuation='sop')


def test_contour_pole_model_gradient_matches_reference_golden(golden):
    """The QP energy and its gradient in (eps, X, D) on the pole model's route
    (residue_route 'sop': poles fitted to wc, then held; the adjoint on wc
    through the integral term's chain, no residues) against the reference's
    qp_gradient_space_time for the three states (`sop.npz`), 1e-8 of each
    adjoint's scale; the same with the fitted poles handed back frozen."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    s = golden('sop')
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = contour.cd_frequency_grid(eps, nocc)
    for i, p in enumerate(g['states']):
        rec = {}
        w, z, eb, xb, db = contour.qp_gradient_space_time(
            g['X'], g['D'], eps, nocc, grid, nu, nu_w, int(p), residue_route='sop', mu=mu,
            route_out=rec)
        assert abs(w - s['grad_roots'][i, 0]) < 1e-9 and abs(z - s['grad_roots'][i, 1]) < 1e-8
        for a, k in ((eb, 'grad_eps_bar'), (xb, 'grad_X_bar'), (db, 'grad_D_bar')):
            ref = s[k][i]
            assert np.abs(a - ref).max() <= 1e-8 * np.abs(ref).max(), (int(p), k)
        assert rec['residue_route'] == 'sop' and rec['residues'] == []
        w2, z2, _, _, db2 = contour.qp_gradient_space_time(
            g['X'], g['D'], eps, nocc, grid, nu, nu_w, int(p), residue_route='sop', mu=mu,
            sop_poles={int(p): rec['sop_poles'][int(p)]})
        assert w2 == w and z2 == z and np.abs(db2 - db).max() <= 1e-12 * np.abs(db).max()


def test_contour_explicit_route_gradient_matches_reference_golden(golden):
    """The QP gradient on the explicit residue route (the residues' W from
    C_ov; their rank-one adjoint taken back to (eps, X, D) without forming
    C_ov's adjoint) for orbitals 1-4, orbital 1 with two residues, against
    the reference's qp_gradient_space_time (`contour_grad_explicit.npz`):
    roots 1e-9, Z 1e-8, adjoints 1e-8 of their scale."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    e = golden('contour_grad_explicit')
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = contour.cd_frequency_grid(eps, nocc)
    for i, p in enumerate(e['states']):
        rec = {}
        w, z, eb, xb, db = contour.qp_gradient_space_time(
            g['X'], g['D'], eps, nocc, grid, nu, nu_w, int(p), residue_route='explicit', mu=mu,
            route_out=rec)
        assert len(rec['residues']) == int(e['residues'][i])
        assert abs(w - e['roots'][i, 0]) < 1e-9 and abs(z - e['roots'][i, 1]) < 1e-8, int(p)
        for a, k in ((eb, 'eps_bar'), (xb, 'X_bar'), (db, 'D_bar')):
            ref = e[k][i]
            assert np.abs(a - ref).max() <= 1e-8 * np.abs(ref).max(), (int(p), k)


def test_contour_pole_route_decisions_match_reference_golden(golden):
    """residue_route 'sop' decides per state as the reference does: orbital 9
    (reach 1.45 gaps) falls back to the explicit residues, a frozen scissor
    mapping or a scalar shift where the compression test fails takes the
    shifted root (Z = 1, no adjoint on the factors), orbital 2 keeps the pole
    model; roots, eps_bar and D_bar against the reference's."""
    import warnings
    from mbptcode_b200 import contour
    g = golden('contour')
    e = golden('contour_grad_explicit')
    eps, nocc, mu = g['eps'], int(g['nocc']), float(g['mu'])
    with warnings.catch_warnings():
        warnings.simplefilter('ignore')
        nu, nu_w, grid, _ = contour.cd_frequency_grid(eps, nocc)
    for j, (p, sc) in enumerate([(9, None), (9, {9: 0.05}), (9, 0.07), (2, 0.07)]):
        rec = {}
        w, z, eb, _, db = contour.qp_gradient_space_time(
            g['X'], g['D'], eps, nocc, grid, nu, nu_w, p, residue_route='sop', mu=mu,
            scissor=sc, route_out=rec)
        assert rec['residue_route'] == str(e[f'route{j}_name']), (p, sc)
        root = e[f'route{j}_root']
        assert abs(w - root[0]) < 1e-9 and abs(z - root[1]) < 1e-8, (p, sc)
        for a, k in ((eb, f'route{j}_eps_bar'), (db, f'route{j}_D_bar')):
            ref = e[k]
            assert np.abs(a - ref).max() <= 1e-8 * max(np.abs(ref).max(), 1e-300), (p, sc, k)


@pytest.mark.parametrize('M,n,nocc,naux,nstates', [(301, 37, 5, 173, 4), (1100, 90, 12, 900, 4),
                                                   (700, 400, 40, 500, 300)])
def test_engine_cta_pairs_match_single_cta(M, n, nocc, naux, nstates, monkeypatch):
    """The engine's 256-wide BF16 products as CTA pairs (cta_group::2, the
    default: Z = D^T Pi, proj, U = D W, Zt = U D^T, the G products of Sigma's
    H and the row contraction) against the same products one CTA per tile
    (MBPT_ENGINE_PAIRS=0), on row-tile counts odd and even (a pair's second
    tile past the last row stores nothing) and state counts whose last
    256-wide column tile overhangs: the same K order per element, so within
    1e-6 of each other, and both within the mixed tolerance of the oracle."""
    rng = np.random.default_rng(11)
    X = rng.standard_normal((M, n)) * 0.08
    D = rng.standard_normal((M, naux)) * 0.08
    eps = np.sort(np.concatenate([rng.uniform(-1.2, -0.4, nocc),
                                  rng.uniform(0.1, 3.0, n - nocc)]))
    axes = grids.space_time_axes(eps, nocc, ntau=8)
    ref = orc.chi0_imaginary_frequency(X, D, eps, nocc, axes.grid)
    W = np.stack([orc.dyson_screening(c, True) for c in ref])
    Wt = torch.as_tensor(np.tensordot(axes.Ctw, W, axes=(1, 0)), device='cuda')
    # 4 states: one overhanging 256-wide column tile; 300: two, the last overhanging
    states = [0, nocc - 1, nocc, n - 1] if nstates == 4 else list(range(nstates))
    out = {}
    for pairs in ('1', '0'):
        monkeypatch.setenv('MBPT_ENGINE_PAIRS', pairs)
        chi = st.chi0_imaginary_frequency(X, D, eps, nocc, axes.grid, precision='mixed')
        br = gw.sigma_branch_sums(X, D, Wt, eps, nocc, axes.tau_sigma, states, axes.mu,
                                  precision='mixed').cpu().numpy()
        out[pairs] = (chi, br)
    assert rel(out['1'][0], out['0'][0]) < 1e-6
    assert rel(out['1'][1], out['0'][1]) < 1e-6
    assert rel(out['1'][0], ref) < MIXED_REL
    br_ref = orc.sigma_branch_sums(X, D, Wt.cpu().numpy(), eps, nocc, axes.tau_sigma, axes.mu,
                                   states)
    assert rel(out['1'][1], br_ref) < 5e-5
