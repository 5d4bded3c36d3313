"""Measurement cases beside the benchmark: small, self-contained invocations
of the route for ncu captures, device timings of the rows beside the sweep,
and the two full-scale experiments (the adjoint against central differences,
the learned warm start). Nothing here is imported by the package.

    python bench_cases.py tau [--M 4096] [--n 682] [--nocc 68] [--states 682]
    python bench_cases.py dyson N [--nfreq 1] [--time]
    python bench_cases.py sweep [--M 7200] [--n 1200] [--nocc 120]
    python bench_cases.py transform N
    python bench_cases.py qp-mlp
    python bench_cases.py rows
    python bench_cases.py ao-sigma
    python bench_cases.py rows-cd
    python bench_cases.py chi0-aux NAUX NOV [--mixed]
    python bench_cases.py fp64-peak N
    python bench_cases.py adjoint-fd [--n 1200] [--nocc 120] [--M 7200] [--directions 32]
    python bench_cases.py adjoint-time [--n 1200] [--nocc 120] [--M 7200]
    python bench_cases.py ozaki-gemm N
    python bench_cases.py warm-start [--train 512] [--eval 64] [--save model.npz]

tau: one tau point of the chi0 sweep and one of the self-energy sweep, mixed
precision. Launches, in order: the branch preparation, the TF32x3
G_occ/G_virt/Pi kernel, Z = D^T Pi, proj = -2 D^T Z^T, the FP64 transform,
then on the self-energy side U = D W, the G_occ/G_virt/Zt kernel with the H
epilogue and the row-contraction kernel -- one launch of each engine kernel.
Device memory stays at a few GB (M = 4096: about 1 GB).

dyson N [--time]: the mixed Dyson step of `nfreq` frequencies of an N x N
chi0 (negative definite, seeded). From 4 frequencies on, the factorisations
are one batched Cholesky of all of them. --time prints CUDA-event times of
the factorisations alone and of the whole step.

sweep: one whole mixed chi0 -> W -> Sigma -> QP sweep (24 points) of a
synthetic system, for the launch list of the benchmark's workload.

transform N: one FP64 tau <-> omega transform of 24 N x N matrices with a
24 x 24 weight matrix (mbpt_transform, the W(i w) -> W(tau) step).

qp-mlp: the latency-bound kernels of the QP solve and the learned warm
start on a C1-sized system (n_orb = 400, N_mu = 2400, 20 points, mixed): one
sweep, the plain and the warm-started Pade + QP kernels and the Pade
evaluation of the features, then 5 training steps of the 4 -> 64 -> 64 -> 1
network on 65536 samples (forward, backward, AdamW).

rows: device times at n_orb = 1200, N_mu = 7200 of the rows built beside the
sweep. rows-cd: the contour's explicit particle-hole backend (continuation
'cd') at the same size.

chi0-aux NAUX NOV [--mixed]: the explicit response alone on a seeded factor,
three calls (the capture case of its engine launch).

fp64-peak N: the FP64 reference rates of this GPU, timed with CUDA events
(best of 5 after a warm-up): cuBLAS DGEMM at N^3 and cuSOLVER's Cholesky of
an N x N SPD matrix.

adjoint-fd: E_c and dE_c/d(eps, X, D) in FP64 on the device, then central
differences (E_c(+h d) - E_c(-h d)) / 2h along seeded unit directions d,
the grid and mu frozen as the adjoint assumes, and the Richardson
combination (4 D(h_r / 2) - D(h_r)) / 3 at h_r = 1e-2 beside it.

warm-start: the learned quasiparticle warm start at the scale it is meant
for: training samples from `--train` method-generated systems, the network
trained on the GPU, then G0W0 and evGW on `--eval` further systems, plainly
and warm-started (one JSON report).
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from mbptcode_b200 import grids  # noqa: E402
from mbptcode_b200.gw import gw_sweep, sigma_branch_sums  # noqa: E402
from mbptcode_b200.space_time import chi0_sweep, dyson_batch  # noqa: E402
from mbptcode_b200.synthetic import synthetic_system_torch  # noqa: E402


def tau_point(a):
    X, D, eps_t = synthetic_system_torch(a.n, a.nocc, a.M, seed=3, variant='calibrated')
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, a.nocc, ntau=24)
    k = axes.ntau // 2
    chi0, _ = chi0_sweep(X, D, eps, a.nocc, axes.grid.tau_points[k:k + 1],
                         axes.grid.cosft_wt[:1, k:k + 1], mu=axes.mu, precision='mixed')
    W = chi0.clone()
    W.diagonal(dim1=-2, dim2=-1).mul_(-1.0)
    br = sigma_branch_sums(X, D, W, eps, a.nocc, axes.tau_sigma[k:k + 1],
                           np.arange(a.states), axes.mu, precision='mixed')
    torch.cuda.synchronize()
    print(f'profile case M={a.M} n={a.n}: |chi0| {float(chi0.abs().max()):.3e}, '
          f'|branch| {float(br.abs().max()):.3e}')


def dyson(a):
    n = a.dyson
    g = torch.Generator(device='cuda').manual_seed(1)
    A = torch.randn(n, n // 2, generator=g, device='cuda', dtype=torch.float64)
    chi0 = (-(A @ A.T) / n * 3.0)[None].repeat(a.nfreq, 1, 1).contiguous()
    del A
    if a.time:
        # the factorisations alone (want_w False), then the whole step, each
        # the best of 3 after a warm-up, on copies of the same chi0
        for want_w in (False, True):
            best = 1e9
            for _ in range(4):
                c = chi0.clone()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                dyson_batch(c, want_w=want_w, precision='mixed')
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            print(f'dyson n={n} nfreq={a.nfreq} want_w={want_w}: {best:.2f} ms '
                  f'({best / a.nfreq:.3f} ms per frequency)', flush=True)
        return
    logdet, _, info, _ = dyson_batch(chi0, want_w=True, precision='mixed')
    torch.cuda.synchronize()
    print(f'dyson case n={n} nfreq={a.nfreq}: info {info.tolist()}, '
          f'logdet[0] {float(logdet[0]):.6e}')


def sweep(a):
    X, D, eps_t = synthetic_system_torch(a.n, a.nocc, a.M, seed=2024, variant='literal')
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, a.nocc, ntau=24)
    res = gw_sweep(X, D, eps, a.nocc, axes=axes, precision='mixed')
    torch.cuda.synchronize()
    print(f'sweep case M={a.M} n={a.n}: E_c {float(res["e_c"]):.6e}')


def transform_case(a):
    from mbptcode_b200.space_time import transform
    n, k = a.transform, 24
    g = torch.Generator(device='cuda').manual_seed(2)
    x = torch.randn(k, n, n, generator=g, device='cuda', dtype=torch.float64)
    w = np.random.default_rng(2).standard_normal((k, k))
    out = transform(x, w)
    torch.cuda.synchronize()
    print(f'transform case n={n} K=J={k}: |out| {float(out.abs().max()):.3e}')


def rows(a):
    """Device times (CUDA events, after a warm-up call) of the rows built
    beside the sweep, at n_orb = 1200, N_mu = 7200 (the C2 shapes), one JSON
    line each."""
    import json
    import time
    from mbptcode_b200 import adjoint, contour, gw, space_time
    n, nocc, M = 1200, 120, 7200
    X, D, eps_t = synthetic_system_torch(n, nocc, M, seed=2024, variant='calibrated')
    eps = eps_t.cpu().numpy()
    states20 = np.arange(nocc - 10, nocc + 10)

    def timed(name, fn, reps=1, **extra):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({'row': name, 's': round(e0.elapsed_time(e1) / 1e3 / reps, 4),
                          'host_s': round((time.perf_counter() - t0) / reps, 4), **extra}),
              flush=True)

    sgrid = grids.static_screening_grid(eps, nocc)
    for prec in ('mixed', 'fp64'):
        timed(f'static W(0), {prec}', lambda prec=prec: space_time.static_screening_matrix(
            X, D, eps, nocc, sgrid, precision=prec), ntau=sgrid.ntau)
    axes = grids.space_time_axes(eps, nocc, ntau=24)
    timed('sweep, freq_block=6, mixed', lambda: gw.gw_sweep(
        X, D, eps, nocc, axes=axes, precision='mixed', freq_block=6))
    Xb, _, eps_b = synthetic_system_torch(n, nocc - 1, M, seed=2025, variant='calibrated')
    ua = grids.space_time_axes_unrestricted([eps, eps_b.cpu().numpy()], [nocc, nocc - 1], ntau=24)
    timed('unrestricted sweep (both channels, 1200 states each), mixed',
          lambda: gw.gw_sweep_unrestricted([X, Xb], D, [eps, eps_b.cpu().numpy()],
                                           [nocc, nocc - 1], axes=ua, precision='mixed'))
    del Xb
    tr = grids.sigma_transforms(eps, nocc, axes.grid.tau_points, axes.grid.omega_points,
                                axes.pade_freq, mu=axes.mu)

    def sigma_adjoint():
        sig, cache = adjoint.selfenergy_diag(X, D, eps_t, nocc, axes.grid, states20, tr, axes.mu)
        a = torch.ones(sig.shape, dtype=torch.float64, device=sig.device)
        adjoint.selfenergy_diag_backward(a, a, X, D, eps_t, nocc, axes.grid, states20, tr,
                                         axes.mu, cache)
    timed('self-energy diagonal + adjoint, 20 states, 24 points, FP64', sigma_adjoint)
    nu, nu_w, cgrid, _ = contour.cd_frequency_grid(eps, nocc)
    proj = contour.polarizability_tau(X, D, eps, nocc, cgrid)
    B = contour.three_index_slices(X, D, states20)
    timed('contour: W(i nu) at 64 frequencies + contraction of 20 states, FP64',
          lambda: contour.cd_screening_contraction_multi(proj, cgrid.cosft_wt, list(B)))
    timed('contour: the same in mixed precision (TF32x3 Dyson inverses, split-BF16 contraction)',
          lambda: contour.cd_screening_contraction_multi(proj, cgrid.cosft_wt, list(B),
                                                         precision='mixed'))
    wcs = contour.cd_screening_contraction_multi(proj, cgrid.cosft_wt, list(B))
    lap = contour.LaplaceRealScreening(proj, cgrid, eps, nocc)
    p = nocc - 1
    timed('contour: Sigma^c(eps_HOMO - 0.05) of the HOMO (residues by the cosh transform)',
          lambda: contour.sigma_cd(p, eps[p] - 0.05, B[9], eps, nocc, nu, nu_w, wc=wcs[9],
                                   real_screening=contour.LaplaceRealScreening(
                                       proj, cgrid, eps, nocc)))


def ao_sigma(a):
    """The full AO self-energy (self_energy_matrix_imaginary_time) at
    n_orb = nao = 1200, N_mu = naux = 7200, 24 points, from the mixed sweep's
    W(i omega): FP64, its int8 emulation and mixed, CUDA events after a
    warm-up call; the mixed and emulated results against the FP64 one."""
    import json
    from mbptcode_b200 import gw
    n, nocc, M = 1200, 120, 7200
    X, D, eps_t = synthetic_system_torch(n, nocc, M, seed=2024, variant='calibrated')
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, nocc, ntau=24)
    chi0, _ = chi0_sweep(X, D, eps, nocc, axes.grid.tau_points, axes.grid.cosft_wt,
                         mu=axes.mu, precision='mixed')
    dyson_batch(chi0, want_w=True, precision='mixed')
    chi0.diagonal(dim1=-2, dim2=-1).add_(1.0)          # W
    g = torch.Generator(device='cpu').manual_seed(5)
    mo = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64))[0].cuda()
    X_ao = X @ mo.T                                    # X_ao mo = X
    out = {}
    for prec in ('fp64', 'fp64_int8', 'mixed'):
        def run(prec=prec):
            return gw.self_energy_matrix_imaginary_time(
                X_ao, D, chi0, mo, eps, nocc, axes.grid.tau_points, axes.grid.omega_points,
                axes.pade_freq, mu=axes.mu, precision=prec)
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out[prec] = run()
        e1.record()
        torch.cuda.synchronize()
        ref = out['fp64']
        err = float((out[prec] - ref).abs().max() / ref.abs().max())
        print(json.dumps({'case': 'ao-sigma', 'precision': prec, 'nao': n, 'naux': M,
                          'ntau': 24, 's': round(e0.elapsed_time(e1) / 1e3, 4),
                          'rel_err_vs_fp64': err}), flush=True)


def explicit_rows(a):
    """Device times of the contour's explicit particle-hole backend
    (continuation 'cd') at n_orb = 1200, nocc = 120, N_mu = 7200: C_ov
    (7200 x 129600) from the occupied slices, the explicit response at one
    real frequency (mbpt_chi0_aux: naux (naux + 1) nov useful flops of a
    symmetric rank-k product) and one W(freq) - I below and above the gap
    (the Dyson step: Cholesky below, LU above). One JSON line each."""
    import json
    from mbptcode_b200 import contour, space_time
    n, nocc, M = 1200, 120, 7200
    X, D, eps_t = synthetic_system_torch(n, nocc, M, seed=2024, variant='calibrated')
    eps = eps_t.cpu().numpy()

    def timed(name, fn, flops=None):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        extra = {'tflops': round(flops / t / 1e12, 1)} if flops else {}
        print(json.dumps({'row': name, 's': round(t, 4), **extra}), flush=True)

    C = contour.three_index_ov(X, D, eps, nocc)
    timed('cd: C_ov (7200 x 129600) from the 120 occupied slices',
          lambda: contour.three_index_ov(X, D, eps, nocc))
    d = contour.ov_energies(eps, nocc)
    gap = eps[nocc] - eps[nocc - 1]
    f = space_time.frequency_factor(d, 0.5 * gap, False)
    out = torch.empty((M, M), dtype=torch.float64, device='cuda')
    naux, nov = C.shape
    timed('cd: explicit chi0 at one real frequency (mbpt_chi0_aux, FP64)',
          lambda: space_time.chi0_aux([(C, f)], 2.0, out=out), flops=naux * (naux + 1) * nov)
    ref = out.clone()
    timed('cd: the same as one split BF16x3 product (mixed; TFLOP/s of the FP64-equivalent '
          'useful flops)',
          lambda: space_time.chi0_aux([(C, f)], 2.0, out=out, precision='mixed'),
          flops=naux * (naux + 1) * nov)
    print(json.dumps({'row': 'cd: mixed explicit chi0, max |error| / max |chi0|',
                      'rel': float((out - ref).abs().max() / ref.abs().max())}), flush=True)
    del ref
    for prec in ('fp64', 'mixed'):
        for label, w in (('below the gap (Cholesky)', 0.5 * gap),
                         ('above the gap (LU)', 1.5 * gap)):
            timed(f'cd: W(freq) - I {label}, chi0 + Dyson, {prec}',
                  lambda w=w, prec=prec: contour.ExplicitRealScreening(
                      C, eps, nocc, precision=prec).w_minus_identity(w))
    del C, out
    # whole contour solves of the HOMO and the LUMO (grid, proj(tau), the
    # contraction of 64 frequencies, the scan with its residues), one call each
    import time
    states = [nocc - 1, nocc]
    for cont, prec in (('laplace', 'fp64'), ('cd', 'mixed')):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r, z, info = contour.contour_roots(X, D, eps, nocc, states, continuation=cont,
                                           precision=prec)
        torch.cuda.synchronize()
        print(json.dumps({'row': f'cd: contour_roots of HOMO and LUMO, {cont}, {prec}',
                          'host_s': round(time.perf_counter() - t0, 3),
                          'roots_Ha': [float(x) for x in r], 'z': [float(x) for x in z],
                          'residues': [rec['residues'] for rec in info['states']]}),
              flush=True)


def chi0_aux_case(a):
    """The explicit particle-hole response alone on a seeded (naux x nov)
    factor, three calls in the requested precision (the capture case of the
    mixed response's engine launch): --chi0-aux NAUX NOV [--mixed]."""
    from mbptcode_b200 import space_time
    naux, nov = a.chi0_aux
    g = torch.Generator(device='cuda').manual_seed(7)
    C = torch.randn(naux, nov, generator=g, device='cuda', dtype=torch.float64) / nov ** 0.5
    f = -np.linspace(0.5, 2.0, nov)
    out = torch.empty((naux, naux), dtype=torch.float64, device='cuda')
    prec = 'mixed' if a.mixed else 'fp64'
    for _ in range(3):
        space_time.chi0_aux([(C, f)], 2.0, out=out, precision=prec)
    torch.cuda.synchronize()
    print(f'chi0_aux {prec} naux={naux} nov={nov}: ok', flush=True)


def fp64_peak(a):
    n = a.fp64_peak
    g = torch.Generator(device='cuda').manual_seed(4)
    A = torch.randn(n, n, generator=g, device='cuda', dtype=torch.float64)
    B = torch.randn(n, n, generator=g, device='cuda', dtype=torch.float64)
    S = A @ A.T / n
    S.diagonal().add_(1.0)

    def best(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return min(ts)
    t_gemm = best(lambda: A @ B)
    t_chol = best(lambda: torch.linalg.cholesky(S))
    print(f'fp64 peak case n={n}: DGEMM {2 * n ** 3 / t_gemm / 1e12:.2f} TFLOP/s '
          f'({t_gemm * 1e3:.3f} ms), Cholesky {n ** 3 / 3 / t_chol / 1e12:.2f} TFLOP/s '
          f'({t_chol * 1e3:.3f} ms)')


def qp_mlp_case(a):
    from mbptcode_b200.gw import qp_solve
    from mbptcode_b200.qp_mlp import MODEL_PATH, QPShiftModel, features
    X, D, eps_t = synthetic_system_torch(400, 40, 2400, seed=5, variant='calibrated')
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, 40, ntau=20)
    res = gw_sweep(X, D, eps, 40, axes=axes, precision='mixed')
    model = QPShiftModel.load(MODEL_PATH)
    warm = model.predict_roots(X, D, eps, 40, axes, sweep=res)
    r = qp_solve(res['sigma'], axes.pade_freq, eps, res['states'], 40, axes.mu, warm=warm)
    x = features(X, D, eps, 40, res)
    xs = x.repeat(int(np.ceil(65536 / x.shape[0])), 1)[:65536].contiguous()
    ys = torch.zeros(65536, dtype=torch.float32, device=xs.device)
    model.fit(xs, ys, steps=5, batch=65536)
    torch.cuda.synchronize()
    print(f'qp/mlp case: warm accepted {int(((r[2] & 16) != 0).sum().item())} of 400')


def adjoint_fd(a):
    """The dRPA adjoint against central differences (one JSON line): a
    random unit direction in ~5e7 parameters meets the gradient at ~1e-4 of
    its norm, so E_c's FP64 rounding (~1e-13 Ha) limits the plain h = 1e-5
    quotient to ~1e-5 relative at this size; the Richardson combination of
    larger steps is reported beside it. Each difference is given relative
    to its direction's derivative and relative to the gradient's norm (the
    first is large for a direction nearly orthogonal to the gradient)."""
    import json
    import time
    from mbptcode_b200 import adjoint
    from mbptcode_b200.space_time import rpa_correlation_energy_space_time
    dev = torch.device('cuda')
    n, nocc, M = a.n or 1200, a.nocc or 120, a.M or 7200
    X, D, eps_t = synthetic_system_torch(n, nocc, M, seed=a.seed, variant='calibrated')
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, nocc, ntau=a.ntau)
    mu = axes.mu
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_c, eb, xb, db, _ = adjoint.rpa_energy_and_adjoint(X, D, eps, nocc, axes.grid, mu=mu)
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t0
    g = torch.Generator(device=dev).manual_seed(a.seed + 1)
    gnorm = float(torch.sqrt((torch.as_tensor(np.asarray(eb.cpu() if torch.is_tensor(eb) else eb),
                                              device=dev) ** 2).sum() + (xb ** 2).sum()
                             + (db ** 2).sum()))
    errs, rich, t_fd = [], [], time.perf_counter()
    abs_plain, abs_rich, projections = [], [], []
    for _ in range(a.directions):
        de = torch.randn(n, generator=g, device=dev, dtype=torch.float64)
        dX = torch.randn(M, n, generator=g, device=dev, dtype=torch.float64)
        dD = torch.randn(M, M, generator=g, device=dev, dtype=torch.float64)
        norm = torch.sqrt((de ** 2).sum() + (dX ** 2).sum() + (dD ** 2).sum())
        de, dX, dD = de / norm, dX / norm, dD / norm
        de_h = de.cpu().numpy()
        ad = float((eb * de).sum() + (xb * dX).sum() + (db * dD).sum())

        def energy(t, dX=dX, dD=dD, de_h=de_h):
            return rpa_correlation_energy_space_time(X + t * dX, D + t * dD, eps + t * de_h,
                                                     nocc, axes.grid, mu=mu, precision='fp64')

        def central(h):
            return (energy(h) - energy(-h)) / (2 * h)
        cp = central(a.h)
        errs.append(abs(cp - ad) / max(abs(ad), 1e-300))
        r = (4 * central(a.h_richardson / 2) - central(a.h_richardson)) / 3
        rich.append(abs(r - ad) / max(abs(ad), 1e-300))
        abs_plain.append(abs(cp - ad) / gnorm)
        abs_rich.append(abs(r - ad) / gnorm)
        projections.append(abs(ad) / gnorm)
    t_fd = time.perf_counter() - t_fd
    print(json.dumps({
        'config': {'n_orb': n, 'nocc': nocc, 'N_mu': M, 'ntau': a.ntau,
                   'variant': 'calibrated', 'directions': a.directions, 'h': a.h},
        'e_c_Ha': float(e_c), 'max_rel_diff': max(errs),
        'median_rel_diff': float(np.median(errs)),
        'richardson_h': a.h_richardson, 'richardson_max_rel_diff': max(rich),
        'richardson_median_rel_diff': float(np.median(rich)),
        'gradient_norm': gnorm,
        'min_projection_over_gradient_norm': float(min(projections)),
        'max_diff_over_gradient_norm': float(max(abs_plain)),
        'richardson_max_diff_over_gradient_norm': float(max(abs_rich)),
        'seconds_energy_and_adjoint': round(t_adj, 3), 'seconds_differences': round(t_fd, 2)}),
        flush=True)



def adjoint_time(a):
    """E_c and dE_c/d(eps, X, D) at n_orb = 1200, N_mu = 7200, 24 points
    (calibrated), timed with CUDA events after a warm-up call; one JSON line
    with the FP64 products' route (MBPT_FP64_GEMM) and the self-energy
    adjoint of 20 states beside it."""
    import json
    import os
    from mbptcode_b200 import adjoint
    n, nocc, M = a.n or 1200, a.nocc or 120, a.M or 7200
    X, D, eps_t = synthetic_system_torch(n, nocc, M, seed=2024, variant='calibrated')
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, nocc, ntau=a.ntau)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3, out
    t_adj, out = timed(lambda: adjoint.rpa_energy_and_adjoint(X, D, eps, nocc, axes.grid,
                                                              mu=axes.mu))
    states20 = np.arange(nocc - 10, nocc + 10)
    tr = grids.sigma_transforms(eps, nocc, axes.grid.tau_points, axes.grid.omega_points,
                                axes.pade_freq, mu=axes.mu)

    def sigma_adjoint():
        sig, cache = adjoint.selfenergy_diag(X, D, eps_t, nocc, axes.grid, states20, tr,
                                             axes.mu)
        ones = torch.ones(sig.shape, dtype=torch.float64, device=sig.device)
        return adjoint.selfenergy_diag_backward(ones, ones, X, D, eps_t, nocc, axes.grid,
                                                states20, tr, axes.mu, cache)
    t_sig, _ = timed(sigma_adjoint)
    print(json.dumps({'case': 'adjoint-time', 'fp64_gemm': os.environ.get('MBPT_FP64_GEMM',
                                                                          'cublas'),
                      'n_orb': n, 'N_mu': M, 'ntau': a.ntau, 'e_c_Ha': float(out[0]),
                      'rpa_energy_and_adjoint_s': round(t_adj, 4),
                      'selfenergy_diag_and_adjoint_20_states_s': round(t_sig, 4),
                      'eps_bar_norm': float(np.linalg.norm(np.asarray(
                          out[1].cpu().numpy() if torch.is_tensor(out[1]) else out[1])))}),
          flush=True)


def ozaki_gemm_case(a):
    """C = A B^T (N x N x N, FP64 row-major) by the int8 Ozaki GEMM
    (mbpt_dgemm_ozaki, 8 digits) and by torch's FP64 product, three calls
    each, CUDA-event timed; the capture case of the Ozaki kernel (one
    launch of chol_update_kernel per call)."""
    import json
    from mbptcode_b200 import _lib
    from mbptcode_b200._lib import check, lib, ptr
    n = a.ozaki_gemm
    g = torch.Generator(device='cuda').manual_seed(11)
    A = torch.randn(n, n, generator=g, device='cuda', dtype=torch.float64)
    B = torch.randn(n, n, generator=g, device='cuda', dtype=torch.float64)
    C = torch.empty(n, n, dtype=torch.float64, device='cuda')
    ws = torch.empty(lib().mbpt_dgemm_ozaki_workspace_bytes(n, n, n, 8), dtype=torch.uint8,
                     device='cuda')

    def oz():
        check(lib().mbpt_dgemm_ozaki(0, 1, n, n, n, 1.0, ptr(A), n, ptr(B), n, 0.0, ptr(C), n, 8,
                                     ptr(ws), ws.numel(), None, _lib.stream_ptr()),
              'mbpt_dgemm_ozaki')

    def best(fn):
        ts = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return min(ts)
    t_oz = best(oz)
    ref = A @ B.T
    t_d = best(lambda: A @ B.T)
    err = float((C - ref).abs().max() / ref.abs().max())
    print(json.dumps({'case': 'ozaki-gemm', 'n': n, 'ozaki_s': round(t_oz, 5),
                      'ozaki_fp64_tflops': round(2 * n ** 3 / t_oz / 1e12, 1),
                      'dgemm_s': round(t_d, 5), 'dgemm_tflops': round(2 * n ** 3 / t_d / 1e12, 1),
                      'max_err_rel': err}), flush=True)

HARTREE_MEV = 27211.386245988


def make_system(n, seed, variant):
    nocc = max(2, n // 10)
    X, D, eps = synthetic_system_torch(n, nocc, 6 * n, seed=seed, variant=variant)
    return X, D, eps.cpu().numpy(), nocc


def frontier(nocc, n, width=10):
    return np.arange(max(0, nocc - width), min(n, nocc + width))


def warm_start(a):
    """The learned warm start at full scale; one JSON report (stdout, and
    --out when given)."""
    import json
    import time
    import warnings
    from mbptcode_b200.evgw import EvGWNotConverged, evgw_device
    from mbptcode_b200.gw import QPNoRoot, QPWeightOutside
    from mbptcode_b200.qp_mlp import QPShiftModel, method_samples, warm_start_compare
    warnings.simplefilter('ignore', QPWeightOutside)
    warnings.simplefilter('ignore', QPNoRoot)
    warnings.simplefilter('ignore', EvGWNotConverged)
    rng = np.random.default_rng(a.seed)
    n_train = rng.integers(a.nmin, a.nmax + 1, a.train)
    n_eval = rng.integers(a.nmin, a.nmax + 1, a.eval)

    # ---- training samples from the method itself ----
    t0 = time.perf_counter()
    xs, ys = [], []
    for i, n in enumerate(n_train):
        sys_ = make_system(int(n), 10_000 + i, a.variant)
        x, y, _ = method_samples([sys_], ntau=a.ntau, precision=a.precision)
        xs.append(x)
        ys.append(y)
        del sys_
    x, y = torch.cat(xs), torch.cat(ys)
    t_samples = time.perf_counter() - t0

    t0 = time.perf_counter()
    model = QPShiftModel(hidden=a.hidden, seed=a.seed)
    log = []
    model.fit(x, y, steps=a.steps, lr=3e-3, log=log)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    if a.save:
        model.save(a.save)
    with torch.no_grad():
        pred = model.predict_shift(x)
        train_mae = float((pred - y).abs().mean().item())
        train_max = float((pred - y).abs().max().item())

    # ---- evaluation: G0W0 and evGW, plain against warm-started ----
    g0w0, evgw = [], []
    t0 = time.perf_counter()
    for j, n in enumerate(n_eval):
        X, D, eps, nocc = make_system(int(n), 20_000 + j, a.variant)
        r = warm_start_compare(model, X, D, eps, nocc, ntau=a.ntau, precision=a.precision)
        g0w0.append(dict(n_orb=int(n), **r))
        tp = time.perf_counter()
        e_p, info_p = evgw_device(X, D, eps, nocc, ntau=a.ntau, precision=a.precision)
        tw = time.perf_counter()
        e_w, info_w = evgw_device(X, D, eps, nocc, ntau=a.ntau, precision=a.precision,
                                       warm=model, verify=True)
        te = time.perf_counter()
        e_q, _ = evgw_device(X, D, eps + 1e-11, nocc, ntau=a.ntau, precision=a.precision)
        ok = np.isfinite(e_p) & np.isfinite(e_w)
        okq = np.isfinite(e_p) & np.isfinite(e_q)
        f = frontier(nocc, int(n))
        evgw.append({
            'n_orb': int(n), 'cycles_plain': info_p['cycles'], 'cycles_warm': info_w['cycles'],
            'converged': bool(info_p['converged'] and info_w['converged']),
            'evals_plain': int(sum(info_p['sigma_evaluations'])),
            'evals_warm': int(sum(info_w['sigma_evaluations'])),
            'warm_accepted': int(sum(info_w['warm_accepted'])),
            'states_solved': int(n) * info_w['cycles'],
            'max_diff_meV': float(np.abs(e_w - e_p)[ok].max() * HARTREE_MEV),
            'frontier_max_diff_meV': float(np.abs(e_w - e_p)[f].max() * HARTREE_MEV),
            'verified_max_diff_meV': max(info_w['verify_max_diff'], default=0.0) * HARTREE_MEV,
            'perturbed_max_diff_meV': float(np.abs(e_q - e_p)[okq].max() * HARTREE_MEV),
            'perturbed_frontier_max_diff_meV': float(np.abs(e_q - e_p)[f].max() * HARTREE_MEV),
            's_plain': tw - tp, 's_warm': te - tw})
        del X, D
    t_eval = time.perf_counter() - t0

    def tot(rows, k):
        return int(sum(r[k] for r in rows))

    report = {
        'config': {'train_systems': a.train, 'eval_systems': a.eval,
                   'n_orb_range': [a.nmin, a.nmax], 'nocc': 'n_orb/10', 'N_mu': '6 n_orb',
                   'ntau': a.ntau, 'precision': a.precision, 'variant': a.variant,
                   'hidden': [a.hidden, a.hidden], 'train_steps': a.steps},
        'training': {'samples': int(x.shape[0]), 'seconds_samples': round(t_samples, 2),
                     'seconds_train': round(t_train, 2),
                     'loss_first': log[0][1], 'loss_last': log[-1][1],
                     'mae_meV': train_mae * HARTREE_MEV, 'max_err_meV': train_max * HARTREE_MEV},
        'g0w0': {'evals_plain': tot(g0w0, 'evals_plain'), 'evals_warm': tot(g0w0, 'evals_warm'),
                 'saved_frac': 1 - tot(g0w0, 'evals_warm') / max(1, tot(g0w0, 'evals_plain')),
                 'accepted_frac': tot(g0w0, 'accepted') / max(1, tot(g0w0, 'states')),
                 'max_root_diff_meV': max(r['max_root_diff'] for r in g0w0) * HARTREE_MEV,
                 'prediction_max_err_meV': max(r['pred_err_max'] for r in g0w0) * HARTREE_MEV},
        'evgw': {'evals_plain': tot(evgw, 'evals_plain'), 'evals_warm': tot(evgw, 'evals_warm'),
                 'saved_frac': 1 - tot(evgw, 'evals_warm') / max(1, tot(evgw, 'evals_plain')),
                 'accepted_frac': tot(evgw, 'warm_accepted') / max(1, tot(evgw, 'states_solved')),
                 'verified_max_diff_meV': max(r['verified_max_diff_meV'] for r in evgw),
                 'final_max_diff_meV': max(r['max_diff_meV'] for r in evgw),
                 'final_frontier_max_diff_meV': max(r['frontier_max_diff_meV'] for r in evgw),
                 'perturbed_final_max_diff_meV': max(r['perturbed_max_diff_meV'] for r in evgw),
                 'perturbed_final_frontier_max_diff_meV':
                     max(r['perturbed_frontier_max_diff_meV'] for r in evgw),
                 'all_converged': all(r['converged'] for r in evgw),
                 'cycles_plain': tot(evgw, 'cycles_plain'), 'cycles_warm': tot(evgw, 'cycles_warm'),
                 's_plain': round(sum(r['s_plain'] for r in evgw), 2),
                 's_warm': round(sum(r['s_warm'] for r in evgw), 2)},
        'seconds_eval': round(t_eval, 2),
        'per_system_evgw': evgw,
    }
    line = json.dumps(report)
    print(line)
    if a.out:
        with open(a.out, 'w') as fh:
            fh.write(line + '\n')
    return report


def main(argv=None):
    p = argparse.ArgumentParser(description='measurement cases beside bench.py')
    p.add_argument('case', choices=['tau', 'dyson', 'sweep', 'transform', 'qp-mlp', 'rows',
                                    'ao-sigma',
                                    'rows-cd', 'chi0-aux', 'fp64-peak', 'adjoint-fd',
                                    'adjoint-time', 'ozaki-gemm', 'warm-start'])
    p.add_argument('size', type=int, nargs='*', default=[])
    p.add_argument('--M', type=int, default=None)
    p.add_argument('--n', type=int, default=None)
    p.add_argument('--nocc', type=int, default=None)
    p.add_argument('--states', type=int, default=682)
    p.add_argument('--nfreq', type=int, default=1)
    p.add_argument('--time', action='store_true')
    p.add_argument('--mixed', action='store_true')
    # adjoint-fd
    p.add_argument('--ntau', type=int, default=24)
    p.add_argument('--directions', type=int, default=32)
    p.add_argument('--h', type=float, default=1e-5)
    p.add_argument('--h-richardson', type=float, default=1e-2)
    p.add_argument('--seed', type=int, default=None)
    # warm-start
    p.add_argument('--train', type=int, default=512)
    p.add_argument('--eval', type=int, default=64)
    p.add_argument('--nmin', type=int, default=100)
    p.add_argument('--nmax', type=int, default=800)
    p.add_argument('--precision', default='mixed', choices=['mixed', 'fp64'])
    p.add_argument('--variant', default='calibrated', choices=['calibrated', 'literal'])
    p.add_argument('--hidden', type=int, default=64)
    p.add_argument('--steps', type=int, default=3000)
    p.add_argument('--out', default=None)
    p.add_argument('--save', default=None, help='write the trained network (.npz)')
    a = p.parse_args(argv)
    torch.cuda.set_device(0)
    sized = {'dyson': 'dyson', 'transform': 'transform', 'fp64-peak': 'fp64_peak',
             'ozaki-gemm': 'ozaki_gemm'}
    if a.case in sized:
        setattr(a, sized[a.case], a.size[0])
    if a.case == 'chi0-aux':
        a.chi0_aux = tuple(a.size[:2])
    if a.seed is None:
        a.seed = 0 if a.case == 'warm-start' else 2024
    run = {'tau': tau_point, 'dyson': dyson, 'sweep': sweep, 'transform': transform_case,
           'ao-sigma': ao_sigma,
           'qp-mlp': qp_mlp_case, 'rows': rows, 'rows-cd': explicit_rows,
           'chi0-aux': chi0_aux_case, 'fp64-peak': fp64_peak, 'adjoint-fd': adjoint_fd,
           'adjoint-time': adjoint_time, 'ozaki-gemm': ozaki_gemm_case,
           'warm-start': warm_start}[a.case]
    if a.case in ('tau', 'sweep'):
        big = a.case == 'sweep'
        a.M = a.M or (7200 if big else 4096)
        a.n = a.n or (1200 if big else 682)
        a.nocc = a.nocc or (120 if big else 68)
    return run(a)


if __name__ == '__main__':
    main()
