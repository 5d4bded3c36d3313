"""Small, self-contained invocations of the route for profiling under ncu.

    python -m mbptcode_b200.profile_case [--M 4096] [--n 682] [--nocc 68] [--states 682]
    python -m mbptcode_b200.profile_case --dyson 4096 [--nfreq 1]
    python -m mbptcode_b200.profile_case --sweep [--M 7200] [--n 1200] [--nocc 120]

Default: one tau point of the chi0 sweep and one of the self-energy sweep,
mixed precision. Launches, in order: the branch preparation, the TF32x3
G_occ/G_virt/Pi kernel, Z = D^T Pi, proj = -2 D^T Z^T, the FP64 transform,
then on the self-energy side U = D W, the G_occ/G_virt/Zt kernel with the H
epilogue and the row-contraction kernel -- one launch of each engine kernel.
Device memory stays at a few GB (M = 4096: about 1 GB).

--dyson N [--time]: the mixed Dyson step of `nfreq` frequencies of an N x N chi0
(negative definite, seeded): cuSOLVER's Cholesky, the shared-memory diagonal
blocks, the TF32-pair recursion (2 engine launches per node; with leaves of
128 the last three engine launches of a frequency are the top node's two
products and W = L^-T L^-1) and the mirrored FP64 store. From 4 frequencies
on, the factorisations are one batched Cholesky of all of them. --time
prints CUDA-event times of the factorisations alone and of the whole step.

--sweep: one whole mixed chi0 -> W -> Sigma -> QP sweep (24 points) of a
synthetic system, for the launch list of the benchmark's workload.

--transform N: one FP64 tau <-> omega transform of 24 N x N matrices with a
24 x 24 weight matrix (mbpt_transform, the W(i w) -> W(tau) step).

--qp-mlp: the latency-bound kernels of the QP solve and the learned warm
start on a C1-sized system (n_orb = 400, N_mu = 2400, 20 points, mixed): one
sweep, the plain and the warm-started Pade + QP kernels and the Pade
evaluation of the features, then 5 training steps of the 4 -> 64 -> 64 -> 1
network on 65536 samples (forward, backward, AdamW).

--rows: device times at n_orb = 1200, N_mu = 7200 of the rows built beside the
sweep: the static screening, the frequency-blocked and the unrestricted sweeps,
the self-energy diagonal with its adjoint (20 states), the contour's
screening contraction (64 frequencies, 20 states) and one Sigma^c evaluation.

--rows-cd: the contour's explicit particle-hole backend (continuation 'cd') at
the same size: C_ov, the explicit response at one real frequency and one
W(freq) - I below and above the particle-hole gap.

--chi0-aux NAUX NOV [--mixed]: the explicit response alone on a seeded factor,
three calls (the capture case of its engine launch).

--fp64-peak N: the FP64 reference rates of this GPU, timed with CUDA events
(best of 5 after a warm-up): cuBLAS DGEMM at N^3 and cuSOLVER's Cholesky of
an N x N SPD matrix (the FP64 factorisation of the Dyson step).
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import grids
from .gw import gw_sweep, sigma_branch_sums
from .space_time import chi0_sweep, dyson_batch
from .synthetic import synthetic_system_torch


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
    from .space_time import transform
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
    from . import adjoint, contour, gw, space_time
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


def explicit_rows(a):
    """Device times of the contour's explicit particle-hole backend
    (continuation 'cd') at n_orb = 1200, nocc = 120, N_mu = 7200: C_ov
    (7200 x 129600) from the occupied slices, the explicit response at one
    real frequency (mbpt_chi0_aux: naux (naux + 1) nov useful flops of a
    symmetric rank-k product) and one W(freq) - I below and above the gap
    (the Dyson step: Cholesky below, LU above). One JSON line each."""
    import json
    from . import contour, space_time
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
    from . import space_time
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
    from .gw import qp_solve
    from .qp_mlp import MODEL_PATH, QPShiftModel, features
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


def main():
    p = argparse.ArgumentParser()
    p.add_argument('--M', type=int, default=None)
    p.add_argument('--n', type=int, default=None)
    p.add_argument('--nocc', type=int, default=None)
    p.add_argument('--states', type=int, default=682)
    p.add_argument('--dyson', type=int, default=0)
    p.add_argument('--nfreq', type=int, default=1)
    p.add_argument('--time', action='store_true')
    p.add_argument('--sweep', action='store_true')
    p.add_argument('--transform', type=int, default=0)
    p.add_argument('--fp64-peak', type=int, default=0)
    p.add_argument('--qp-mlp', action='store_true')
    p.add_argument('--rows', action='store_true')
    p.add_argument('--rows-cd', action='store_true')
    p.add_argument('--chi0-aux', type=int, nargs=2, default=None)
    p.add_argument('--mixed', action='store_true')
    a = p.parse_args()
    torch.cuda.set_device(0)
    if a.qp_mlp:
        return qp_mlp_case(a)
    if a.rows:
        return rows(a)
    if a.rows_cd:
        return explicit_rows(a)
    if a.chi0_aux:
        return chi0_aux_case(a)
    if a.fp64_peak:
        return fp64_peak(a)
    if a.dyson:
        return dyson(a)
    if a.transform:
        return transform_case(a)
    big = a.sweep
    a.M = a.M or (7200 if big else 4096)
    a.n = a.n or (1200 if big else 682)
    a.nocc = a.nocc or (120 if big else 68)
    return sweep(a) if a.sweep else tau_point(a)


if __name__ == '__main__':
    main()
