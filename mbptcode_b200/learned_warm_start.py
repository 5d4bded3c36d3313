"""The learned quasiparticle warm start at the scale it is meant for.

    python -m mbptcode_b200.learned_warm_start [--train 512] [--eval 64] [--out report.json]

Training: `--train` seeded synthetic systems (n_orb uniform in [100, 800],
nocc = n_orb / 10, N_mu = 6 n_orb, the calibrated generator) each go through
one G0W0 sweep of the method itself; every orbital's features (eps_i,
Sigma_x,ii, Re Sigma_c,ii at eps_i -+ 0.1 Ha) and graphical-solve QP shift
become one sample. The 4 -> 64 -> 64 -> 1 network is trained on the GPU by
libmbpt_b200's forward, backward and AdamW kernels.

Evaluation: `--eval` further systems, each solved by the evGW loop
(eigenvalue self-consistency with Pulay DIIS) plainly (the graphical scan of
every state) and warm-started (the network's roots seed the kernel's Newton
solve; the scan stays the fallback for any state whose Newton solve is not
accepted). Reported: Sigma evaluations of both runs and the fraction of warm
starts accepted; the QP error of the warm start, checked every cycle against
the plain scan on the same Sigma (meV); and a G0W0 comparison of the same
systems. The two runs' final spectra are reported too, next to the spread
that a 1e-11 Ha change of the mean-field energies alone causes in the plain
loop: far from the gap the evGW fixed point selects between near-equal QP
roots, so any rounding-level change moves those states by up to hundreds
of meV, and the final-spectrum difference measures that conditioning rather
than the warm start.

The report is one JSON object (stdout, and `--out` when given).
"""
from __future__ import annotations

import argparse
import json
import time
import warnings

import numpy as np
import torch

from .evgw import EvGWNotConverged, evgw_eigenvalues
from .gw import QPNoRoot, QPWeightOutside
from .qp_mlp import QPShiftModel, method_samples, warm_start_compare
from .synthetic import synthetic_system_torch

HARTREE_MEV = 27211.386245988


def make_system(n, seed, variant):
    nocc = max(2, n // 10)
    X, D, eps = synthetic_system_torch(n, nocc, 6 * n, seed=seed, variant=variant)
    return X, D, eps.cpu().numpy(), nocc


def frontier(nocc, n, width=10):
    return np.arange(max(0, nocc - width), min(n, nocc + width))


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument('--train', type=int, default=512)
    p.add_argument('--eval', type=int, default=64)
    p.add_argument('--nmin', type=int, default=100)
    p.add_argument('--nmax', type=int, default=800)
    p.add_argument('--ntau', type=int, default=24)
    p.add_argument('--precision', default='mixed', choices=['mixed', 'fp64'])
    p.add_argument('--variant', default='calibrated', choices=['calibrated', 'literal'])
    p.add_argument('--hidden', type=int, default=64)
    p.add_argument('--steps', type=int, default=3000)
    p.add_argument('--seed', type=int, default=0)
    p.add_argument('--out', default=None)
    p.add_argument('--save', default=None, help='write the trained network (.npz)')
    a = p.parse_args(argv)
    torch.cuda.set_device(0)
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
        e_p, info_p = evgw_eigenvalues(X, D, eps, nocc, ntau=a.ntau, precision=a.precision)
        tw = time.perf_counter()
        e_w, info_w = evgw_eigenvalues(X, D, eps, nocc, ntau=a.ntau, precision=a.precision,
                                       warm=model, verify=True)
        te = time.perf_counter()
        e_q, _ = evgw_eigenvalues(X, D, eps + 1e-11, nocc, ntau=a.ntau, precision=a.precision)
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


if __name__ == '__main__':
    main()
