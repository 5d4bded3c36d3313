"""The dRPA adjoint against central differences at the precision
configuration's size.

    python -m mbptcode_b200.adjoint_check [--n 1200] [--nocc 120] [--M 7200]
        [--ntau 24] [--directions 32] [--h 1e-5] [--out report.json]

E_c and dE_c/d(eps, X, D) in FP64 on the device (the reverse sweep recomputes
G(tau) per tau), then (E_c(+h d) - E_c(-h d)) / 2h along `directions` seeded
unit directions d in (eps, X, D), with the grid and mu frozen as the adjoint
assumes, and the Richardson combination (4 D(h_r / 2) - D(h_r)) / 3 of
central differences at h_r = 1e-2 (truncation O(h^4)): a random unit direction
in ~5e7 parameters meets the gradient at ~1e-4 of its norm, so E_c's FP64
rounding limits the plain h = 1e-5 quotient to ~1e-5 relative. Prints one
JSON object: the largest and median relative differences and the timings.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import adjoint, grids
from .space_time import rpa_correlation_energy_space_time
from .synthetic import synthetic_system_torch


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument('--n', type=int, default=1200)
    p.add_argument('--nocc', type=int, default=120)
    p.add_argument('--M', type=int, default=7200)
    p.add_argument('--ntau', type=int, default=24)
    p.add_argument('--directions', type=int, default=32)
    p.add_argument('--h', type=float, default=1e-5)
    p.add_argument('--h-richardson', type=float, default=1e-2)
    p.add_argument('--variant', default='calibrated', choices=['calibrated', 'literal'])
    p.add_argument('--seed', type=int, default=2024)
    p.add_argument('--out', default=None)
    a = p.parse_args(argv)
    torch.cuda.set_device(0)
    dev = torch.device('cuda')
    X, D, eps_t = synthetic_system_torch(a.n, a.nocc, a.M, seed=a.seed, variant=a.variant)
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, a.nocc, ntau=a.ntau)
    mu = axes.mu
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_c, eb, xb, db, _ = adjoint.rpa_energy_and_adjoint(X, D, eps, a.nocc, axes.grid, mu=mu)
    torch.cuda.synchronize()
    t_adj = time.perf_counter() - t0
    g = torch.Generator(device=dev).manual_seed(a.seed + 1)
    errs, rich, t_fd = [], [], time.perf_counter()
    for _ in range(a.directions):
        de = torch.randn(a.n, generator=g, device=dev, dtype=torch.float64)
        dX = torch.randn(a.M, a.n, generator=g, device=dev, dtype=torch.float64)
        dD = torch.randn(a.M, a.M, generator=g, device=dev, dtype=torch.float64)
        norm = torch.sqrt((de ** 2).sum() + (dX ** 2).sum() + (dD ** 2).sum())
        de, dX, dD = de / norm, dX / norm, dD / norm
        de_h = de.cpu().numpy()
        ad = float((eb * torch.as_tensor(de_h, device=dev)).sum() + (xb * dX).sum()
                   + (db * dD).sum())

        def energy(t, dX=dX, dD=dD, de_h=de_h):
            return rpa_correlation_energy_space_time(X + t * dX, D + t * dD, eps + t * de_h,
                                                     a.nocc, axes.grid, mu=mu,
                                                     precision='fp64')

        def central(h):
            return (energy(h) - energy(-h)) / (2 * h)
        errs.append(abs(central(a.h) - ad) / max(abs(ad), 1e-300))
        r = (4 * central(a.h_richardson / 2) - central(a.h_richardson)) / 3
        rich.append(abs(r - ad) / max(abs(ad), 1e-300))
    t_fd = time.perf_counter() - t_fd
    report = {'config': {'n_orb': a.n, 'nocc': a.nocc, 'N_mu': a.M, 'ntau': a.ntau,
                         'variant': a.variant, 'directions': a.directions, 'h': a.h},
              'e_c_Ha': float(e_c.item()) if torch.is_tensor(e_c) else float(e_c),
              'max_rel_diff': max(errs), 'median_rel_diff': float(np.median(errs)),
              'richardson_h': a.h_richardson, 'richardson_max_rel_diff': max(rich),
              'richardson_median_rel_diff': float(np.median(rich)),
              'seconds_energy_and_adjoint': round(t_adj, 3),
              'seconds_differences': round(t_fd, 2)}
    line = json.dumps(report)
    print(line)
    if a.out:
        with open(a.out, 'w') as fh:
            fh.write(line + '\n')
    return report


if __name__ == '__main__':
    main()
