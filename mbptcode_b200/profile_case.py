"""One tau point of the chi0 sweep and one of the self-energy sweep, mixed
precision, for profiling the tensor-core engine under ncu.

    python -m mbptcode_b200.profile_case [--M 4096] [--n 682] [--nocc 68] [--states 682]

Launches, in order: the branch preparation, the TF32x3 G_occ/G_virt/Pi
kernel, Z = D^T Pi, proj = -2 D^T Z^T, the FP64 transform, then on the
self-energy side U = D W, the G_occ/G_virt/Zt kernel with the H epilogue and
the row-contraction kernel -- one launch of each engine kernel. Device
memory stays at a few GB (M = 4096: about 1 GB).
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from . import grids
from .gw import sigma_branch_sums
from .space_time import chi0_sweep
from .synthetic import synthetic_system_torch


def main():
    p = argparse.ArgumentParser()
    p.add_argument('--M', type=int, default=4096)
    p.add_argument('--n', type=int, default=682)
    p.add_argument('--nocc', type=int, default=68)
    p.add_argument('--states', type=int, default=682)
    a = p.parse_args()
    torch.cuda.set_device(0)
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


if __name__ == '__main__':
    main()
