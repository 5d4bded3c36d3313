"""Learned warm start of the quasiparticle root search.

A 4 -> H -> H -> 1 perceptron (SiLU, FP32) predicts each orbital's QP shift
w - eps_i from (eps_i, Sigma_x,ii, Re Sigma_c,ii(eps_i - 0.1), Re Sigma_c,ii(eps_i + 0.1))
(Hartree). The prediction seeds a safeguarded Newton solve in the QP kernel;
the plain graphical scan (MBPTcode ``Solvers/qp_equation.py:1353-1393``)
remains the fallback and the check of the prediction.

Features: Sigma_x,ii = -sum_PQ X_Pi (G_occ(0) o V)_PQ X_Qi with
G_occ(0) = X_o X_o^T and V = D D^T, the exchange of the ISDF factors (the
synthetic systems carry no other exchange integrals); it is the lesser
self-energy branch at tau = 0 with W replaced by the bare Coulomb factor, so
the self-energy kernel computes it. Sigma_c at eps_i +- 0.1 Ha comes from the
state's Pade continuation (mbpt_pade_eval).

Every arithmetic step -- features, forward, backward, AdamW -- runs in
libmbpt_b200; torch only holds the buffers.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from ._lib import WORKSPACE, check, host_array, lib, ptr, require_device, stream_ptr
from .gw import gw_sweep, sigma_branch_sums
from .space_time import _eps_host, to_device

FEATURE_OFFSET = 0.1  # Ha, the two real frequencies Sigma_c is read at
#: the network trained by `python bench_cases.py warm-start --save`
#: (512 method-generated systems, n_orb 100-800, mixed precision)
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data',
                          'qp_shift_model.npz')


def exchange_diagonal(X, D, eps, nocc, states, mu, precision='fp64', err=None):
    """Sigma_x,ii of `states` (device FP64). It depends on X, D and nocc only
    (G_occ(0) = X_o X_o^T carries no orbital energy), so an evGW loop
    computes it once."""
    dev = require_device()
    X, D = to_device(X, dev), to_device(D, dev)
    br = sigma_branch_sums(X, D, None, eps, nocc, [0.0], states, mu, precision=precision,
                           err=err)
    return -br[0, 0]


def sigma_at(sigma, pade_freq, states, nocc, mu, query):
    """Re Sigma_c(query[s, q]) from the continuation of state s (device FP64)."""
    dev = sigma.device
    sig = torch.view_as_real(sigma.contiguous()).contiguous()
    S, npade = sigma.shape
    pf_h, pp = host_array(pade_freq)
    st = torch.as_tensor(np.asarray(states, dtype=np.int64), device=dev)
    q = query.contiguous()
    out = torch.empty_like(q)
    ws = WORKSPACE.get(1 << 16, dev)
    check(lib().mbpt_pade_eval(ptr(sig), pp, npade, ptr(st), S, int(nocc), float(mu), 1,
                               ptr(q), q.shape[1], ptr(out), ptr(ws), ws.numel(),
                               stream_ptr()), 'mbpt_pade_eval')
    return out


def features(X, D, eps_anchor, nocc, sweep, sx=None):
    """(S, 4) FP32 device features of the states of a finished sweep; `sx`,
    the exchange diagonal of those states, is computed when not given."""
    states = sweep['states']
    axes = sweep['axes']
    dev = sweep['sigma'].device
    e = torch.as_tensor(np.asarray(_eps_host(eps_anchor), float)[states], device=dev)
    if sx is None:
        sx = exchange_diagonal(X, D, sweep.get('eps_sweep', eps_anchor), nocc, states, axes.mu)
    q = torch.stack([e - FEATURE_OFFSET, e + FEATURE_OFFSET], dim=1)
    sc = sigma_at(sweep['sigma'], axes.pade_freq, states, nocc, axes.mu, q)
    return torch.stack([e, sx, sc[:, 0], sc[:, 1]], dim=1).to(torch.float32).contiguous()


class QPShiftModel:
    """The network, its input/target standardisation and its optimiser state."""

    def __init__(self, hidden=64, seed=0, device=None):
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.hidden = hidden
        n = lib().mbpt_mlp_param_count(hidden)
        g = torch.Generator(device='cpu').manual_seed(seed)
        H = hidden
        parts = [torch.randn(H * 4, generator=g) * (2.0 / 4) ** 0.5, torch.zeros(H),
                 torch.randn(H * H, generator=g) * (2.0 / H) ** 0.5, torch.zeros(H),
                 torch.randn(H, generator=g) * (1.0 / H) ** 0.5, torch.zeros(1)]
        self.params = torch.cat(parts).to(torch.float32).to(self.device).contiguous()
        assert self.params.numel() == n
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.x_mean = torch.zeros(4, device=self.device)
        self.x_std = torch.ones(4, device=self.device)
        self.y_scale = 1.0

    # -- raw network on standardised inputs --
    def _forward(self, xs, act=None):
        y = torch.empty(xs.shape[0], dtype=torch.float32, device=self.device)
        check(lib().mbpt_mlp_forward(ptr(self.params), self.hidden, ptr(xs), xs.shape[0],
                                     ptr(y), ptr(act), stream_ptr()), 'mbpt_mlp_forward')
        return y

    def _grad(self, xs, ys):
        B = xs.shape[0]
        act = torch.empty((B, 4 * self.hidden), dtype=torch.float32, device=self.device)
        y = self._forward(xs, act)
        grad = torch.empty_like(self.params)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        check(lib().mbpt_mlp_backward(ptr(self.params), self.hidden, ptr(xs), B, ptr(act),
                                      ptr(y), ptr(ys), ptr(grad), ptr(loss), stream_ptr()),
              'mbpt_mlp_backward')
        return grad, loss

    def _adamw(self, grad, lr, wd=1e-5):
        self.step += 1
        check(lib().mbpt_mlp_adamw(ptr(self.params), ptr(grad), ptr(self.m), ptr(self.v),
                                   self.params.numel(), lr, 0.9, 0.999, 1e-8, wd, self.step,
                                   stream_ptr()), 'mbpt_mlp_adamw')

    def standardise(self, x):
        return ((x - self.x_mean) / self.x_std).contiguous()

    def fit(self, x, shift, steps=2000, lr=3e-3, batch=8192, seed=0, log=None):
        """Train on features x (N, 4) and targets `shift` (N,) (device)."""
        x = x.to(self.device, torch.float32)
        shift = shift.to(self.device, torch.float32)
        self.x_mean = x.mean(0)
        self.x_std = x.std(0).clamp_min(1e-6)
        self.y_scale = float(shift.abs().max().item()) or 1.0
        xs = self.standardise(x)
        ys = (shift / self.y_scale).contiguous()
        g = torch.Generator(device=self.device).manual_seed(seed)
        N = xs.shape[0]
        for it in range(steps):
            if N > batch:
                idx = torch.randint(0, N, (batch,), generator=g, device=self.device)
                xb, yb = xs[idx].contiguous(), ys[idx].contiguous()
            else:
                xb, yb = xs, ys
            rate = lr * 0.5 * (1 + np.cos(np.pi * it / steps))
            grad, loss = self._grad(xb, yb)
            self._adamw(grad, float(rate))
            if log is not None and (it % 200 == 0 or it == steps - 1):
                log.append((it, float(loss.item()) * self.y_scale ** 2))
        return self

    def predict_shift(self, x):
        return self._forward(self.standardise(x.to(self.device, torch.float32))) * self.y_scale

    def predict_roots(self, X, D, eps, nocc, axes, eps_anchor=None, precision=None, sweep=None,
                      sx=None):
        """Predicted QP roots of the sweep's states for the warm start, from
        the finished sweep `sweep` (whose Sigma the features read) and, when
        given, the states' exchange diagonal `sx`."""
        anchor = eps if eps_anchor is None else eps_anchor
        if sweep is None:
            raise ValueError('predict_roots needs the sweep whose Sigma it reads')
        x = features(X, D, anchor, nocc, sweep, sx=sx)
        e = x[:, 0].double()
        return e + self.predict_shift(x).double()

    def state_dict(self):
        return {'hidden': self.hidden, 'params': self.params.cpu().numpy(),
                'x_mean': self.x_mean.cpu().numpy(), 'x_std': self.x_std.cpu().numpy(),
                'y_scale': self.y_scale}

    def save(self, path):
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path, device=None):
        d = np.load(path)
        m = cls(int(d['hidden']), device=device)
        m.params = torch.as_tensor(d['params'], device=m.device).contiguous()
        m.x_mean = torch.as_tensor(d['x_mean'], device=m.device)
        m.x_std = torch.as_tensor(d['x_std'], device=m.device)
        m.y_scale = float(d['y_scale'])
        return m


def method_samples(systems, ntau=20, precision='fp64'):
    """(features, shifts, sweeps) from the plain method on `systems`
    [(X, D, eps, nocc)]: every orbital's Sigma, features and the QP shift of
    the graphical solve."""
    xs, ys, sweeps = [], [], []
    for X, D, eps, nocc in systems:
        res = gw_sweep(X, D, eps, nocc, ntau=ntau, precision=precision)
        x = features(X, D, eps, nocc, res)
        y = res['roots'] - torch.as_tensor(_eps_host(eps), device=res['roots'].device)
        ok = torch.isfinite(y) & torch.isfinite(x).all(1)
        xs.append(x[ok])
        ys.append(y[ok].float())
        sweeps.append(res)
    return torch.cat(xs), torch.cat(ys), sweeps


def warm_start_compare(model, X, D, eps, nocc, ntau=20, precision='fp64'):
    """Solve one system plainly and warm-started from the model's roots.
    Returns the Sigma evaluations of both, the number of warm starts the
    kernel accepted and the largest root difference (Hartree)."""
    from .gw import qp_solve
    res = gw_sweep(X, D, eps, nocc, ntau=ntau, precision=precision)
    axes = res['axes']
    warm = model.predict_roots(X, D, eps, nocc, axes, sweep=res)
    r_w, z_w, f_w, e_w = qp_solve(res['sigma'], axes.pade_freq, _eps_host(eps), res['states'],
                                  nocc, axes.mu, warm=warm)
    r_p, e_p = res['roots'], res['evals']
    ok = torch.isfinite(r_p) & torch.isfinite(r_w)
    return {'evals_plain': int(e_p.sum().item()), 'evals_warm': int(e_w.sum().item()),
            'accepted': int(((f_w & 16) != 0).sum().item()), 'states': int(len(res['states'])),
            'max_root_diff': float((r_w - r_p)[ok].abs().max().item()),
            'pred_err_max': float((warm - r_p)[ok].abs().max().item())}
