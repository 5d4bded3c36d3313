"""Benchmark of the space-time chi0 -> W -> Sigma -> QP sweep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

Workload (the precision configuration): n_orb = 1200, nocc = 120, N_mu = 7200
interpolation points, 24 tau/omega points, synthetic seeded ISDF factors (no
dataset exists for this path), the Sigma diagonal and QP roots of all 1200
states. One step = one whole sweep (chi0 over 24 tau points, 24 FP64 Cholesky
factorisations with log-determinants and inverses, W(tau), Sigma over 24 tau
points, Pade + QP root search) in mixed precision on device-resident inputs.

Reported: `value` = seconds per mixed-precision sweep of the whole job (one GPU:
the sweep time; N replicas: the slowest rank's sweep time / N), the
learned warm start of the QP solve included, the plain FP64 GPU sweep beside it, the accuracy of mixed against FP64 (E_c in
uHa and uHa/electron, the 20 HOMO/LUMO-region QP energies in meV), `e2e` =
the same sweep through the public call with host inputs (pinned host ->
device copies of X, D, eps and the roots back inside the timed region),
`roofline` of the dominant tensor-core kernel timed live with CUDA events,
and `cpu_baseline` = the NumPy oracle (the reference's algorithm) timed on a
bounded sample of the same workload on the host cores.

--impl reference: the reference's algorithm (the NumPy oracle port; the
reference itself is Python and cannot run where this runs) on the host
cores: one whole sweep timed once is the line's value, and each of the K
steps is a bounded sample extrapolated to a sweep, reported beside it.

Multi-GPU: the sweep does not shard in this build (one GPU per system), so
--gpus N runs N independent replicas ("weak" scaling), no collective on the
data path; the metric is time-like, so `value` is the job's seconds per
sweep (max-over-ranks sweep time / N), `sweeps_per_s` the job throughput and
`per_replica_s_per_sweep` the slowest rank's own sweep time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ('χ0→W→Σ sweep s at n_orb=1200: mixed vs FP64 GPU at '
          '≤10 meV QP / ≤1µHa/e E_c')
HARTREE_EV = 27.211386245988
N_ORB, NOCC, M, NTAU = 1200, 120, 7200, 24
SEED = 2024

# algorithmic FLOPs of one launch of each engine kernel at this workload
# (the split products' 3x and the padding are not counted). Pi, proj and H are
# symmetric: those launches form the 128 x 128 tiles on and above the
# diagonal only (T (T + 1) / 2 of T^2, T = 57 tile rows) and count that work.
_T = -(-M // 128)
SYM = (_T * (_T + 1) / 2) / (_T * _T)
FLOPS = {
    'hadamard': SYM * 2.0 * M * M * N_ORB,              # G_occ and G_virt of one tau
    'split': 2.0 * M * M * M,                           # D^T Pi  /  D Wt
    'f32': SYM * 2.0 * M * M * M,                       # D^T (Pi D) and Zt = U D^T
    'sigma_hadamard': SYM * 2.0 * M * M * N_ORB,        # G_occ, G_virt (o Zt)
    'row_contraction': 2.0 * 2.0 * M * M * N_ORB,       # (G o Zt) X_s, both branches
}
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# engine kernels at this workload, from one ncu capture of a tau point at full
# size (python bench_cases.py tau --M 7200 --n 1200 --nocc 120
# --states 1200, the seven engine launches of one tau point)
TRAFFIC_BYTES = {'hadamard': 362.1e6, 'split': 1955.8e6, 'f32': 1143.4e6,
                 'sigma_hadamard': 591.7e6, 'row_contraction': 702.7e6}
# algorithmic FLOPs of the Dyson step's inverse per frequency (triangular inverse
# n^3/3 + L^-T L^-1 n^3/3, the classical SPD-inverse count), spread over launches
# of many sizes: rated on their summed time
DYSON_INV_FLOPS = 2.0 / 3.0 * M ** 3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=3)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='mine', choices=['mine', 'reference'])
    p.add_argument('--variant', default='literal', choices=['literal', 'calibrated'])
    p.add_argument('--no-cpu', action='store_true', help='skip the CPU-baseline sample')
    p.add_argument('--no-accuracy-other', action='store_true')
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
            d = json.load(fh)
        return d, 'measured'
    except OSError:
        return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0,
                'bf16_tflops_sustained': 1400.0}, 'fallback'


# --------------------------------------------------------------- CPU sample
def cpu_sample(X, D, eps, axes, steps=1):
    """Time the oracle on a bounded sample of the workload and extrapolate to
    one sweep: one tau point of the chi0 sweep, one frequency of the Dyson
    inversion, one tau point of the self-energy for all states, and the QP
    solve of 20 states; scaled by 24, 24, 24 and 1200/20."""
    from threadpoolctl import threadpool_info, threadpool_limits
    from oracle import st_oracle as orc
    cores = len(os.sched_getaffinity(0))
    with threadpool_limits(limits=cores):
        X_o, X_v, e_o, e_v, mu = orc.split_branches(X, eps, NOCC, axes.mu)
        per = []
        for _ in range(steps):
            t0 = time.perf_counter()
            proj = orc.polarizability_projected_tau(X_o, X_v, e_o, e_v, D,
                                                    axes.grid.tau_points[NTAU // 2])
            t1 = time.perf_counter()
            chi = np.tensordot(axes.grid.cosft_wt[:1, NTAU // 2], proj[None], axes=(0, 0))
            W = orc.dyson_screening(chi, correlation=True)
            t2 = time.perf_counter()
            sig = orc.sigma_branch_sums(X, D, W[None], eps, NOCC,
                                        axes.tau_sigma[NTAU // 2:NTAU // 2 + 1], axes.mu,
                                        np.arange(N_ORB))
            t3 = time.perf_counter()
            st = np.arange(NOCC - 10, NOCC + 10)
            s_iw = orc.sigma_frequency(np.repeat(sig, NTAU, axis=1)[:, :, st] / NTAU,
                                       axes.C, axes.S)
            orc.finish_qp(s_iw, eps, NOCC, st, axes.mu, axes.pade_freq)
            t4 = time.perf_counter()
            per.append(NTAU * (t1 - t0) + NTAU * (t2 - t1) + NTAU * (t3 - t2)
                       + (N_ORB / 20.0) * (t4 - t3))
            sample_s = t4 - t0
        blas = [f"{i.get('internal_api')} {i.get('version')} ({i.get('num_threads')} threads)"
                for i in threadpool_info()]
    return float(np.mean(per)), cores, sample_s, blas


def cpu_whole_sweep(X, D, eps, axes):
    """Time one whole sweep of the oracle on the host cores: chi0 at every
    frequency (24 tau points), E_c from its log-determinants, the Dyson
    inversion of every frequency, W(tau), the Sigma diagonal of all 1200
    states (the diagonal form of the self-energy, cheaper than the
    reference's AO build) and the QP roots of all states. Returns (seconds,
    per-stage seconds, cores)."""
    from threadpoolctl import threadpool_limits
    from oracle import st_oracle as orc
    cores = len(os.sched_getaffinity(0))
    states = np.arange(N_ORB)
    with threadpool_limits(limits=cores):
        t0 = time.perf_counter()
        chi0 = orc.chi0_imaginary_frequency(X, D, eps, NOCC, axes.grid, axes.mu)
        t1 = time.perf_counter()
        e_c = 0.0
        for k in range(len(chi0)):
            c = chi0[k]
            e_c += axes.grid.omega_weights[k] * (
                orc.dielectric_log_determinant(np.eye(c.shape[0]) - c, k) + np.trace(c))
            chi0[k] = orc.dyson_screening(c, correlation=True)
        t2 = time.perf_counter()
        Wt = np.tensordot(axes.Ctw, chi0, axes=(1, 0))
        del chi0
        sig = orc.sigma_branch_sums(X, D, Wt, eps, NOCC, axes.tau_sigma, axes.mu, states)
        del Wt
        sigma = orc.sigma_frequency(sig, axes.C, axes.S)
        t3 = time.perf_counter()
        orc.finish_qp(sigma, eps, NOCC, states, axes.mu, axes.pade_freq)
        t4 = time.perf_counter()
    stages = {'t_chi0': t1 - t0, 't_dyson_and_e_c': t2 - t1, 't_sigma': t3 - t2,
              't_qp': t4 - t3}
    return t4 - t0, {k: round(v, 2) for k, v in stages.items()}, cores


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling every 200 ms. Started a few seconds before the
    timed region (its start-up stalls the GPU's clients for a moment), with
    `window` marking the timed region; only samples inside it are kept."""

    def __init__(self, index):
        # the samples go to a temporary file unless MBPT_CLOCKS_CSV names one
        self.path = os.environ.get('MBPT_CLOCKS_CSV') or os.path.join(
            tempfile.mkdtemp(prefix='mbpt_clocks_'), f'clocks_{index}.csv')
        os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
        self.t0 = self.t1 = None
        q = ('timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
        try:
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={q}', '--format=csv',
                                          '-lms', '200', '-i', str(index)], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def window(self, start):
        import datetime
        now = datetime.datetime.now()
        if start:
            self.t0 = now
        else:
            self.t1 = now

    def stop(self):
        import datetime
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        time.sleep(0.3)
        self.proc.terminate()
        self.proc.wait()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in open(self.path).read().splitlines()[1:]:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], '%Y/%m/%d %H:%M:%S.%f')
                if (self.t0 and ts < self.t0) or (self.t1 and ts > self.t1):
                    continue
                sm.append(float(f[1].split()[0]))
                smax = float(f[2].split()[0])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == 'active':
                    reasons.add(name)
        return {'sm_mhz': float(np.median(sm)) if sm else None, 'sm_max_mhz': smax,
                'reasons': sorted(reasons), 'samples': len(sm)}


# ------------------------------------------------------------------ helpers
def frontier_states():
    return np.arange(NOCC - 10, NOCC + 10)


def accuracy(mixed, fp64):
    st = frontier_states()
    rm, rf = mixed['roots'].cpu().numpy(), fp64['roots'].cpu().numpy()
    dq = np.abs(rm[st] - rf[st]) * HARTREE_EV * 1e3
    de = abs(float(mixed['e_c']) - float(fp64['e_c']))
    return {'e_c_fp64_Ha': float(fp64['e_c']), 'e_c_err_uHa': de * 1e6,
            'e_c_err_uHa_per_e': de * 1e6 / (2 * NOCC),
            'qp_err_meV_max': float(dq.max()), 'qp_err_meV_mean': float(dq.mean()),
            'qp_states': [int(st[0]), int(st[-1])],
            'qp_all_err_meV_max': float(np.nanmax(np.abs(rm - rf)) * HARTREE_EV * 1e3)}


def main():
    args = parse()
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        return reference_arm(args, world, rank)

    import torch
    import torch.distributed as dist
    from mbptcode_b200 import _lib, grids
    from mbptcode_b200.gw import gw_space_time, gw_sweep, qp_solve
    from mbptcode_b200.qp_mlp import MODEL_PATH, QPShiftModel
    from mbptcode_b200.synthetic import synthetic_system_torch

    torch.cuda.set_device(local)
    dev = _lib.require_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=300),
                                device_id=torch.device('cuda', local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    X, D, eps_t = synthetic_system_torch(N_ORB, NOCC, M, seed=SEED + rank,
                                         variant=args.variant, device=dev)
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, NOCC, ntau=NTAU)
    states = np.arange(N_ORB)

    # the learned QP warm start (trained by `bench_cases.py warm-start` on
    # method-generated systems, shipped with the package): the mixed sweep's QP
    # solve is warm-started, the plain FP64 path solves by the graphical scan
    model = QPShiftModel.load(MODEL_PATH, device=dev)

    def sweep(precision):
        return gw_sweep(X, D, eps, NOCC, states=states, axes=axes, precision=precision,
                        warm=model if precision == 'mixed' else None)

    clocks = Clocks(torch.cuda.current_device()) if rank == 0 else None
    for _ in range(args.warmup):
        sweep('mixed')
    torch.cuda.synchronize()

    # ---- timed region: K mixed sweeps on resident inputs ----
    # the engine's single-shape kernels are event-timed inside the region;
    # the Dyson inverse's ~100 small products per frequency are timed in a
    # separate sweep below (events around each would slow the region down)
    _lib.gemm_timing(True, families=False)
    n0 = _lib.launch_count()
    barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.window(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        res_mixed = sweep('mixed')
    e1.record()
    torch.cuda.synchronize()
    if clocks:
        clocks.window(False)
    barrier()
    launches = _lib.launch_count() - n0
    kern = _lib.gemm_timing(False, read=True)
    clk = clocks.stop() if clocks else None
    ms_step = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    # the Dyson inverse's products as a family, one more sweep (untimed)
    _lib.gemm_timing(True)
    sweep('mixed')
    fam = _lib.gemm_timing(False, read=True).get('dyson_tf32')

    # per-stage device times (outside the timed region): the minimum of each
    # stage over two sweeps, which drops a stage that met a clock dip
    def stage_times(precision, warm):
        best = {}
        for _ in range(2):
            t = {}
            gw_sweep(X, D, eps, NOCC, states=states, axes=axes, precision=precision,
                     timings=t, warm=warm)
            for k, v in t.items():
                if k.startswith('t_'):
                    best[k] = min(best.get(k, v), v)
        return best

    stages = stage_times('mixed', model)

    # ---- the plain FP64 GPU sweep (the >= 5x denominator) ----
    stages_fp64 = stage_times('fp64', None)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nf = max(1, min(2, args.steps))
    f0.record()
    for _ in range(nf):
        res_fp64 = sweep('fp64')
    f1.record()
    torch.cuda.synchronize()
    ms_fp64 = max_over_ranks(f0.elapsed_time(f1) / nf)
    acc = accuracy(res_mixed, res_fp64)
    # the warm start checked against the plain scan on the same (mixed) Sigma
    r_plain, _, _, e_plain = qp_solve(res_mixed['sigma'], axes.pade_freq, eps, states, NOCC,
                                      axes.mu)
    ok = torch.isfinite(r_plain) & torch.isfinite(res_mixed['roots'])
    warm_info = {
        'accepted': int(((res_mixed['flags'] & 16) != 0).sum().item()), 'states': N_ORB,
        'sigma_evals_warm': int(res_mixed['evals'].sum().item()),
        'sigma_evals_plain': int(e_plain.sum().item()),
        'max_root_diff_meV': float((res_mixed['roots'] - r_plain)[ok].abs().max().item()
                                   * HARTREE_EV * 1e3)}

    other = None
    if not args.no_accuracy_other:
        ov = 'calibrated' if args.variant == 'literal' else 'literal'
        Xo, Do, eo = synthetic_system_torch(N_ORB, NOCC, M, seed=SEED + 1, variant=ov,
                                            device=dev)
        eo_h = eo.cpu().numpy()
        ax_o = grids.space_time_axes(eo_h, NOCC, ntau=NTAU)
        rm = gw_sweep(Xo, Do, eo_h, NOCC, states=states, axes=ax_o, precision='mixed',
                      warm=model)
        rf = gw_sweep(Xo, Do, eo_h, NOCC, states=states, axes=ax_o, precision='fp64')
        other = dict(variant=ov, **accuracy(rm, rf))
        del Xo, Do, rm, rf

    # ---- e2e: the public call on host inputs (pinned), roots back to the host ----
    Xh = X.cpu().pin_memory()
    Dh = D.cpu().pin_memory()
    eh = eps_t.cpu().pin_memory()
    gw_space_time(Xh, Dh, eh, NOCC, ntau=NTAU, precision='mixed', warm=model)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        gw_space_time(Xh, Dh, eh, NOCC, ntau=NTAU, precision='mixed', warm=model)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)
    h2d = Xh.numel() * 8 + Dh.numel() * 8 + eh.numel() * 8
    d2h = N_ORB * 8

    # ---- roofline of the dominant engine kernel (live CUDA-event timing) ----
    pk, pk_kind = peaks()
    # the dominant single-shape engine kernel; the Dyson inverse's products
    # (about a hundred shapes per frequency, on a second stream) are reported
    # as a family in `kernels`, rated on their summed time
    fixed = {k: v for k, v in kern.items() if k in FLOPS}
    top, (top_ms, top_n) = max(fixed.items(), key=lambda kv: kv[1][0]) if fixed else ('', (0, 0))
    peak = float(pk.get('bf16_tflops_sustained', pk.get('bf16_tflops')))
    def alg_tflops(k, ms, n):
        return FLOPS.get(k, 0.0) / (ms / max(n, 1) / 1e3) / 1e12

    achieved = alg_tflops(top, top_ms, top_n) if top_n else None
    kernels = {k: {'launches': n, 'total_ms': round(ms, 3),
                   'avg_ms': round(ms / max(n, 1), 4),
                   'tflops_alg': round(alg_tflops(k, ms, n), 1)}
               for k, (ms, n) in kern.items()}
    if fam:
        ms, n = fam
        kernels['dyson_tf32'] = {
            'launches': n, 'total_ms': round(ms, 3), 'avg_ms': round(ms / max(n, 1), 4),
            'tflops_alg': round(DYSON_INV_FLOPS * NTAU / (ms / 1e3) / 1e12, 1),
            'note': 'one sweep outside the timed region; summed over the family'}
    traffic = TRAFFIC_BYTES.get(top)

    cpu = None
    if rank == 0 and not args.no_cpu:
        Xn, Dn = X.cpu().numpy(), D.cpu().numpy()
        val, cores, sample_s, blas = cpu_sample(Xn, Dn, eps, axes)
        cpu = {'value': round(val, 3), 'unit': 's', 'cores': cores, 'kind': 'port',
               'sample': (f'one tau point of chi0, one Dyson frequency, one tau point of '
                          f'Sigma (1200 states) and 20 QP solves of this workload, '
                          f'{sample_s:.1f} s of CPU work, scaled to one sweep; BLAS: '
                          f'{"; ".join(blas)}')}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    s_step = ms_step / 1e3
    # whole-job aggregate: N replicas each finish a sweep per s_step (max over
    # ranks), so the job's seconds per sweep are s_step / N (N = 1: s_step)
    line = {
        'metric': METRIC, 'value': round(s_step / world, 5), 'unit': 's', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': round(ms_step, 3),
        'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'bf16x3 split products, fp32 accumulate; fp64 transforms, Cholesky, '
                 'quadrature sums and QP',
        'data': 'synthetic (seeded ISDF factors; no dataset exists for this path)',
        'config': {'workload': 'precision configuration: n_orb=1200, nocc=120, N_mu=7200, '
                               '24 tau/omega points, Sigma + QP of all 1200 states',
                   'variant': args.variant, 'n_orb': N_ORB, 'nocc': NOCC, 'N_mu': M,
                   'ntau': NTAU, 'states': N_ORB,
                   'l2': 'inputs larger than L2 (D alone is 415 MB)',
                   'parallelism': f'replicas x{world}'},
        'sweeps_per_s': round(world / s_step, 4),
        'per_replica_s_per_sweep': round(s_step, 5),
        'fp64_s_per_sweep': round(ms_fp64 / 1e3, 5),
        'speedup_vs_fp64': round(ms_fp64 / ms_step, 3),
        'stages_s': {k: round(v, 4) for k, v in stages.items() if k.startswith('t_')},
        'stages_fp64_s': {k: round(v, 4) for k, v in stages_fp64.items() if k.startswith('t_')},
        'accuracy': acc, 'accuracy_other_variant': other, 'qp_warm_start': warm_info,
        'e2e': {'value': round(e2e_s / world, 5), 'unit': 's', 'h2d_bytes_per_step': int(h2d),
                'd2h_bytes_per_step': int(d2h)},
        'gpu_launches': int(launches),
        'kernels': kernels,
        'roofline': {'bound': 'tensor', 'kernel': top,
                     'achieved': None if achieved is None else round(achieved, 1),
                     'peak': peak, 'unit': 'TFLOP/s',
                     'frac': None if achieved is None else round(achieved / peak, 4),
                     'tensor_pipe_frac': None if achieved is None else round(3 * achieved / peak, 4),
                     'peak_source': f'{pk_kind} bf16 sustained (kernel timed inside a long step)',
                     'traffic': traffic},
        'clocks': clk,
        'cpu_baseline': cpu,
    }
    print(json.dumps(line))


def reference_arm(args, world, rank):
    """The reference's algorithm on the host cores: one whole sweep timed
    once gives the line's value (seconds per sweep); the K steps are bounded
    samples of the same workload (one tau point of chi0, one Dyson frequency,
    one tau point of Sigma, 20 QP solves), each extrapolated to a sweep and
    reported beside it with its error; ms_per_step is a sample's duration."""
    if rank != 0:
        return
    from mbptcode_b200 import grids
    from mbptcode_b200.synthetic import synthetic_system
    X, D, eps = synthetic_system(N_ORB, NOCC, M, seed=SEED, variant=args.variant)
    axes = grids.space_time_axes(eps, NOCC, ntau=NTAU)
    whole_s, whole_stages, cores = cpu_whole_sweep(X, D, eps, axes)
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_sample(X, D, eps, axes)
    vals, durations = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        v, cores, sample_s, blas = cpu_sample(X, D, eps, axes)
        durations.append(time.perf_counter() - t0)
        vals.append(v)
    estimate = float(np.mean(vals))
    sample = (f'value: one whole sweep of this workload timed once ({whole_s:.1f} s: chi0 '
              f'at 24 frequencies, E_c, 24 Dyson inversions, W(tau), the Sigma diagonal and '
              f'QP roots of all 1200 states); steps: {args.steps} bounded samples (one tau '
              f'point of chi0, one Dyson frequency, one tau point of Sigma, 20 QP solves, '
              f'{sample_s:.1f} s each), each scaled to a sweep; NumPy oracle of the '
              f'reference algorithm; BLAS: {"; ".join(blas)}')
    print(json.dumps({
        'impl': 'reference', 'metric': METRIC, 'value': round(whole_s, 3), 'unit': 's',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': round(float(np.mean(durations)) * 1e3, 1), 'higher_is_better': False,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': 'precision configuration: n_orb=1200, nocc=120, N_mu=7200, '
                               '24 tau/omega points, Sigma + QP of all 1200 states',
                   'variant': args.variant, 'n_orb': N_ORB, 'nocc': NOCC, 'N_mu': M,
                   'ntau': NTAU, 'states': N_ORB},
        'whole_sweep_s': round(whole_s, 3), 'whole_sweep_stages_s': whole_stages,
        'sampled_estimate_s': round(estimate, 3),
        'sampled_estimate_error': round(estimate / whole_s - 1.0, 4),
        'cpu_baseline': {'value': round(whole_s, 3), 'unit': 's', 'cores': cores,
                         'kind': 'port', 'sample': sample},
        'e2e': {'value': round(whole_s, 3), 'unit': 's', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0}}))

if __name__ == '__main__':
    main()
