"""Host-side logic on the CPU: DIIS, the mixed-precision refusal, the MLP
oracle's own gradient, and the replica plumbing over two gloo ranks."""
import os

import numpy as np
import pytest


def test_diis_matches_oracle_and_accelerates():
    from mbptcode_b200.evgw import DIIS
    from oracle.st_oracle import PulayDIIS
    rng = np.random.default_rng(0)
    A = np.eye(6) * 0.6 + 0.05 * rng.standard_normal((6, 6))
    b = rng.standard_normal(6)
    fix = np.linalg.solve(np.eye(6) - A, b)

    def run(acc, steps=25):
        x = np.zeros(6)
        for _ in range(steps):
            xn = A @ x + b
            x = acc.update(xn, xn - x) if acc is not None else xn
        return x
    d, o = run(DIIS(8, 2)), run(PulayDIIS(8, 2))
    assert np.allclose(d, o, rtol=1e-10, atol=1e-12)
    assert np.abs(d - fix).max() < 1e-8
    assert np.abs(run(DIIS(8, 2), 10) - fix).max() < np.abs(run(None, 10) - fix).max()


def test_mixed_precision_refuses_ill_conditioned_weights():
    from mbptcode_b200 import space_time as st
    st.check_mixed_weights('mixed', np.ones((3, 3)) * 40.0)
    st.check_mixed_weights('fp64', np.ones((3, 3)) * 1e9)
    with pytest.raises(ValueError, match='mixed precision'):
        st.check_mixed_weights('mixed', np.ones((3, 3)) * 1e9)
    with pytest.raises(ValueError):
        st.set_default_precision('fp16')


def test_mlp_oracle_gradient_by_finite_differences():
    from oracle import mlp_oracle as mo
    H = 8
    rng = np.random.default_rng(2)
    p = rng.standard_normal(H * H + 7 * H + 1) * 0.3
    x, t = rng.standard_normal((20, 4)), rng.standard_normal(20)
    _, g = mo.loss_and_grad(p, H, x, t)
    h = 1e-6
    for k in rng.choice(len(p), 12, replace=False):
        e = np.zeros_like(p)
        e[k] = h
        fd = (mo.loss_and_grad(p + e, H, x, t)[0] - mo.loss_and_grad(p - e, H, x, t)[0]) / (2 * h)
        assert abs(fd - g[k]) < 1e-7 + 1e-6 * abs(fd)


def test_grid_axes_of_the_precision_configuration():
    # n_orb = 1200 spectra: 24 points, regularised fits, moderate weights
    from mbptcode_b200 import grids
    rng = np.random.default_rng(1)
    eps = np.concatenate([np.sort(rng.uniform(-1.5, -0.3, 120)),
                          np.sort(np.exp(rng.uniform(np.log(0.05), np.log(5), 1080)))])
    axes = grids.space_time_axes(eps, 120, ntau=24)
    assert axes.grid.cosft_wt.shape == (24, 24) and axes.C.shape == (16, 24)
    assert max(np.abs(w).max() for w in (axes.grid.cosft_wt, axes.Ctw, axes.C, axes.S)) < 1e3


def _replica_worker(rank, world, port, out):
    import torch.distributed as dist
    from mbptcode_b200 import replicas
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        mine = replicas.shard(7, rank, world)
        t = replicas.max_over_ranks(1.5 + rank)
        all_shards = replicas.gather(mine)
        out.put((rank, mine, t, all_shards))
    finally:
        dist.destroy_process_group()


def test_replicas_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, g0), (r1, m1, t1, g1) = res
    assert m0 == [0, 2, 4, 6] and m1 == [1, 3, 5]
    assert t0 == t1 == 2.5
    assert g0 == g1 == [[0, 2, 4, 6], [1, 3, 5]]


def test_plugin_rebinds_and_restores_reference_names():
    ref = os.environ.get('MBPTCODE_ROOT', '/root/reference')
    if not os.path.isdir(os.path.join(ref, 'src')):
        pytest.skip('no MBPTcode checkout here')
    import sys
    sys.path.insert(0, ref)
    try:
        import importlib
        from mbptcode_b200 import plugin, space_time
        lr = importlib.import_module(plugin.LR)
        orig = lr.chi0_imaginary_frequency
        bound, skipped = plugin.install()
        assert lr.chi0_imaginary_frequency is space_time.chi0_imaginary_frequency
        assert lr.static_screening_matrix is space_time.static_screening_matrix
        it = importlib.import_module(plugin.IT)
        from mbptcode_b200 import adjoint as adj_mod
        assert it.selfenergy_diag is adj_mod.selfenergy_diag
        # the static screening's other importers need pyscf, absent here
        assert {plugin.BSE, plugin.CD, plugin.RF} <= set(skipped)
        assert 'dyson_screening' in bound[plugin.IT]
        from mbptcode_b200 import contour
        rs = importlib.import_module(plugin.RS)
        assert rs.ExplicitRealScreening is contour.ExplicitRealScreening
        assert plugin.ST in skipped      # MBPTcode's GW module imports pyscf, absent here
        adj = importlib.import_module(plugin.ADJ)
        assert adj.rpa_correlation_energy_space_time is \
            space_time.rpa_correlation_energy_space_time
        plugin.uninstall()
        assert lr.chi0_imaginary_frequency is orig
    finally:
        sys.path.remove(ref)


def test_shipped_qp_shift_model_file():
    """The trained warm-start network ships with the package: a 4 -> 64 -> 64 -> 1
    parameter vector plus its input standardisation and target scale."""
    from mbptcode_b200.qp_mlp import MODEL_PATH
    d = np.load(MODEL_PATH)
    H = int(d['hidden'])
    assert H == 64
    assert d['params'].shape == (4 * H + H + H * H + H + H + 1,)
    assert d['x_mean'].shape == (4,) and d['x_std'].shape == (4,)
    assert np.all(np.isfinite(d['params'])) and float(d['y_scale']) > 0
