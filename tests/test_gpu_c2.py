"""The precision configuration as a test: n_orb = 1200, nocc = 120,
N_mu = 7200, 24 tau/omega points, the whole sweep (chi0, the Dyson step, W,
Sigma and the QP roots of all 1200 states) in mixed precision against the
plain FP64 device sweep, on both generators.

Bars: the 20 HOMO/LUMO-region QP energies within 10 meV and E_c within
1 uHa per electron (240 electrons). The states outside that window whose
mixed root moves by more than 10 meV are reported with their pole strength
Z, the distance of their level from the gap and whether the plain root is a
quasiparticle (Z in (1/2, 1]); the test holds every quasiparticle root of
the window and reports the rest."""
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from mbptcode_b200 import grids, gw                                 # noqa: E402
from mbptcode_b200.synthetic import synthetic_system_torch          # noqa: E402

N, NOCC, M, NTAU, SEED = 1200, 120, 7200, 24, 2024
MEV = 27211.386245988


@pytest.mark.parametrize('variant', ['calibrated', 'literal'])
def test_c2_mixed_within_the_precision_bars(variant):
    X, D, eps_t = synthetic_system_torch(N, NOCC, M, seed=SEED, variant=variant)
    eps = eps_t.cpu().numpy()
    axes = grids.space_time_axes(eps, NOCC, ntau=NTAU)
    res = {p: gw.gw_sweep(X, D, eps, NOCC, axes=axes, precision=p) for p in ('fp64', 'mixed')}
    r64, rmx = (res[p]['roots'].cpu().numpy() for p in ('fp64', 'mixed'))
    z64 = res['fp64']['z'].cpu().numpy()
    f = np.arange(NOCC - 10, NOCC + 10)
    err = np.abs(rmx - r64) * MEV
    e64, emx = (float(res[p]['e_c']) for p in ('fp64', 'mixed'))
    gap_lo, gap_hi = eps[NOCC - 1], eps[NOCC]
    far = [{'state': int(p), 'err_meV': round(float(err[p]), 3), 'z_fp64': round(float(z64[p]), 5),
            'eps_Ha': round(float(eps[p]), 5),
            'depth_Ha': round(float(max(gap_lo - eps[p], eps[p] - gap_hi, 0.0)), 5)}
           for p in np.nonzero(err > 10.0)[0]]
    report = {'variant': variant, 'e_c_fp64_Ha': e64,
              'e_c_err_uHa_per_e': abs(emx - e64) * 1e6 / (2 * NOCC),
              'frontier_err_meV_max': float(err[f].max()),
              'frontier_err_meV_mean': float(err[f].mean()),
              'all_err_meV_max': float(np.nanmax(err)),
              'states_over_10meV': far}
    print(json.dumps(report))
    where = os.environ.get('MBPT_TEST_REPORTS')
    if where:
        os.makedirs(where, exist_ok=True)
        with open(os.path.join(where, f'c2_accuracy_{variant}.json'), 'w') as fh:
            json.dump(report, fh, indent=1)
    assert np.isfinite(r64[f]).all() and np.isfinite(rmx[f]).all()
    assert err[f].max() < 10.0, report
    assert abs(emx - e64) < 1e-6 * 2 * NOCC, report
