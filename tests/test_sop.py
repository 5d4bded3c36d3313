"""The contour's pole model (continuation 'sop', `mbptcode_b200.sum_over_poles`)
against the reference's own (`tests/golden/sop.npz`, made by
`make_golden.py --only sop`): on the contour system's screening contraction,
the fitted poles and amplitudes (12 poles at the default stride, 8 at stride
1, 12 log-spaced unfitted), Sigma and its slope, the quasiparticle roots
with Z and the roots followed along labelled and unlabelled branches, the
compression test; and the pole-sum root finder on seeded sums of positive
and of mixed-sign weights (coinciding poles among them), unfollowed and
following. Host algebra: no device needed. Poles to 1e-10 relative, roots
to 1e-10, Z to 1e-9."""
import os
import warnings

import numpy as np
import pytest

from mbptcode_b200 import sum_over_poles as sop

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


@pytest.fixture(scope='module')
def g():
    return np.load(os.path.join(HERE, 'sop.npz'))


@pytest.fixture(scope='module')
def c():
    return np.load(os.path.join(HERE, 'contour.npz'))


@pytest.mark.parametrize('tag,kw', [('fit12', {}), ('fit8s1', dict(n_poles=8, stride=1)),
                                    ('log12', dict(relocate=False))])
def test_pole_model_matches_reference(g, c, tag, kw):
    eps, nocc, nu = c['eps'], int(c['nocc']), c['nu']
    for i, p in enumerate(c['states']):
        poles, amp = sop.sop_from_wc(c['wc'][i], nu, eps, nocc, **kw)
        ref = g[f'{tag}_poles'][i]
        ref = ref[np.isfinite(ref)]
        assert poles.shape == ref.shape, (tag, p)
        assert np.abs(poles - ref).max() <= 1e-10 * ref.max(), (tag, p)
        ra = g[f'{tag}_amps'][i][:len(ref)]
        assert np.abs(amp - ra).max() <= 1e-8 * np.abs(ra).max(), (tag, p)
        for j, d in enumerate(g['shifts']):
            s = sop.sigma_sop(eps[p] + d, amp, poles, eps, nocc, check=False)
            assert abs(s - g[f'{tag}_sigma'][i, j]) <= 1e-10, (tag, p, d)
            ds = sop.sigma_sop_slope(eps[p] + d, amp, poles, eps, nocc)
            assert abs(ds - g[f'{tag}_slope'][i, j]) <= 1e-9 * max(1.0, abs(ds)), (tag, p, d)
        br = {}
        w, z = sop.qp_energy_sop(int(p), amp, poles, eps, nocc, branch=br)
        assert abs(w - g[f'{tag}_roots'][i, 0]) < 1e-10 and abs(z - g[f'{tag}_roots'][i, 1]) < 1e-9
        rows = [r for r in g[f'{tag}_follow'] if int(r[0]) == i]
        lab = br['labels']
        for r, follow in zip(rows, ((w + 2e-3, lab), (w + 2e-3, None), (w, (lab[0], None)),
                                    (w - 0.3, None))):
            b2 = {}
            with warnings.catch_warnings():
                warnings.simplefilter('ignore')
                w2, z2 = sop.qp_energy_sop(int(p), amp, poles, eps, nocc, follow=follow,
                                           branch=b2)
            assert abs(w2 - r[3]) < 1e-10 and abs(z2 - r[4]) < 1e-9, (tag, p, follow)
            assert {None: -1.0, False: 0.0, True: 1.0}[b2['followed']] == r[6], (tag, p)
            assert float(b2['flipped']) == r[7], (tag, p, follow)
            if not np.isnan(r[5]):
                assert abs(b2['largest'][0] - r[5]) < 1e-10


def test_compression_test_matches_reference(g, c):
    eps, nocc = c['eps'], int(c['nocc'])
    starts = [sop.qp_start(eps, int(p), nocc) for p in c['states']]
    assert np.allclose(starts, g['starts'], rtol=0, atol=0)
    for i, w in enumerate(starts):
        ok, reach = sop.compressible(w, eps, nocc)
        assert ok == bool(g['admits'][i]) and abs(reach - g['reach'][i]) < 1e-14


def test_pole_sum_finder_matches_reference(g):
    """Unfollowed (the root of largest valid weight and the labels of its
    interval) and following an unlabelled point (the interval holding it)."""
    for row in g['sum_cases']:
        if row[2] != -2:
            continue                      # labelled follows: the next test
        k = int(row[0])
        pol = g['sum_poles'][k]
        n = int(np.isfinite(pol).sum())
        pol, num, a = pol[:n], g['sum_nums'][k][:n], float(g['sum_a'][k])
        follow = None if np.isnan(row[1]) else (float(row[1]), None)
        b = {}
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            w, z = sop.solve_qp_equation_poles(num, pol, a, follow=follow, out=b)
        where = (k, row[1])
        assert abs(w - row[3]) < 1e-10 and abs(z - row[4]) < 1e-9, where
        assert {None: -1.0, False: 0.0, True: 1.0}[b['followed']] == row[6], where
        assert float(b['flipped']) == row[7], where
        lab = b['labels']
        assert (np.isnan(row[8]) if lab[0] is None else lab[0] == row[8]), where
        assert (np.isnan(row[9]) if lab[1] is None else lab[1] == row[9]), where


def test_pole_sum_finder_follows_labelled_branches(g):
    """Following the kept root's own branch, named by the labels of the two
    poles that bound it, from 1e-3 away: the reference's root and record."""
    rows = {}
    for row in g['sum_cases']:
        rows.setdefault(int(row[0]), []).append(row)
    checked = 0
    for k, rs in rows.items():
        base = rs[0]
        lab = (None if np.isnan(base[8]) else int(base[8]),
               None if np.isnan(base[9]) else int(base[9]))
        for row in rs[1:]:
            if row[2] != 0:
                continue
            pol = g['sum_poles'][k]
            n = int(np.isfinite(pol).sum())
            b = {}
            with warnings.catch_warnings():
                warnings.simplefilter('ignore')
                w, z = sop.solve_qp_equation_poles(g['sum_nums'][k][:n], pol[:n],
                                                   float(g['sum_a'][k]),
                                                   follow=(float(row[1]), lab), out=b)
            assert abs(w - row[3]) < 1e-10 and abs(z - row[4]) < 1e-9, k
            assert {None: -1.0, False: 0.0, True: 1.0}[b['followed']] == row[6], k
            assert float(b['flipped']) == row[7], k
            checked += 1
    assert checked >= 30
