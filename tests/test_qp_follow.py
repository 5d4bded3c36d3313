"""Root following on the scan against the reference's own scan
(`tests/golden/qp_follow.npz`, made by `make_golden.py --only follow`): on
seeded pole-sum self-energies, the root, its Z and the branch record (the
root of largest weight beside it, whether the previous root's branch
continued, whether the largest weight has left it, no root, Z outside
(0, 1]) that `contour.solve_qp_equation_scan` hands to `out`, for followed
points beside each root, between roots and outside every window, with the
largest-weight rescan on and off, and positive_weight on and off. Host
callables: no device needed. Roots to 1e-10, Z to 1e-9."""
import os
import warnings

import numpy as np
import pytest

from mbptcode_b200 import contour

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def _model(a, pol, amp):
    pol, amp = pol[np.isfinite(pol)], amp[:np.isfinite(pol).sum()]

    def f(w):
        return w - a - float(np.sum(amp / (w - pol)))

    def fp(w):
        return 1.0 + float(np.sum(amp / (w - pol) ** 2))
    return f, fp


@pytest.fixture(scope='module')
def fixture():
    return np.load(os.path.join(HERE, 'qp_follow.npz'))


def test_followed_roots_and_branches_match_the_reference(fixture):
    g = fixture
    col = {c: i for i, c in enumerate(g['columns'])}
    for row in g['cases']:
        m = int(row[col['model']])
        a = float(g['a'][m])
        f, fp = _model(a, g['poles'][m], g['amps'][m])
        t = None if np.isnan(row[col['follow']]) else float(row[col['follow']])
        out = {}
        with warnings.catch_warnings():
            warnings.simplefilter('ignore')
            w, z = contour.solve_qp_equation_scan(f, fp, a, follow=t, out=out,
                                                  positive_weight=bool(g['positive'][m]),
                                                  rescan=bool(row[col['rescan']]))
        where = (m, t, bool(row[col['rescan']]))
        assert abs(w - row[col['w']]) < 1e-10 and abs(z - row[col['z']]) < 1e-9, where
        followed = {None: -1.0, False: 0.0, True: 1.0}[out['followed']]
        assert followed == row[col['followed']], where
        assert float(out['flipped']) == row[col['flipped']], where
        assert float(out['no_root']) == row[col['no_root']], where
        assert float(out['z_outside']) == row[col['z_outside']], where
        lg = out['largest']
        if np.isnan(row[col['largest_w']]):
            assert lg is None, where
        else:
            assert abs(lg[0] - row[col['largest_w']]) < 1e-10, where
            assert abs(lg[1] - row[col['largest_z']]) < 1e-9, where


def test_a_weak_followed_root_warns_without_an_out_dict(fixture):
    """Without `out`, a followed root that the largest weight has left is
    kept with a RuntimeWarning naming both."""
    g = fixture
    col = {c: i for i, c in enumerate(g['columns'])}
    rows = [r for r in g['cases'] if r[col['flipped']] == 1.0 and r[col['followed']] == 1.0]
    assert rows
    r = rows[0]
    m = int(r[col['model']])
    f, fp = _model(float(g['a'][m]), g['poles'][m], g['amps'][m])
    with pytest.warns(RuntimeWarning, match='largest weight is now'):
        w, _ = contour.solve_qp_equation_scan(f, fp, float(g['a'][m]),
                                              follow=float(r[col['follow']]),
                                              positive_weight=bool(g['positive'][m]),
                                              rescan=bool(r[col['rescan']]))
    assert abs(w - r[col['w']]) < 1e-10
