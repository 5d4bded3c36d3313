"""The drop-in, call by call: every seam call that MBPTcode's own drivers made
on a synthetic system (its G0W0 driver ``GW/space_time.py:631-863``, its dRPA
energy ``LinearResponse/space_time.py:1100-1183`` and adjoint
``gradients/rpa/space_time_adjoint.py:473-563``), recorded with its
arguments and result by tests/golden/make_golden.py (--only drop_in), is
replayed here through the function `plugin.install()` binds under that name
in that module, with the same positional and keyword arguments, and its
result compared with what the reference's own function returned.

The reference is Python and is not present where this runs; the recording
is what carries its calls here. Arguments the recording cannot carry (a
scratch buffer the reference passes to reuse, the mean-field object the
device seam does not read) are passed as None."""
import json
from types import SimpleNamespace

import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from mbptcode_b200 import plugin                                    # noqa: E402

GRID_FIELDS = ('tau_points', 'tau_weights', 'omega_points', 'omega_weights', 'cosft_wt')

# tolerance per seam: FP64 device arithmetic against NumPy/LAPACK, 1e-9
# relative. The G0W0 driver sizes its grid itself (16 points here), whose
# unregularised transform weights reach 3e8 and turn FP64 summation-order
# differences into ~1e-7 relative on what passes through a transform (chi0,
# W(i w) from that chi0, W(tau), Sigma); a QP root of a state far from the
# gap carries the Pade continuation's amplification
TOL = {'solve_qp_from_imaginary_axis': 1e-6, 'chi0_imaginary_frequency': 1e-6,
       'dyson_screening': 1e-6, '_transform_screened': 1e-6, '_sigma_mo_diagonal': 1e-6}


def _decode(desc, g):
    if 'array' in desc:
        return np.array(g[desc['array']])
    if 'grid' in desc:
        f = {k: np.array(g[f"{desc['grid']}_{k}"]) for k in GRID_FIELDS}
        return SimpleNamespace(**f, nfreq=len(f['omega_points']), ntau=len(f['tau_points']))
    if 'opaque' in desc:
        return None
    return desc['value']


def _host(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return x


def test_recorded_reference_calls_replay_through_the_device_seams(golden):
    g = golden('drop_in')
    calls = json.loads(str(g['calls']))
    table = plugin.replacements()
    checked = {}
    for c in calls:
        fn = table[c['module']][c['name']]
        args = [_decode(a, g) for a in c['args']]
        kwargs = {k: _decode(v, g) for k, v in c['kwargs'].items()}
        out = fn(*args, **kwargs)
        got = out if c['result_tuple'] else (out,)
        want = [_decode(r, g) for r in c['result']]
        tol = TOL.get(c['name'], 1e-9)
        for j, (a, b) in enumerate(zip(got, want)):
            if b is None:
                continue
            a = np.asarray(_host(a))
            b = np.asarray(b)
            assert a.shape == b.shape, (c['name'], j, a.shape, b.shape)
            scale = max(float(np.abs(b).max()), 1e-300) if b.size else 1.0
            err = float(np.abs(a - b).max()) / scale if b.size else 0.0
            assert err < tol, (c['module'], c['name'], j, err)
        checked[c['name']] = checked.get(c['name'], 0) + 1
    # every kind of seam the drivers reach was replayed
    assert {'chi0_imaginary_frequency', 'dyson_screening', '_transform_screened',
            '_sigma_mo_diagonal', 'solve_qp_from_imaginary_axis', 'dielectric_log_determinant',
            'polarizability_projected_sweep', 'polarizability_backward',
            'rpa_correlation_energy_space_time', 'rpa_energy_and_adjoint'} <= set(checked)
