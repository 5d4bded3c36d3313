"""Swap the device route into an MBPTcode checkout.

MBPTcode has no plugin registry: its kernels are module-level functions that
importing modules bind by name (``GW/space_time.py:66-79``,
``GW/imaginary_time.py:33-36``, ``gradients/rpa/space_time_adjoint.py:84-87``;
the static screening in ``BSE/solve.py:70``, ``GW/contour_deformation.py:104``,
``gradients/gwbse/reaction_field_adjoint.py:33``; the contour's explicit
residue backend in ``GW/real_screening.py:57`` and
``GW/contour_deformation.py:96``; the evGW loop, which ``GW/qp_energy.py:242``
reaches as ``evGW.evgw_eigenvalues``),
and its own tests substitute them with ``monkeypatch.setattr(module, name,
...)`` (``tests/test_rpa_log_determinant.py:57-72``). `install()` does the
same for every module that holds one of the names, so every caller --
``solve_qp_energy_space_time``, ``calc_qp_energy(mode='space-time')``,
``evgw_eigenvalues``, ``RPAGroundStateChain`` -- reaches the B200 kernels;
`uninstall()` puts the originals back. Modules that cannot be imported (the
drivers need pyscf) are skipped and reported.
"""
from __future__ import annotations

import importlib

import numpy as np

from . import adjoint, contour, evgw, gw, space_time

LR = 'src.SingleReference.LinearResponse.space_time'
IT = 'src.SingleReference.GW.imaginary_time'
ST = 'src.SingleReference.GW.space_time'
ADJ = 'src.gradients.rpa.space_time_adjoint'
QS = 'src.SingleReference.GW.qp_solve'
QG = 'src.gradients.gwbse.qp_space_time'
# importers of the static screening W(omega = 0)
BSE = 'src.SingleReference.BSE.solve'
CD = 'src.SingleReference.GW.contour_deformation'
RF = 'src.gradients.gwbse.reaction_field_adjoint'
RS = 'src.SingleReference.GW.real_screening'
EV = 'src.SingleReference.GW.evGW'

_SAVED: dict = {}


def _sigma_mo_diagonal(X_mo, D, W_omega, mf, eps, nocc, tau_points, freq_points, pade_freq,
                       mu, p_state, Wt_tau=None, tau_indices=None, reduce_over=None,
                       X_ao=None, coords=None, screen_r_cut=None, block_memory_gb=None,
                       mo_coeff=None, ranges=None):
    """``GW/space_time.py:501-532``: Sigma_c(i w) on the p_state diagonal,
    (nstates, nfreq) (a bare (nfreq,) for a scalar state). The MO diagonal
    of the AO build equals the diagonal contraction with the MO collocation
    X_mo = X_ao C, which the device sweep forms directly."""
    if reduce_over is not None or tau_indices is not None or screen_r_cut:
        raise NotImplementedError('rank splits and distance screening are outside the '
                                  'one-GPU route')
    from .grids import COSINE_TW, COSINE_WT, SINE_TW, sigma_fit_ranges, transform_weights
    states = np.atleast_1d(p_state)
    rW, rS = ranges or sigma_fit_ranges(eps, nocc, mu=mu)
    if Wt_tau is None:
        Ctw, _ = transform_weights(COSINE_WT, tau_points, freq_points, *rW, warn=False)
        Wm = space_time.to_device(W_omega, space_time.require_device()).clone()
        Wm.diagonal(dim1=-2, dim2=-1).sub_(1.0)
        Wt = gw.w_tau_from_frequencies(Wm, Ctw)
    else:
        Wt = Wt_tau
    C, _ = transform_weights(COSINE_TW, tau_points, pade_freq, *rS, warn=False)
    S, _ = transform_weights(SINE_TW, tau_points, pade_freq, *rS, warn=False)
    br = gw.sigma_branch_sums(X_mo, D, Wt, eps, nocc, tau_points, states, mu)
    sigma = gw.sigma_frequency(br, C, S).cpu().numpy()
    return sigma[0] if np.ndim(p_state) == 0 else sigma


def replacements():
    """{module: {name: replacement}} of the drop-in."""
    seams = {
        'chi0_imaginary_frequency': space_time.chi0_imaginary_frequency,
        'polarizability_projected_sweep': space_time.polarizability_projected_sweep,
        'polarizability_projected_tau': space_time.polarizability_projected_tau,
        'dyson_screening': space_time.dyson_screening,
        'dielectric_log_determinant': space_time.dielectric_log_determinant,
        'rpa_correlation_energy_space_time': space_time.rpa_correlation_energy_space_time,
        'static_screening_matrix': space_time.static_screening_matrix,
        'static_screening_matrix_unrestricted': space_time.static_screening_matrix_unrestricted,
    }
    static = {k: seams[k] for k in ('static_screening_matrix',
                                    'static_screening_matrix_unrestricted')}
    return {
        LR: dict(seams),
        IT: {**{k: v for k, v in seams.items()
                if k in ('dyson_screening', 'polarizability_projected_sweep',
                         'polarizability_projected_tau')},
             'selfenergy_diag': adjoint.selfenergy_diag,
             'self_energy_matrix_imaginary_time': gw.self_energy_matrix_imaginary_time,
             'sigma_ao_to_mo_diagonal': gw.sigma_ao_to_mo_diagonal,
             'screened_interaction_tau': gw.screened_interaction_tau,
             '_transform_screened': gw._transform_screened},
        ST: {'chi0_imaginary_frequency': space_time.chi0_imaginary_frequency,
             'dyson_screening': space_time.dyson_screening,
             '_sigma_mo_diagonal': _sigma_mo_diagonal, **static},
        QS: {'solve_qp_from_imaginary_axis': gw.solve_qp_from_imaginary_axis,
             'imaginary_axis_sample_points': gw.imaginary_axis_sample_points},
        QG: {'qp_gradient_space_time': contour.qp_gradient_space_time},
        BSE: dict(static),
        CD: {**static,
             'cd_screening_contraction_multi': contour.cd_screening_contraction_multi,
             'ExplicitRealScreening': contour.ExplicitRealScreening,
             'wc_explicit': contour.wc_explicit},
        RS: {'ExplicitRealScreening': contour.ExplicitRealScreening},
        EV: {'evgw_eigenvalues': evgw.evgw_eigenvalues},
        RF: dict(static),
        ADJ: {'polarizability_backward': adjoint.polarizability_backward,
              'selfenergy_diag_backward': adjoint.selfenergy_diag_backward,
              'screened_interaction_tau_backward': adjoint.screened_interaction_tau_backward,
              'rpa_energy_and_adjoint': adjoint.rpa_energy_and_adjoint,
              'rpa_correlation_energy_space_time':
                  space_time.rpa_correlation_energy_space_time,
              'chi0_imaginary_frequency': space_time.chi0_imaginary_frequency},
    }


def install(precision='fp64'):
    """Rebind the names; returns {module: [names]} bound and the modules
    skipped with their import error."""
    space_time.set_default_precision(precision)
    bound, skipped = {}, {}
    for modname, names in replacements().items():
        try:
            mod = importlib.import_module(modname)
        except Exception as exc:  # noqa: BLE001 -- e.g. pyscf absent
            skipped[modname] = f'{type(exc).__name__}: {exc}'
            continue
        for name, fn in names.items():
            if not hasattr(mod, name):
                continue
            _SAVED.setdefault((modname, name), getattr(mod, name))
            setattr(mod, name, fn)
            bound.setdefault(modname, []).append(name)
    return bound, skipped


def uninstall():
    """Restore every name `install` rebound."""
    for (modname, name), fn in list(_SAVED.items()):
        mod = importlib.import_module(modname)
        setattr(mod, name, fn)
        del _SAVED[(modname, name)]
