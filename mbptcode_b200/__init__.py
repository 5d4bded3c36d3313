"""mbptcode_b200: MBPTcode's space-time ISDF RPA/GW route on NVIDIA B200.

The route -- G(tau) on the interpolation points, chi0(tau), the minimax
tau <-> omega transforms, W(i omega) by a per-frequency Cholesky (with the
RPA log-determinant), W(tau), the correlation self-energy and the
quasiparticle roots -- runs in libmbpt_b200.so (hand-written sm_100a CUDA
behind the C ABI of include/mbpt_b200.h). This package is the host side: the
imaginary-axis grids (FP64, tiny) and Python entry points with the names and
arguments of MBPTcode's own (see `plugin.install` for swapping them into an
MBPTcode checkout).
"""
from .space_time import (chi0_imaginary_frequency, dielectric_log_determinant,   # noqa: F401
                         dyson_screening, polarizability_projected_sweep,
                         polarizability_projected_tau, rpa_correlation_energy_space_time,
                         set_default_precision, split_branches)
from .gw import (gw_space_time, gw_sweep, solve_qp_diagonal_space_time,         # noqa: F401
                 solve_qp_energy_space_time)
from .grids import TimeFrequencyGrid, space_time_axes                           # noqa: F401

__version__ = '0.1.0'
