"""ctypes binding of libmbpt_b200.so (the C ABI in include/mbpt_b200.h).

The library is loaded from this package directory. There is no fallback: a
missing library or a device that is not sm_100 raises, so no call silently
runs elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import torch

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'libmbpt_b200.so')
_LIB = None
_LOCK = threading.Lock()

MODE_FP64, MODE_MIXED, MODE_FP64_INT8 = 0, 1, 2
MODES = {'fp64': MODE_FP64, 'mixed': MODE_MIXED, 'fp64_int8': MODE_FP64_INT8}

OK, ERR_SHAPE, ERR_NOT_SPD, ERR_NONFINITE, ERR_NO_ROOT, ERR_TIMEOUT, ERR_CUDA, \
    ERR_WORKSPACE, ERR_UNSUPPORTED = range(9)

_p, _i64, _i, _d, _f, _sz = C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_float, C.c_size_t

_SIGNATURES = {
    'mbpt_abi_version': (_i, []),
    'mbpt_status_string': (C.c_char_p, [_i]),
    'mbpt_device_supported': (_i, [_i]),
    'mbpt_launch_count': (C.c_longlong, []),
    'mbpt_gemm_timing': (_i, [_i, _p, _p]),
    'mbpt_wait_selftest': (_i, [_i, _i, _p, _p]),
    'mbpt_energy_sum': (_i, [_p, _p, _p, _i, _p, _p]),
    'mbpt_chi0_workspace_bytes': (_sz, [_i64, _i64, _i64, _i64, _i, _i]),
    'mbpt_chi0_sweep': (_i, [_p, _i64, _i64, _i64, _p, _d, _p, _i64, _p, _i, _p, _i, _i, _p,
                             _p, _p, _sz, _p, _p]),
    'mbpt_dyson_workspace_bytes': (_sz, [_i64, _i, _i]),
    'mbpt_dyson': (_i, [_p, _i64, _i, _i, _i, _p, _p, _p, _p, _p, _sz, _p, _p]),
    'mbpt_dyson_deferred': (_i, [_p, _i64, _i, _i, _i, _p, _p, _p, _p, _sz, _p, _p]),
    'mbpt_rpa_energy_workspace_bytes': (_sz, [_i64, _i64, _i64, _i64, _i, _i, _i]),
    'mbpt_rpa_energy': (_i, [_p, _i64, _i64, _i64, _p, _d, _p, _i64, _p, _i, _p, _p, _i, _i,
                             _p, _p, _p, _p, _sz, _p, _p]),
    'mbpt_transform': (_i, [_p, _i, _i64, _p, _i, _p, _p]),
    'mbpt_transform_acc': (_i, [_p, _i, _i64, _p, _i, _p, _p]),
    'mbpt_sigma_workspace_bytes': (_sz, [_i64, _i64, _i64, _i64, _i, _i, _i]),
    'mbpt_sigma_branch_sums': (_i, [_p, _i64, _i64, _i64, _p, _d, _p, _i64, _p, _p, _i, _p,
                                    _i, _i, _p, _p, _sz, _p, _p]),
    'mbpt_sigma_frequency': (_i, [_p, _i, _i, _p, _p, _i, _p, _p]),
    'mbpt_qp_solve': (_i, [_p, _p, _i, _p, _p, _p, _i, _i64, _d, _i, _p, _p, _p, _p, _p, _p,
                           _sz, _p]),
    'mbpt_pade_eval': (_i, [_p, _p, _i, _p, _i, _i64, _d, _i, _p, _i, _p, _p, _sz, _p]),
    'mbpt_chi0_backward_workspace_bytes': (_sz, [_i64, _i64, _i64, _i64, _i]),
    'mbpt_chi0_backward': (_i, [_p, _p, _i64, _i64, _i64, _p, _d, _p, _i64, _p, _i, _i, _p,
                                _p, _p, _p, _sz, _p, _p]),
    'mbpt_energy_adjoint_seed': (_i, [_p, _i64, _i, _p, _p]),
    'mbpt_sigma_backward_workspace_bytes': (_sz, [_i64, _i64, _i64, _i64, _i]),
    'mbpt_sigma_backward': (_i, [_p, _i64, _i64, _i64, _p, _d, _p, _i64, _p, _i, _p, _p, _i,
                                 _p, _p, _i, _p, _p, _p, _p, _p, _sz, _p, _p]),
    'mbpt_sigma_ao_workspace_bytes': (_sz, [_i64, _i64, _i64, _i64, _i64, _i]),
    'mbpt_sigma_ao': (_i, [_p, _i64, _i64, _p, _i64, _i64, _p, _d, _p, _i64, _p, _p, _i, _i,
                           _p, _p, _sz, _p, _p]),
    'mbpt_three_index_slices_workspace_bytes': (_sz, [_i64, _i64]),
    'mbpt_three_index_slices': (_i, [_p, _i64, _i64, _p, _i64, _p, _i, _p, _p, _sz, _p]),
    'mbpt_chol_solve': (_i, [_p, _i64, _p, _i, _p]),
    'mbpt_cd_integral_terms': (_i, [_p, _i, _i, _i64, _p, _p, _p, _i, _i, _d, _d, _d, _d, _p,
                                    _p, _i64, _p, _p, _p]),
    'mbpt_laplace_representation_error': (_i, [_p, _i64, _p, _p, _i, _p, _i64, _p, _p]),
    'mbpt_chi0_aux_workspace_bytes': (_sz, [_i64, _i64, _i]),
    'mbpt_chi0_aux': (_i, [_p, _i64, _i64, _i64, _p, _d, _i, _i, _p, _p, _sz, _p, _p]),
    'mbpt_screening_contraction_workspace_bytes': (_sz, [_i64, _i64, _i]),
    'mbpt_screening_contraction': (_i, [_p, _i, _i64, _p, _i64, _i, _p, _p, _sz, _p, _p]),
    'mbpt_cd_integral_backward_workspace_bytes': (_sz, [_i64, _i64]),
    'mbpt_cd_integral_backward': (_i, [_p, _i, _i64, _p, _i64, _p, _p, _p, _p, _sz, _p]),
    'mbpt_three_index_slice_backward_workspace_bytes': (_sz, [_i64, _i64, _i64]),
    'mbpt_three_index_slice_backward': (_i, [_p, _i64, _i64, _p, _i64, _i64, _p, _p, _p, _p,
                                             _sz, _p]),
    'mbpt_dyson_backward_workspace_bytes': (_sz, [_i64]),
    'mbpt_dyson_backward': (_i, [_p, _p, _i64, _i, _i, _p, _sz, _p]),
    'mbpt_mlp_param_count': (_i, [_i]),
    'mbpt_mlp_forward': (_i, [_p, _i, _p, _i, _p, _p, _p]),
    'mbpt_mlp_backward': (_i, [_p, _i, _p, _i, _p, _p, _p, _p, _p, _p]),
    'mbpt_mlp_adamw': (_i, [_p, _p, _p, _p, _i, _f, _f, _f, _f, _f, _i, _p]),
    'mbpt_gemm_split_workspace_bytes': (_sz, [_i64, _i64, _i64]),
    'mbpt_gemm_split': (_i, [_p, _p, _i64, _i64, _i64, _d, _p, _i64, _p, _sz, _p, _p]),
    'mbpt_gemm_split_tf32_workspace_bytes': (_sz, [_i64, _i64, _i64]),
    'mbpt_gemm_split_tf32': (_i, [_p, _p, _i64, _i64, _i64, _d, _p, _i64, _p, _sz, _p, _p]),
    'mbpt_dgemm_ozaki_workspace_bytes': (_sz, [_i64, _i64, _i64, _i]),
    'mbpt_dgemm_ozaki': (_i, [_i, _i, _i64, _i64, _i64, _d, _p, _i64, _p, _i64, _d, _p, _i64, _i,
                              _p, _sz, _p, _p]),
    'mbpt_gemm_split_static_capacity': (_sz, []),
    'mbpt_gemm_split_static': (_i, [_p, _p, _i64, _i64, _i64, _d, _p, _i64, _p, _p]),
}


class MBPTError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        super().__init__(f'{where}: {status_string(status)} (status {status})')


def lib():
    global _LIB
    if _LIB is None:
        with _LOCK:
            if _LIB is None:
                if not os.path.exists(_PATH):
                    raise RuntimeError(f'{_PATH} is not built; run python -m mbptcode_b200.build')
                handle = C.CDLL(_PATH)
                for name, (res, args) in _SIGNATURES.items():
                    fn = getattr(handle, name)
                    fn.restype, fn.argtypes = res, args
                _LIB = handle
    return _LIB


def exported_symbols():
    return list(_SIGNATURES)


def status_string(status):
    return lib().mbpt_status_string(int(status)).decode()


def check(status, where):
    if status != OK:
        raise MBPTError(status, where)
    return status


_SUPPORTED = set()  # device indices already checked


def require_device(device=None):
    """The CUDA device the route runs on: an sm_100 part, else an error."""
    if not torch.cuda.is_available():
        raise RuntimeError('mbptcode_b200 needs a CUDA device (sm_100a); none is visible')
    dev = torch.device('cuda', torch.cuda.current_device() if device is None else device)
    if dev.index not in _SUPPORTED:
        if not lib().mbpt_device_supported(dev.index):
            raise RuntimeError(f'{torch.cuda.get_device_name(dev)} is not an sm_100 device; '
                               f'libmbpt_b200 is built for sm_100a only')
        _SUPPORTED.add(dev.index)
    return dev


def ptr(t):
    """Device address of a CUDA tensor (None for None). A tensor anywhere
    else is refused here, before any kernel could dereference it."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or t.device.type != 'cuda':
        raise ValueError(f'a device pointer is needed, got {type(t).__name__} on '
                         f'{getattr(t, "device", "host")}')
    return C.c_void_p(t.data_ptr())


def launch_count():
    """Kernels of libmbpt_b200 launched by this process so far."""
    return int(lib().mbpt_launch_count())


EPILOGUES = ('split', 'f32', 'hadamard', 'sigma_hadamard', 'row_contraction', 'f32_acc',
             'tf32_pair', 'dyson_tf32')


def gemm_timing(enable=True, read=False, families=True):
    """Start/stop CUDA-event timing of the tensor-core engine; with read,
    return {epilogue: (total ms, launches)} of what was recorded. families
    False leaves out the Dyson inverse's products (about a hundred small
    launches per frequency, which per-launch events would slow down)."""
    import numpy as np
    code = 0 if not enable else (1 if families else 2)
    if not read:
        check(lib().mbpt_gemm_timing(code, None, None), 'mbpt_gemm_timing')
        return None
    ms = np.zeros(8)
    n = np.zeros(8, dtype=np.int64)
    check(lib().mbpt_gemm_timing(code, ms.ctypes.data_as(C.c_void_p),
                                 n.ctypes.data_as(C.c_void_p)), 'mbpt_gemm_timing')
    return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(EPILOGUES) if n[i]}


def stream_ptr(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def host_array(a):
    """A contiguous FP64 host copy and its pointer (kept alive by the caller)."""
    import numpy as np
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return arr, arr.ctypes.data_as(C.c_void_p)


class Workspace:
    """A grow-only device scratch buffer per device, reused across calls."""

    def __init__(self):
        self._buf = {}

    def get(self, nbytes, device):
        key = device.index
        buf = self._buf.get(key)
        if buf is None or buf.numel() < nbytes:
            self._buf.pop(key, None)
            buf = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)
            self._buf[key] = buf
        return buf

    def release(self):
        self._buf.clear()


WORKSPACE = Workspace()


class Buffers:
    """Grow-only named device arrays per device, reused across calls: the
    sweep's large intermediates (chi0 / W - I and W(tau), 10 GB each at
    naux = 7200 and 24 points), so that repeated sweeps neither allocate nor
    free them. As with the workspace, calls on one device are stream-ordered
    and a result that must outlive the next call is copied (or asked for with
    the sweep's keep option, which allocates its own)."""

    def __init__(self):
        self._buf = {}

    def take(self, name, shape, device, dtype=torch.float64):
        n = 1
        for d in shape:
            n *= int(d)
        key = (device.index, name)
        buf = self._buf.get(key)
        if buf is None or buf.numel() < n or buf.dtype != dtype:
            self._buf.pop(key, None)
            buf = torch.empty(max(n, 1), dtype=dtype, device=device)
            self._buf[key] = buf
        return buf[:n].view(*shape)

    def release(self):
        self._buf.clear()


BUFFERS = Buffers()
