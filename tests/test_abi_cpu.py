"""CPU-side checks of the C ABI: the library builds, loads and exports every
entry point include/mbpt_b200.h declares (no compute call: no GPU here)."""
import os
import re

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), '..'))


def declared():
    text = open(os.path.join(ROOT, 'include', 'mbpt_b200.h')).read()
    return sorted(set(re.findall(r'\b(mbpt_[a-z0-9_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol():
    from mbptcode_b200 import _lib
    lib = _lib.lib()
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.exported_symbols())


def test_host_only_queries():
    from mbptcode_b200 import _lib
    lib = _lib.lib()
    assert lib.mbpt_abi_version() == 2
    assert _lib.status_string(_lib.ERR_NOT_SPD).startswith('1 - chi0')
    assert lib.mbpt_mlp_param_count(64) == 64 * 64 + 7 * 64 + 1
    # workspace queries are pure host arithmetic
    w_fp64 = lib.mbpt_chi0_workspace_bytes(7200, 1200, 120, 7200, 24, 0)
    w_mix = lib.mbpt_chi0_workspace_bytes(7200, 1200, 120, 7200, 24, 1)
    assert w_fp64 > 2 * 7200 * 7200 * 8 and w_mix > 24 * 7296 * 7296 * 4
    assert lib.mbpt_gemm_split_workspace_bytes(100, 100, 100) > 0


def test_product_path_refuses_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is visible')
    from mbptcode_b200 import _lib
    with pytest.raises(RuntimeError):
        _lib.require_device()


def test_host_tensors_are_refused_before_any_kernel():
    import numpy as np
    import torch
    from mbptcode_b200 import _lib
    with pytest.raises(ValueError):
        _lib.ptr(torch.zeros(3))
    with pytest.raises(ValueError):
        _lib.ptr(np.zeros(3))
    assert _lib.ptr(None) is None

