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
    assert lib.mbpt_abi_version() == 1
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


def test_integration_stub_matches_the_binding():
    """The ctypes stub a maintainer would paste into MBPTcode (INTEGRATION.md,
    section 3) declares the same argument and return types as the package's
    own binding, entry by entry."""
    import ctypes as C
    import os
    import re
    from mbptcode_b200 import _lib
    text = open(os.path.join(os.path.dirname(__file__), '..', 'INTEGRATION.md')).read()
    names = {'_p': C.c_void_p, '_i64': C.c_int64, '_i': C.c_int, '_d': C.c_double,
             '_sz': C.c_size_t}
    argtypes = dict(re.findall(r'_L\.(mbpt_\w+)\.argtypes = \[([^\]]*)\]', text, re.S))
    restypes = dict(re.findall(r'_L\.(mbpt_\w+)\.restype = (\w+)', text))
    assert argtypes, 'no stub found'
    for name, args in argtypes.items():
        got = [names[a.strip()] for a in args.replace('\n', ' ').split(',') if a.strip()]
        assert got == _lib._SIGNATURES[name][1], name
    for name, res in restypes.items():
        assert names[res] == _lib._SIGNATURES[name][0], name
