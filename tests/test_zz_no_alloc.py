"""The allocation-free split GEMM, mbpt_gemm_split_static, through the C ABI.

It serves callers that cannot allocate device memory -- hosts whose device
memory is all owned by their own allocator and which therefore cannot hand
the library a workspace. Here it must give the same product as the
workspace entry point mbpt_gemm_split, on two calls in a row with different
inputs and sizes (so that anything a first call leaves in the shared scratch
array would show in the second), and refuse sizes beyond its fixed scratch.
"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu


def _workspace_gemm(lib, _lib, A, B, m, n, k, dev):
    C = torch.empty((m, n), dtype=torch.float32, device=dev)
    ws = torch.empty(lib.mbpt_gemm_split_workspace_bytes(m, n, k), dtype=torch.uint8,
                     device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(lib.mbpt_gemm_split(_lib.ptr(A), _lib.ptr(B), m, n, k, 1.0, _lib.ptr(C), n,
                                   _lib.ptr(ws), ws.numel(), _lib.ptr(err), _lib.stream_ptr()),
               'mbpt_gemm_split')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C.cpu().numpy()


def test_static_scratch_gemm_matches_workspace_gemm_on_two_calls():
    from mbptcode_b200 import _lib
    lib = _lib.lib()
    dev = _lib.require_device()
    rng = np.random.default_rng(11)
    for m, n, k in ((517, 129, 1000), (300, 260, 200)):
        A = torch.as_tensor(rng.standard_normal((m, k)), device=dev)
        B = torch.as_tensor(rng.standard_normal((n, k)), device=dev)
        C = torch.full((m, n), float('nan'), dtype=torch.float32, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(lib.mbpt_gemm_split_static(_lib.ptr(A), _lib.ptr(B), m, n, k, 1.0,
                                              _lib.ptr(C), n, _lib.ptr(err),
                                              _lib.stream_ptr()), 'mbpt_gemm_split_static')
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        got = C.cpu().numpy()
        ref = _workspace_gemm(lib, _lib, A, B, m, n, k, dev)
        # the tolerance of the split-GEMM parity test, against the workspace entry
        scale = np.sqrt(k) * float(A.abs().max()) * float(B.abs().max())
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() <= 3e-5 * scale
        exact = A.cpu().numpy() @ B.cpu().numpy().T
        assert np.abs(got - exact).max() <= 3e-5 * scale


def test_static_scratch_gemm_refuses_sizes_beyond_its_array():
    from mbptcode_b200 import _lib
    lib = _lib.lib()
    cap = lib.mbpt_gemm_split_static_capacity()
    assert cap == 32 << 20
    # 4096^3 needs 4 (mp kp + np kp) + 4 mp np = 192 MiB of scratch
    rc = lib.mbpt_gemm_split_static(None, None, 4096, 4096, 4096, 1.0, None, 4096, None, None)
    assert rc == _lib.ERR_WORKSPACE
