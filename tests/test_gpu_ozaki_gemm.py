"""The FP64-accurate GEMM on the int8 tensor cores (mbpt_dgemm_ozaki)
against torch's FP64 product: every transpose combination, sizes that are
not multiples of the tiles, alpha/beta, rows of very different magnitude
(each row and column carries its own scale), and a K above one pass (32768),
taken in two. Error bar: 8 digits per operand give ~2^-56 K max|row|
max|column| per entry; held to 1e-13 of that scale (K <= 5000) and the
7-digit form to 1e-11."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from mbptcode_b200 import _lib                                      # noqa: E402
from mbptcode_b200._lib import check, lib, ptr                      # noqa: E402


def ozaki(A, B, ta, tb, alpha=1.0, beta=0.0, C=None, slices=8):
    m = A.shape[1] if ta else A.shape[0]
    k = A.shape[0] if ta else A.shape[1]
    n = B.shape[0] if tb else B.shape[1]
    C = torch.zeros((m, n), dtype=torch.float64, device='cuda') if C is None else C
    ws = torch.empty(lib().mbpt_dgemm_ozaki_workspace_bytes(m, n, k, slices),
                     dtype=torch.uint8, device='cuda')
    err = torch.zeros(1, dtype=torch.int32, device='cuda')
    check(lib().mbpt_dgemm_ozaki(int(ta), int(tb), m, n, k, float(alpha), ptr(A), A.stride(0),
                                 ptr(B), B.stride(0), float(beta), ptr(C), C.stride(0), slices,
                                 ptr(ws), ws.numel(), ptr(err), _lib.stream_ptr()),
          'mbpt_dgemm_ozaki')
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C


def scale_of(A, B, ta, tb):
    a = (A.T if ta else A).abs().amax(1)
    b = (B.T if tb else B).abs().amax(0)
    k = A.shape[0] if ta else A.shape[1]
    return k * (a[:, None] * b[None, :])


@pytest.mark.parametrize('ta,tb', [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize('m,n,k', [(300, 200, 173), (129, 65, 4999), (1, 1, 1)])
def test_ozaki_dgemm_matches_fp64(ta, tb, m, n, k):
    g = torch.Generator(device='cuda').manual_seed(m * 7 + n + k)
    A = torch.randn((k, m) if ta else (m, k), generator=g, device='cuda', dtype=torch.float64)
    B = torch.randn((n, k) if tb else (k, n), generator=g, device='cuda', dtype=torch.float64)
    # rows of op(A) over twelve decades, a decaying spectrum along K
    opa = A.T if ta else A
    opa *= torch.logspace(-6, 6, m, device='cuda', dtype=torch.float64)[:, None]
    opa *= torch.exp(-torch.linspace(0, 5, k, device='cuda', dtype=torch.float64))[None, :]
    ref = (A.T if ta else A) @ (B.T if tb else B)
    got = ozaki(A, B, ta, tb)
    bound = scale_of(A, B, ta, tb)
    assert float(((got - ref).abs() / bound).max()) < 1e-13
    C0 = torch.randn(m, n, generator=g, device='cuda', dtype=torch.float64)
    got = ozaki(A, B, ta, tb, alpha=-2.0, beta=0.5, C=C0.clone())
    assert float(((got - (-2.0 * ref + 0.5 * C0)).abs() / (2 * bound + C0.abs())).max()) < 1e-13
    got7 = ozaki(A, B, ta, tb, slices=7)
    assert float(((got7 - ref).abs() / bound).max()) < 1e-11


def test_ozaki_dgemm_long_k_in_two_passes():
    g = torch.Generator(device='cuda').manual_seed(5)
    A = torch.randn(96, 40000, generator=g, device='cuda', dtype=torch.float64)
    B = torch.randn(72, 40000, generator=g, device='cuda', dtype=torch.float64)
    ref = A @ B.T
    got = ozaki(A, B, False, True)
    bound = scale_of(A, B, False, True)
    assert float(((got - ref).abs() / bound).max()) < 1e-12
