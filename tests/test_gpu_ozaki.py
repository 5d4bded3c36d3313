"""The batched Cholesky's trailing updates on the int8 tensor cores (the
Ozaki scheme, csrc/ozaki.cu) against the same factorisation with cuBLAS
DGEMM updates and against LAPACK: log-determinants and W - I of a batch of
frequencies, FP64 mode, with 8 and with 7 signed 7-bit digit slices and with
6 signed 8-bit digits (base 254).

Sizes: n = 1000 (seven full 128-column panels and a last one of 104, so the
second 64-column half of the last panel is partly masked) and n = 300 (a last
panel of 44 columns, whose second half is empty), four and five frequencies
(the batched path starts at four)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')
pytestmark = pytest.mark.gpu

from mbptcode_b200.space_time import dyson_batch                    # noqa: E402


def _chi0_batch(n, nfreq, seed):
    rng = np.random.default_rng(seed)
    out = []
    for f in range(nfreq):
        A = rng.standard_normal((n, n // 2)) / np.sqrt(n)
        out.append(-(A @ A.T) * (1.0 + f))       # negative semidefinite: 1 - chi0 >= I
    return np.stack(out)


def _run(chi0, ozaki, slices=8):
    old = {k: os.environ.get(k) for k in ('MBPT_DYSON_OZAKI', 'MBPT_DYSON_OZAKI_SLICES')}
    os.environ['MBPT_DYSON_OZAKI'] = '1' if ozaki else '0'
    os.environ['MBPT_DYSON_OZAKI_SLICES'] = str(slices)
    try:
        c = torch.as_tensor(chi0, device='cuda').clone()
        logdet, _, info, _ = dyson_batch(c, want_w=True, precision='fp64')
        torch.cuda.synchronize()
        return logdet.cpu().numpy(), c.cpu().numpy(), info
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize('n,nfreq', [(1000, 4), (300, 5)])
def test_ozaki_cholesky_matches_dgemm_updates_and_lapack(n, nfreq):
    chi0 = _chi0_batch(n, nfreq, seed=n)
    ld_ref = np.array([np.linalg.slogdet(np.eye(n) - c)[1] for c in chi0])
    w_ref = np.stack([np.linalg.inv(np.eye(n) - c) - np.eye(n) for c in chi0])
    ld_b, w_b, info_b = _run(chi0, ozaki=False)
    assert not info_b.any()
    for slices, tol_w in ((8, 1e-12), (7, 5e-12), (6, 2e-11)):
        ld_o, w_o, info_o = _run(chi0, ozaki=True, slices=slices)
        assert not info_o.any()
        print(f'n={n} slices={slices}: log-det {np.abs(ld_o - ld_ref).max() / np.abs(ld_ref).max():.2e}'
              f', W {np.abs(w_o - w_ref).max() / np.abs(w_ref).max():.2e} (relative to the largest)')
        assert np.abs(ld_o - ld_ref).max() <= 1e-12 * np.abs(ld_ref).max(), slices
        assert np.abs(ld_o - ld_b).max() <= 1e-12 * np.abs(ld_b).max(), slices
        scale = np.abs(w_ref).max()
        assert np.abs(w_o - w_ref).max() <= tol_w * scale, (slices,
                                                            np.abs(w_o - w_ref).max() / scale)
        assert np.abs(w_o - w_b).max() <= tol_w * scale, slices


def test_ozaki_cholesky_flags_a_non_spd_frequency():
    """A frequency whose 1 - chi0 is indefinite fails its Cholesky on the
    int8 path as on the DGEMM path and is redone by LU (same W - I)."""
    n, nfreq = 256, 4
    rng = np.random.default_rng(7)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    mats = []
    for f in range(nfreq):
        lam = -rng.uniform(0.05, 3.0, n)
        if f == 2:
            lam[5] = 1.4                           # an eigenvalue of chi0 above 1
        mats.append((Q * lam) @ Q.T)
    chi0 = np.stack(mats)
    ld_b, w_b, info_b = _run(chi0, ozaki=False)
    ld_o, w_o, info_o = _run(chi0, ozaki=True)
    assert info_o[2] != 0 and info_b[2] != 0
    assert not info_o[[0, 1, 3]].any()
    assert np.abs(w_o - w_b).max() <= 1e-11 * np.abs(w_b).max()
