"""The full-size synthetic FP64 configuration shared by the golden generator
and the tests: sizes, seed, and the 32 seeded unit directions in (eps, X, D)
on which the reference's adjoint is projected."""
import numpy as np

C1 = dict(n_orb=400, nocc=40, M=2400, ntau=16, seed=400)
C1_DIRECTIONS = 32


def c1_directions(n_orb, M, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(C1_DIRECTIONS):
        de = rng.standard_normal(n_orb)
        dX = rng.standard_normal((M, n_orb))
        dD = rng.standard_normal((M, M))
        norm = np.sqrt((de ** 2).sum() + (dX ** 2).sum() + (dD ** 2).sum())
        out.append((de / norm, dX / norm, dD / norm))
    return out
