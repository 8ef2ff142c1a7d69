"""Seeded inputs shared by the golden-fixture generator and the tests (numpy PCG64).

The fixtures store only the reference's outputs; the inputs are regenerated from these seeds.
"""
import numpy as np

M = 256        # square: the reference handles m x m only (m % 128 == 0)
C = 64         # samples (c % 8 == 0, c <= m)
STEPS = 12
VR = 4
NSTEPS = 8     # step-by-step dumps
PICK_N, PICK_C = 1000, 512


def symmetric_matrix(seed: int = 11, m: int = M) -> np.ndarray:
    """Symmetric A (the reference computes A·A with two OP_N GEMVs, i.e. A·Aᵀ for symmetric A)
    with heavy column scales, so sampling is far from uniform."""
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((m, m))
    s = rng.lognormal(0.0, 1.0, m)
    A = (B + B.T) * 0.5
    A = A * np.sqrt(np.outer(s, s))          # keeps symmetry, scales row/column j by sqrt(s_j)
    A += 0.25                                # non-zero column means: exercises the centring
    return A.astype(np.float32)


def states(seed: int = 12, count: int = M) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(1, 2**32, size=count, dtype=np.uint64).astype(np.uint32)


def start_vector(seed: int = 13, m: int = M) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal(m).astype(np.float32)


def top_eigenvector(A: np.ndarray) -> np.ndarray:
    A64 = A.astype(np.float64)
    w, V = np.linalg.eigh(A64 @ A64.T)
    v = V[:, -1]
    return v if v.sum() >= 0 else -v


def pick_inputs(seed: int = 14):
    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 2.0, PICK_N).astype(np.float32)
    w[rng.random(PICK_N) < 0.1] = 0.0
    cdf = np.cumsum(w.astype(np.float64)).astype(np.float32)
    st = rng.integers(0, 2**32, size=PICK_C, dtype=np.uint64).astype(np.uint32)
    return cdf, st
