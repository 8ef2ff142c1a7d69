"""Shared helpers for the GPU tests: seeded inputs and tolerances."""
import numpy as np

# FP32 tolerance for λ traces and products against the FP64-accumulating oracle: the GPU
# accumulates each column dot and the per-CTA partial sums in FP32 (as the reference does),
# so a step's relative error is ~sqrt(m)·2^-24 per dot; 2e-5 leaves a wide margin.
RTOL_LAMBDA_F32 = 2e-5
RTOL_VEC_F32 = 1e-4


def scaled_gaussian(m, n, seed, sigma=1.0, shift=0.0, dtype=np.float32):
    """N(0,1) entries times per-column lognormal(0, sigma) scales (+ shift), FP64 then cast."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((m, n)) * rng.lognormal(0.0, sigma, n) + shift
    return A.astype(dtype)


def states(count, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(1, 2**32, size=count, dtype=np.uint64).astype(np.uint32)


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def vec_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
