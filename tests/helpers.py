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


def zigzag_pairs(count):
    """The first `count` 2-D frequency pairs (f1, f2) in zig-zag order, (0, 0) excluded: along
    the anti-diagonals f1 + f2 = s = 1, 2, ..., f1 rising on odd s and falling on even s."""
    out = []
    s = 1
    while len(out) < count:
        f1s = range(0, s + 1) if s % 2 else range(s, -1, -1)
        for f1 in f1s:
            out.append((f1, s - f1))
            if len(out) == count:
                break
        s += 1
    return out


def eigenfaces_like(n, seed, side=64, terms=50, noise=0.02, scale_sigma=0.5):
    """Synthetic stand-in for face images (side² x n, FP32): column = Σ_{k<terms} a_k·P_k +
    noise·N(0,1), with P_k the unit-norm 2-D cosine of the k-th zig-zag frequency pair and
    a_k ~ N(0, k^-1.5) (variance, k counted from 1); columns mean-centred, then scaled by
    lognormal(0, scale_sigma)."""
    rng = np.random.default_rng(seed)
    i = (np.arange(side) + 0.5) / side
    P = []
    for f1, f2 in zigzag_pairs(terms):
        p = np.outer(np.cos(np.pi * f1 * i), np.cos(np.pi * f2 * i)).ravel()
        P.append(p / np.linalg.norm(p))
    P = np.stack(P, axis=1)                                   # side² x terms
    k = np.arange(1, terms + 1)
    a = rng.standard_normal((terms, n)) * (k ** -0.75)[:, None]
    X = P @ a + noise * rng.standard_normal((side * side, n))
    X -= X.mean(axis=0, keepdims=True)
    X *= rng.lognormal(0.0, scale_sigma, n)[None, :]
    return X.astype(np.float32)
