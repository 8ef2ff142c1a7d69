"""CPU oracle for the power method on C = A·Aᵀ: exact, previous AMM, proposed AMM, proposed AMM v2.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA library is compared
against; it is imported by ``tests/``, by ``__graft_entry__.smoke()`` and by the CPU-baseline
leg of ``bench.py``, and by nothing in the product path.  It restates, in numpy, the algorithm
of Takuya-Okuyama/eigenvalueComputation_by_AMM; every function cites the reference file:line
it follows.

Conventions
-----------
* ``A`` is an (m, n) numpy array.  Column j is ``A[:, j]`` (the reference stores A column-major
  with lda = m, so "column j" is the contiguous run ``dA + m*j``).  The reference only handles
  square m x m matrices; here n may differ from m, and every per-column quantity has length n
  while x, y, z, v have length m.
* Arithmetic the reference does in FP32 and stores in FP32 is rounded to FP32 here at the same
  points; sums the reference accumulates in FP32 with a GPU-specific order (cuBLAS, CUB,
  BlockReduce, atomics) are accumulated in FP64 here and rounded once.  So FP32 results agree
  with the reference to FP32 rounding, and integer results (xorshift states, sampled indices)
  agree bit for bit.
* Two CDF precisions exist.  ``"f32"`` reproduces the reference's ``pick_index`` exactly for a
  given FP32 CDF array (the reference builds that array with ``cub::DeviceScan::InclusiveSum``,
  whose association order is CUB's; ``cdf_f32`` below is the correctly rounded prefix, which is
  what the CUDA library builds in compat mode).  ``"f64"`` is the production mode: an FP64 CDF
  and an FP64 target.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

F32 = np.float32
F64 = np.float64
U32 = np.uint32

__all__ = [
    "get_norms", "alpha_squared", "set_weights", "cdf_f32", "cdf_f64", "update_weights",
    "xorshift32", "pick_index", "sample_sorted", "previous_amm", "proposed_amm", "dots",
    "exact_product", "dot_product_and_generate_x", "normalize", "generate_zv",
    "PowerTrace", "power_method", "reported_eigenvalue", "grad_lambda", "lambda_max_f64",
    "batch_seed_states", "batch_start_block", "batch_cdf", "batch_block_power", "BatchTrace",
    "shard_cdf", "sharded_weights", "sharded_previous",
]


# --------------------------------------------------------------------------------------------
# Column statistics and sampling probabilities
# --------------------------------------------------------------------------------------------

def get_norms(A: np.ndarray):
    """Per-column mean, norm and centred norm (device_memory.h:34-59, ``get_norms``).

    The reference accumulates ``sum`` and ``sum_pow2`` in FP64 over the m rows of column j and
    writes ``alpha = (float)(sum/m)``, ``normA = (float)sqrt(sum_pow2)`` and
    ``normAprime = (float)sqrt(sum_pow2 - mean*mean*m)``.  The last expression can go slightly
    negative through cancellation for a constant column (the reference then stores NaN); it is
    clamped at 0 here and in the CUDA library.
    """
    A64 = np.asarray(A, dtype=F64)
    m = A64.shape[0]
    s = A64.sum(axis=0)
    q = np.einsum("ij,ij->j", A64, A64)
    mean = s / F64(m)
    alpha = mean.astype(F32)
    norm = np.sqrt(q).astype(F32)
    normp = np.sqrt(np.maximum(q - mean * mean * F64(m), 0.0)).astype(F32)
    return alpha, norm, normp


def alpha_squared(alpha: np.ndarray) -> float:
    """‖α‖² (device_memory.h:335-336: ``cublasSnrm2`` of α, squared).  Accumulated in FP64."""
    a = np.asarray(alpha, dtype=F64)
    return float(np.dot(a, a))


def set_weights(norm: np.ndarray) -> np.ndarray:
    """weight_j = norm_j² in FP32 (common.h:34-40, ``set_weights``)."""
    norm = np.asarray(norm, dtype=F32)
    return (norm * norm).astype(F32)


def cdf_f64(weight: np.ndarray) -> np.ndarray:
    """Unnormalised inclusive prefix sum of the weights, in FP64 (production CDF; it replaces
    the FP32 ``cub::DeviceScan::InclusiveSum`` at powerMethod_by_previous.cuh:26-32)."""
    return np.cumsum(np.asarray(weight, dtype=F64), dtype=F64)


def cdf_f32(weight: np.ndarray) -> np.ndarray:
    """FP32 CDF used by compat mode: the correctly rounded prefix sum of the FP32 weights.

    The reference's FP32 CDF (powerMethod_by_previous.cuh:26-32) comes from CUB's scan, whose
    rounding depends on CUB's tile order; any FP32 scan is within a few ulps of this one.
    """
    return cdf_f64(weight).astype(F32)


def update_weights(weight: np.ndarray, total: float, c: int, precision: str = "f64") -> np.ndarray:
    """Inverse-probability scale w_j = total / (weight_j · c) = 1/(c·p_j) (common.h:42-53).

    ``precision="f32"`` divides in FP32 like the reference (which, compiled with
    ``--use_fast_math``, uses an approximate division: within 2 ulp of this); ``"f64"``
    divides in FP64 and rounds once (what the CUDA library stores).
    """
    if precision == "f32":
        w = np.asarray(weight, dtype=F32)
        with np.errstate(divide="ignore", invalid="ignore"):
            return (F32(total) / (w * F32(c))).astype(F32)
    w = np.asarray(weight, dtype=F64)
    with np.errstate(divide="ignore", invalid="ignore"):
        return (F64(total) / (w * F64(c))).astype(F32)


# --------------------------------------------------------------------------------------------
# Random draws and inverse-CDF sampling (integer work: bit exact)
# --------------------------------------------------------------------------------------------

def xorshift32(states: np.ndarray):
    """One xorshift32 step per state and the derived uniform (device_memory.h:506-514).

    y ^= y << 13; y ^= y >> 17; y ^= y << 5 (uint32 wrap-around).  The uniform is the float
    with exponent 0 and the low 23 bits of y as mantissa, minus 1: exact, in [0, 1).
    Returns (new_states, u) with u float32.
    """
    y = np.array(states, dtype=U32, copy=True)
    y ^= (y << U32(13))
    y ^= (y >> U32(17))
    y ^= (y << U32(5))
    bits = (y & U32(0x007FFFFF)) | U32(0x3F800000)
    u = bits.view(F32) - F32(1.0)
    return y, u.astype(F32)


def pick_index(cdf: np.ndarray, states: np.ndarray, c: int):
    """Inverse-CDF sampling of c column indices (device_memory.h:516-545, ``pick_index``).

    Sample k advances ``states[k]`` once and searches for the first index i in [0, n-1] with
    ``cdf[i] > target``, where target = cdf[n-1] · u_k; if there is none it returns n-1 (the
    upper bound the reference's bisection starts from).  For a non-decreasing CDF every correct
    bisection returns this same index, so the search order does not matter.

    With an FP32 CDF the target is the FP32 product (as in the reference); with an FP64 CDF it
    is the FP64 product of the FP64 total and the (exact) uniform.
    Returns (indices uint32[c], new_states); states beyond the first c are not touched.
    """
    cdf = np.asarray(cdf)
    states = np.asarray(states, dtype=U32)
    n = cdf.shape[0]
    new_states = states.copy()
    s, u = xorshift32(states[:c])
    new_states[:c] = s
    if cdf.dtype == F32:
        target = (F32(cdf[n - 1]) * u).astype(F32)
    else:
        target = F64(cdf[n - 1]) * u.astype(F64)
    idx = np.searchsorted(cdf, target, side="right")
    idx = np.minimum(idx, n - 1).astype(U32)
    return idx, new_states


def sample_sorted(cdf: np.ndarray, states: np.ndarray, c: int):
    """``pick_index`` followed by the ascending sort the reference does with
    ``cub::DeviceRadixSort::SortKeys`` (powerMethod_by_previous.cuh:56-70)."""
    idx, new_states = pick_index(cdf, states, c)
    return np.sort(idx), new_states


# --------------------------------------------------------------------------------------------
# Products
# --------------------------------------------------------------------------------------------

def exact_product(A: np.ndarray, x: np.ndarray) -> np.ndarray:
    """y = A·(Aᵀ·x), FP64 accumulation, FP32 result.

    The reference computes ``tmp = A·x; y = A·tmp`` with two ``cublasSgemv(OP_N)`` calls
    (powerMethod_by_exact.cuh:31-53); for its symmetric A that is A·Aᵀ·x.  For a rectangular
    A the meaning kept here is C·x with C = A·Aᵀ.
    """
    A64 = np.asarray(A, dtype=F64)
    t = A64.T @ np.asarray(x, dtype=F64)
    return (A64 @ t).astype(F32)


def previous_amm(A, x, x_memo, y_memo, idx_sorted, w):
    """One previous-AMM product (core_previousAMM.cuh:4-263 with the launch at
    powerMethod_by_previous.cuh:73-96).

    kernel1: tmp_k = w[s_k] · (A_{s_k}ᵀ (x − x_memo))            (:163-168)
             y ← y_memo                                              (:170-174)
    kernel2: y += Σ_k A_{s_k} · tmp_k                                 (:203-262)
    Returns (tmp float32[c], y float32[m]).
    """
    A = np.asarray(A)
    dx = np.asarray(x, dtype=F32) - np.asarray(x_memo, dtype=F32)     # FP32 subtraction
    cols = A[:, idx_sorted].astype(F64)
    d = cols.T @ dx.astype(F64)
    tmp = (d.astype(F32) * np.asarray(w, dtype=F32)[idx_sorted]).astype(F32)
    y = np.asarray(y_memo, dtype=F64) + cols @ tmp.astype(F64)
    return tmp, y.astype(F32)


def dots(x, x_memo, z):
    """(Σ dx, z·dx) in FP64 with dx = x − x_memo in FP32 (common.h:55-87, ``dots``)."""
    dx = (np.asarray(x, dtype=F32) - np.asarray(x_memo, dtype=F32)).astype(F64)
    return float(dx.sum()), float(np.dot(dx, np.asarray(z, dtype=F64)))


def generate_zv(A, alpha, alpha2):
    """z = A·α and v = z − ‖α‖² (powerMethod_by_proposed.cuh:132-145 and
    core_proposedAMM.cuh:4-15).  FP64 accumulation, FP32 storage."""
    z = (np.asarray(A, dtype=F64) @ np.asarray(alpha, dtype=F64)).astype(F32)
    v = (z.astype(F64) - F64(alpha2)).astype(F32)
    return z, v


def proposed_amm(A, alpha, x, x_memo, y_memo, idx_sorted, w, z, v):
    """One proposed-AMM product (core_proposedAMM.cuh:17-313, launched at
    powerMethod_by_proposed.cuh:258-313).

    dots:    Σdx and z·dx                                            (common.h:55-87)
    kernel1: tmp_k = (A_{s_k}ᵀ dx − α_{s_k}·Σdx) · w[s_k]              (:191-196)
             y ← y_memo + Σdx·v + z·dx   (FP64, rounded to FP32)      (:198-212)
    kernel2: y += Σ_k (A_{s_k} − α_{s_k}) · tmp_k                      (:257-312)
    Returns (tmp float32[c], y float32[m]).
    """
    A = np.asarray(A)
    sum_dx, zdx = dots(x, x_memo, z)
    dx = np.asarray(x, dtype=F32) - np.asarray(x_memo, dtype=F32)
    cols = A[:, idx_sorted].astype(F64)
    al = np.asarray(alpha, dtype=F32)[idx_sorted].astype(F64)
    d = cols.T @ dx.astype(F64)
    tmp = ((d - al * sum_dx) * np.asarray(w, dtype=F32)[idx_sorted].astype(F64)).astype(F32)
    base = (np.asarray(y_memo, dtype=F64) + (sum_dx * np.asarray(v, dtype=F64) + zdx)).astype(F32)
    corr = cols @ tmp.astype(F64) - np.dot(al, tmp.astype(F64))
    y = base.astype(F64) + corr
    return tmp, y.astype(F32)


# --------------------------------------------------------------------------------------------
# Normalisation and Rayleigh step
# --------------------------------------------------------------------------------------------

def normalize(x):
    """x / ‖x‖ with an FP64 sum of squares and an FP32 scale (common.h:156-183)."""
    x = np.asarray(x, dtype=F32)
    ss = float(np.dot(x.astype(F64), x.astype(F64)))
    scale = F32(1.0 / np.sqrt(ss))
    return (x * scale).astype(F32)


def dot_product_and_generate_x(x, y, vstar=None):
    """Rayleigh quotient, error, cosine and the next iterate (common.h:89-154).

    λ = x·y, ‖y‖² and e = y·v* are FP64 sums; scale = 1/sqrt(‖y‖²) in FP64;
    err = e·scale, cos = λ·scale; x_new = (float)scale · y in FP32.
    Returns (lam, err, cos, x_new).
    """
    x64 = np.asarray(x, dtype=F32).astype(F64)
    y32 = np.asarray(y, dtype=F32)
    y64 = y32.astype(F64)
    lam = float(np.dot(y64, x64))
    yy = float(np.dot(y64, y64))
    e = float(np.dot(y64, np.asarray(vstar, dtype=F64))) if vstar is not None else 0.0
    scale = 1.0 / np.sqrt(yy)
    x_new = (y32 * F32(scale)).astype(F32)
    return lam, e * scale, lam * scale, x_new


def reported_eigenvalue(lam, offset=0.0):
    """The reference's printed eigenvalue max(0, sqrt(max(0, λ)) − offset)
    (powerMethod_by_exact.cuh:83): an eigenvalue of its symmetric, diagonally shifted A."""
    lam = np.asarray(lam, dtype=F64)
    return np.maximum(0.0, np.sqrt(np.maximum(0.0, lam)) - offset)


# --------------------------------------------------------------------------------------------
# Drivers
# --------------------------------------------------------------------------------------------

@dataclasses.dataclass
class PowerTrace:
    eigs: np.ndarray                     # λ per step (FP64)
    errs: np.ndarray                     # (y·v*)/‖y‖ per step
    coss: np.ndarray                     # cos∠(x_i, x_{i+1}) per step
    modes: list                          # "exact", "exact_nomemo", "previous", "proposed"
    indices: list                        # sorted sampled indices per AMM step (None otherwise)
    x: np.ndarray                        # final iterate
    y: np.ndarray                        # final product
    states: np.ndarray                   # xorshift states after the run
    cdf: dict                            # CDF per weighting ("norm", "normp") actually used


def _sampling_tables(A, which, c, n, cdf_precision, sanity, cdf_override):
    alpha, norm, normp = get_norms(A)
    base = norm if which == "norm" else normp
    f32 = cdf_precision == "f32"
    if sanity and c == n:
        weight = np.ones(n, dtype=F32 if f32 else F64)                 # device_memory.h:500-504
    elif f32:
        weight = set_weights(base)
    else:
        # FP64 mode: the exact square of the FP32 norm (no FP32 rounding of norm²)
        weight = base.astype(F64) * base.astype(F64)
    if cdf_override is not None and which in cdf_override:
        cdf = np.asarray(cdf_override[which])
    else:
        cdf = cdf_f32(weight) if f32 else cdf_f64(weight)
    w = update_weights(weight, float(cdf[n - 1]), c,
                       precision="f32" if cdf.dtype == F32 else "f64")
    return cdf, w


def power_method(A, x0, *, method="exact", step=10, c=None, states=None, vr_period=0,
                 vr_adaptive_threshold=0.0, sanity=False, cdf_precision="f64", vstar=None,
                 cdf_override: Optional[dict] = None):
    """One call of ``powerMethod_by_{exact,previous,proposed,proposed_v2}``.

    exact       powerMethod_by_exact.cuh:4-100
    previous    powerMethod_by_previous.cuh:100-210 (square_of_A_by_previous at :7-98)
    proposed    powerMethod_by_proposed.cuh:317-447 (square_of_A_by_proposed at :7-103)
    proposed_v2 powerMethod_by_proposed_v2.cuh:199-377

    ``x0`` is the raw start vector (the reference draws it with ``curandGenerateNormal`` and
    then calls ``normalize``); it is normalised here.  ``states`` are the xorshift states
    (the reference's ``d_rnd``); they are advanced once per sample of every AMM step and the
    advanced states are returned.  Variance reduction (VR) follows the reference:

    * previous:    VR when ``(i+1) % vr_period == 0`` or ``cos > 1 − thr``  (:135-137)
    * proposed:    the same, and only when ``i > last_exact + 1``             (:371-373)
    * proposed_v2: phase 1 is ``vr_period − 1`` previous-AMM steps; step ``vr_period − 1``
      is exact without a memo update; phase 2 is proposed AMM with periodic VR (:234-347).

    A VR step computes the exact product and copies [x | y] into [x_memo | y_memo].
    ``sanity`` (with c == n) is the reference's ``-sanity`` known-answer mode: all weights 1 and
    indices 0..n−1, so every AMM step equals the exact product.
    """
    A = np.asarray(A)
    m, n = A.shape
    if c is None:
        c = n
    x = normalize(x0)
    memo_x = np.zeros(m, dtype=F32)
    memo_y = np.zeros(m, dtype=F32)
    y = np.zeros(m, dtype=F32)
    states = np.zeros(max(c, 1), dtype=U32) if states is None else np.array(states, dtype=U32)
    variance_reduction = vr_period > 0 or vr_adaptive_threshold > 0.0
    alpha, norm, normp = get_norms(A)
    a2 = alpha_squared(alpha)
    z, v = generate_zv(A, alpha, a2)
    use_seq = sanity and c == n
    cdfs = {}

    eigs, errs, coss, modes, indices = [], [], [], [], []

    def amm_step(which):
        nonlocal states, y
        if which not in cdfs:
            cdfs[which] = _sampling_tables(A, which, c, n, cdf_precision, sanity, cdf_override)
        cdf, w = cdfs[which]
        if use_seq:
            idx = np.arange(n, dtype=U32)                              # device_memory.h:547-551
        else:
            idx, states = sample_sorted(cdf, states, c)
        if which == "norm":
            _, y = previous_amm(A, x, memo_x, memo_y, idx, w)
        else:
            _, y = proposed_amm(A, alpha, x, memo_x, memo_y, idx, w, z, v)
        indices.append(idx)

    def rayleigh():
        nonlocal x
        lam, err, cos, x_new = dot_product_and_generate_x(x, y, vstar)
        eigs.append(lam)
        errs.append(err)
        coss.append(cos)
        x = x_new
        return cos

    dot = 0.0
    if method == "exact":
        for _ in range(step):
            y = exact_product(A, x)
            modes.append("exact_nomemo")
            indices.append(None)
            rayleigh()
    elif method in ("previous", "proposed"):
        which = "norm" if method == "previous" else "normp"
        last_exact = 0
        for i in range(step):
            vr_now = variance_reduction and (
                (vr_period > 0 and (i + 1) % vr_period == 0)
                or (vr_adaptive_threshold > 0.0 and dot > 1.0 - vr_adaptive_threshold))
            if method == "proposed":
                vr_now = vr_now and i > last_exact + 1
            if vr_now:
                y = exact_product(A, x)
                memo_x, memo_y = x.copy(), y.copy()
                last_exact = i
                modes.append("exact")
                indices.append(None)
            else:
                amm_step(which)
                modes.append(method)
            dot = rayleigh()
    elif method == "proposed_v2":
        if vr_period < 1 or step < vr_period:
            raise ValueError("proposed_v2 needs 1 <= vr_period <= step")
        for _ in range(vr_period - 1):
            amm_step("norm")
            modes.append("previous")
            rayleigh()
        y = exact_product(A, x)                   # [z, tmp] = A·[α, x]; y = A·tmp (:255-294)
        modes.append("exact_nomemo")
        indices.append(None)
        rayleigh()
        for i in range(vr_period, step):
            if variance_reduction and (i + 1) % vr_period == 0:
                y = exact_product(A, x)
                memo_x, memo_y = x.copy(), y.copy()
                modes.append("exact")
                indices.append(None)
            else:
                amm_step("normp")
                modes.append("proposed")
            rayleigh()
    else:
        raise ValueError(f"unknown method {method!r}")

    return PowerTrace(np.array(eigs, dtype=F64), np.array(errs, dtype=F64),
                      np.array(coss, dtype=F64), modes, indices, x, y, states,
                      {k: v_[0] for k, v_ in cdfs.items()})


# --------------------------------------------------------------------------------------------
# Batched block power iteration (an extension: the reference solves one vector of one matrix per
# run).  The products and sampling follow the reference's single-vector path column by column:
# the exact product is powerMethod_by_exact.cuh:37-53, the sampled product is
# previousAMM_kernel1+2 (core_previousAMM.cuh:163-174, 225-232) with pick_index
# (device_memory.h:506-545), and variance reduction follows powerMethod_by_previous.cuh:135-157,
# applied to a block of K vectors.
# --------------------------------------------------------------------------------------------

_M64 = (1 << 64) - 1


def batch_seed_states(seed: int, total: int) -> np.ndarray:
    """The batch's xorshift32 states: a splitmix64 stream from ``seed`` (the high 32 bits of
    each output; a zero, xorshift32's fixed point, is replaced by 0x6A09E667).  Matrix b owns
    the c_b states after those of the matrices before it."""
    out = np.empty(total, dtype=U32)
    z = int(seed) & _M64
    for k in range(total):
        z = (z + 0x9E3779B97F4A7C15) & _M64
        x = z
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M64
        x ^= x >> 31
        v = x >> 32
        out[k] = v if v else 0x6A09E667
    return out


def batch_start_block(seed: int, mi: int, m: int, K: int) -> np.ndarray:
    """The start block of matrix ``mi`` (m x K, FP32): a counter-based hash of (seed, matrix,
    row, vector) mapped to [-1, 1)."""
    rows = np.arange(m, dtype=np.uint64)[:, None]
    vecs = np.arange(K, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) ^ (np.uint64(0x9E3779B97F4A7C15) * np.uint64(mi + 1))
             ^ (rows << np.uint64(20)) ^ (vecs << np.uint64(52)))
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    hi = (z >> np.uint64(32)).astype(np.uint32).view(np.int32)
    return (hi.astype(F32) * F32(1.0 / 2147483648.0)).astype(F32)


def batch_cdf(A) -> np.ndarray:
    """The FP32 sampling CDF of previous AMM for one matrix: ‖A_j‖² (get_norms / set_weights,
    device_memory.h:34-59, common.h:34-40), prefix-summed in FP64 and stored in FP32 (the
    reference's CUB InclusiveSum, powerMethod_by_previous.cuh:26-32)."""
    A64 = np.asarray(A, dtype=F64)
    w = (A64 * A64).sum(axis=0).astype(F32)
    return np.cumsum(w.astype(F64)).astype(F32)


@dataclasses.dataclass
class BatchTrace:
    ritz: np.ndarray          # K Ritz values of the last Rayleigh–Ritz step, descending
    vector: np.ndarray        # unit top Ritz vector (m)
    picks: list               # per product: uint32[c] raw picks (None for an exact product)
    kinds: list               # per product: "exact" or "amm"
    states: np.ndarray        # the states after the run


def _orth(Y):
    """An orthonormal basis of span(Y) (any basis serves: every step below is invariant under
    a rotation of the block)."""
    q, _ = np.linalg.qr(Y)
    return q


def batch_block_power(A, *, K: int, max_iter: int, c: int = 0, states=None, cdf=None,
                      vr_period: int = 0, seed: int = 1234, mi: int = 0) -> BatchTrace:
    """Block power iteration with Rayleigh–Ritz on C = A·Aᵀ for one matrix of the batch, run
    for exactly ``max_iter`` products (no early stop), in FP64.

    X_0 is the orthonormalised start block.  Product p multiplies the current orthonormal
    block X:
      * exact (c == 0, or with variance reduction when (p + 1) % vr_period == 0 or p is the
        last product): Y = A·(Aᵀ·X), and with variance reduction (X_memo, Y_memo) <- (X, Y);
      * sampled: c draws by pick_index from ``cdf`` and ``states`` (advanced once per sampled
        product), column j weighted mult_j·total/(c·(cdf[j] − cdf[j−1])) with the FP32 CDF
        values (the realised probability of the draw), and
        Y = Y_memo·S + Σ_j w_j·A_j·(A_jᵀ·D),  D = X − X_memo·S,  S = X_memoᵀ·X
        (S = 0 before the first exact product: Y = Ĉ·X).
    After each product the next block is an orthonormal basis of span(Y); the Ritz values are
    the eigenvalues of sym(XᵀY) of the last product.
    """
    A64 = np.asarray(A, dtype=F64)
    m, n = A64.shape
    X = _orth(batch_start_block(seed, mi, m, K).astype(F64))
    st = None if states is None else np.asarray(states, dtype=U32).copy()
    cdf32 = None if cdf is None else np.asarray(cdf, dtype=F32)
    Xm = Ym = None
    picks, kinds = [], []
    Y = None
    for p in range(max_iter):
        exact = c == 0 or (vr_period > 0 and ((p + 1) % vr_period == 0 or p + 1 >= max_iter))
        if exact:
            Y = A64 @ (A64.T @ X)
            if vr_period > 0 and c > 0:
                Xm, Ym = X.copy(), Y.copy()
            picks.append(None)
            kinds.append("exact")
        else:
            idx, st = pick_index(cdf32, st, c)
            picks.append(idx)
            kinds.append("amm")
            cols, mult = np.unique(idx, return_counts=True)
            total = F64(cdf32[-1])
            prev = np.where(cols > 0, cdf32[np.maximum(cols.astype(np.int64) - 1, 0)].astype(F64), 0.0)
            step = cdf32[cols].astype(F64) - prev
            w = (mult.astype(F64) * total / (F64(c) * step)).astype(F32).astype(F64)
            if Xm is not None:
                S = Xm.T @ X
                D = X - Xm @ S
            else:
                S, D = None, X
            As = A64[:, cols]
            Y = As @ (w[:, None] * (As.T @ D))
            if S is not None:
                Y = Y + Ym @ S
        if p + 1 < max_iter:
            Xn = _orth(Y)
            X_last, Y_last = X, Y
            X = Xn
        else:
            X_last, Y_last = X, Y
    H = 0.5 * (X_last.T @ Y_last + Y_last.T @ X_last)
    th, V = np.linalg.eigh(H)
    order = np.argsort(th)[::-1]
    v = X_last @ V[:, order[0]]
    return BatchTrace(ritz=th[order], vector=v / np.linalg.norm(v), picks=picks, kinds=kinds,
                      states=st)


# --------------------------------------------------------------------------------------------
# Column-sharded previous AMM (an extension: the reference runs on one GPU).  Each shard builds
# the FP64 CDF of ‖A_j‖² over its columns (set_weights and the CDF scan, common.h:34-40 and
# powerMethod_by_previous.cuh:26-32); the global CDF shifts each shard's by the totals of the
# shards before it.  Every rank draws the same picks from it (pick_index,
# device_memory.h:506-545) and multiplies by its own picked columns (previousAMM_kernel1+2,
# core_previousAMM.cuh:163-174, 225-232); the partial products are summed (one all-reduce).
# --------------------------------------------------------------------------------------------

def shard_cdf(A_shard) -> np.ndarray:
    """One shard's FP64 CDF: the prefix of (double)norm_j² with norm_j the FP32 column norm."""
    _, norm, _ = get_norms(A_shard)
    n64 = norm.astype(F64)
    return np.cumsum(n64 * n64, dtype=F64)


def sharded_weights(cdf, idx):
    """The distinct picked columns, and w_j = fl32(mult_j·total/(c·(cdf[j] − cdf[j−1]))) (the
    realised probability of the draw), for the c picks idx."""
    cdf = np.asarray(cdf, dtype=F64)
    cols, mult = np.unique(np.asarray(idx), return_counts=True)
    c = len(idx)
    prev = np.where(cols > 0, cdf[np.maximum(cols.astype(np.int64) - 1, 0)], 0.0)
    step = cdf[cols] - prev
    w = (mult.astype(F64) * cdf[-1] / (F64(c) * step)).astype(F32)
    return cols, w


def sharded_previous(A, bounds, *, c, states, step, vr_period=0, x0, cdf=None):
    """The column-sharded previous-AMM power method in one process, shard by shard.

    ``bounds``: the shards' [col0, col1) in rank order.  ``cdf``: the global CDF to draw from
    (default: the shards' FP64 CDFs shifted by the preceding shards' totals, summed in rank
    order).  Step i is an exact, memoised step when vr_period > 0 and (i + 1) % vr_period == 0
    (powerMethod_by_previous.cuh:135-157).  Each shard's partial product is rounded to FP32,
    and the partials are summed in rank order (y_memo added by the first shard).
    Returns (eigs, kinds, states, global cdf, the picks of every AMM step).
    """
    A = np.asarray(A)
    if cdf is None:
        parts, offset = [], 0.0
        for a, b in bounds:
            cg = shard_cdf(A[:, a:b])
            parts.append(cg + offset)
            offset = offset + float(cg[-1])
        cdf = np.concatenate(parts)
    cdf = np.asarray(cdf, dtype=F64)
    st = np.asarray(states, dtype=U32).copy()
    m = A.shape[0]
    x = normalize(x0)
    x_memo = np.zeros(m, F32)
    y_memo = np.zeros(m, F32)
    eigs, kinds, picks = [], [], []
    for i in range(step):
        if vr_period > 0 and (i + 1) % vr_period == 0:
            y = np.zeros(m, F32)
            for a, b in bounds:
                y = (y + exact_product(A[:, a:b], x)).astype(F32)
            x_memo, y_memo = x.copy(), y.copy()
            kinds.append("exact")
        else:
            idx, st = pick_index(cdf, st, c)
            picks.append(idx)
            cols, w = sharded_weights(cdf, idx)
            dx = (np.asarray(x, F32) - x_memo).astype(F64)
            y = np.zeros(m, F32)
            for r, (a, b) in enumerate(bounds):
                sel = (cols >= a) & (cols < b)
                As = A[:, cols[sel]].astype(F64)
                tmp = ((As.T @ dx).astype(F32) * w[sel]).astype(F32)
                part = (y_memo.astype(F64) if r == 0 else 0.0) + As @ tmp.astype(F64)
                y = (y + part.astype(F32)).astype(F32)
            kinds.append("previous")
        lam, _, _, x = dot_product_and_generate_x(x, y)
        eigs.append(lam)
    return np.array(eigs), kinds, st, cdf, picks


# --------------------------------------------------------------------------------------------
# Extensions: FP64 truth and the gradient of λ_max
# --------------------------------------------------------------------------------------------

def lambda_max_f64(A) -> float:
    """λ_max(A·Aᵀ) by FP64 LAPACK ``syevd`` on C (the same call calculate_largest_eigenvalue.py:
    1-13 makes on its matrix, via numpy ``eigh``)."""
    A64 = np.asarray(A, dtype=F64)
    C = A64 @ A64.T
    return float(np.linalg.eigvalsh(C)[-1])


def grad_lambda(A, v) -> np.ndarray:
    """∂λ_max/∂A = 2·v·(vᵀA) for a unit top eigenvector v of A·Aᵀ (FP64)."""
    A64 = np.asarray(A, dtype=F64)
    v64 = np.asarray(v, dtype=F64)
    v64 = v64 / np.linalg.norm(v64)
    return 2.0 * np.outer(v64, v64 @ A64)
