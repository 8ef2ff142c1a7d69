"""The headline workload at its full size: A 16384 x 65536 stored as BF16 (2 GiB), c = 4096.

At this size the oracle checks what holds column by column or pick by pick:

* the column statistics (α_j, ‖A_j‖, ‖A_j − α_j‖) and z = A·α, v = z − ‖α‖² of all 65536
  columns against FP64 sums of the same BF16 values (the tolerances of the small shapes);
* the 4096 picks of both weightings, bit for bit, given the library's own CDF;
* the proposed-AMM power method with the bench's schedule (variance reduction every 6 steps,
  7 steps: one exact step, at step 5, as the reference's rule places it) within 1e-3 of an FP64
  power method on the FP32 matrix, and the exact BF16 power method within 1e-3 after 7 steps.

The matrix and start vector are the bench's (seed 2024), built in host memory (4 GiB FP32).
"""
import numpy as np
import pytest
import torch

import amm_oracle as O
from helpers import states, vec_rel

pytestmark = pytest.mark.gpu

M, N, C = 16384, 65536, 4096
SEED = 2024
CHUNK = 4096


def _fp64_power(A32, x0, iters=400):
    """FP64 power method on the GPU (test infrastructure), as the bench's truth."""
    A64 = A32.double()
    x = x0.double() / x0.double().norm()
    lam_prev = 0.0
    for it in range(iters):
        y = A64 @ (A64.t() @ x)
        lam = float(x @ y)
        x = y / y.norm()
        if it > 10 and abs(lam - lam_prev) <= 1e-14 * abs(lam):
            break
        lam_prev = lam
    del A64
    torch.cuda.empty_cache()
    return lam


def test_full_size_bf16_headline_workload():
    import bench
    from eigenvaluecomputation_by_amm_b200 import AMMContext

    At = bench.make_matrix(M, N, SEED)
    x0 = torch.from_numpy(bench.start_vector(M, SEED)).cuda()
    At_d = torch.from_numpy(At).cuda()
    del At
    A32 = At_d.t()
    A16 = At_d.to(torch.bfloat16).t()  # (M, N) column-major

    ctx = AMMContext(M, N, c=C, step=7, vr_period=6, dtype="bf16")
    ctx.set_matrix(A16)
    st = ctx.column_stats()

    # column statistics and z = A·α over column chunks of the same BF16 values, FP64 sums
    alpha = np.empty(N, np.float32)
    norm = np.empty(N, np.float32)
    normp = np.empty(N, np.float32)
    z64 = np.zeros(M, np.float64)
    for j0 in range(0, N, CHUNK):
        blk = A16[:, j0:j0 + CHUNK].float().cpu().numpy()
        a, nr, npr = O.get_norms(blk)
        alpha[j0:j0 + CHUNK], norm[j0:j0 + CHUNK], normp[j0:j0 + CHUNK] = a, nr, npr
        z64 += blk.astype(np.float64) @ a.astype(np.float64)
    np.testing.assert_allclose(st["alpha"].cpu().numpy(), alpha, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(st["norm"].cpu().numpy(), norm, rtol=1e-6)
    np.testing.assert_allclose(st["normp"].cpu().numpy(), normp, rtol=1e-5)
    a2 = O.alpha_squared(alpha)
    assert abs(st["alpha2"] - a2) <= 1e-6 * a2
    z = z64.astype(np.float32)
    v = (z.astype(np.float64) - a2).astype(np.float32)
    assert vec_rel(st["z"].cpu().numpy(), z) < 1e-5
    assert vec_rel(st["v"].cpu().numpy(), v) < 1e-5

    # the picks of both weightings, bit-exact given the library's CDF
    s0 = states(C, SEED + 7)
    ctx.set_rng_state(torch.from_numpy(s0.view(np.int32)).cuda())
    for which in (0, 1):
        gcdf, _ = ctx.sampling_tables(which)
        got = ctx.sample_indices(which).cpu().numpy().view(np.uint32)
        want, _ = O.pick_index(gcdf.cpu().numpy(), s0, C)
        assert np.array_equal(got, want)

    # the power methods against the FP64 truth
    lam_true = _fp64_power(A32, x0)
    ctx.set_rng_state(torch.from_numpy(s0.view(np.int32)).cuda())
    ctx.power_method("proposed", x0)
    tr = ctx.trace()
    assert tr["kinds"] == ["proposed"] * 5 + ["exact"] + ["proposed"]
    assert abs(tr["eigs"][-1] - lam_true) <= 1e-3 * lam_true
    ctx.power_method("exact", x0)
    tr = ctx.trace()
    assert tr["steps_run"] == 7
    assert abs(tr["eigs"][-1] - lam_true) <= 1e-3 * lam_true
    ctx.close()
