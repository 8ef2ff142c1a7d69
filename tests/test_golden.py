"""CPU pins of the oracle against golden vectors produced by the REFERENCE's own kernels and
drivers (tests/golden/ref_golden.npz, generated on a B200 by tests/golden/make_golden.py from
oracle/_ref, which is compiled from the reference sources).  Inputs are regenerated from the
seeds in tests/golden/inputs.py."""
import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))

import inputs as I  # noqa: E402
import amm_oracle as O  # noqa: E402

GOLD = HERE / "golden" / "ref_golden.npz"
pytestmark = pytest.mark.skipif(not GOLD.exists(), reason="golden fixtures not generated yet")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLD))


def test_pick_index_bit_exact(g):
    cdf, st = I.pick_inputs()
    idx, new = O.pick_index(cdf, st, len(st))
    assert np.array_equal(idx, g["pick_idx"])
    assert np.array_equal(new, g["pick_states"])


def test_column_stats_match_reference(g):
    A = I.symmetric_matrix()
    alpha, norm, normp = O.get_norms(A)
    np.testing.assert_allclose(norm, g["run_exact_norm"], rtol=1e-6)
    np.testing.assert_allclose(normp, g["run_exact_normp"], rtol=1e-5)
    np.testing.assert_allclose(alpha, g["run_exact_alpha"], rtol=1e-6, atol=1e-8)


@pytest.mark.parametrize("kernel,which", [("previousAMM", "norm"), ("proposedAMM", "normp")])
def test_step_by_step(g, kernel, which):
    A = I.symmetric_matrix()
    st = I.states()
    x = O.normalize(I.start_vector())
    ref_cdf = g[f"steps_{kernel}_cdf"]
    # the reference's CUB-built CDF is within a few ulps of the correctly rounded one
    own = O.cdf_f32(O.set_weights(O.get_norms(A)[1 if which == "norm" else 2]))
    ulps = np.abs(own.view(np.int32).astype(np.int64) - ref_cdf.view(np.int32).astype(np.int64))
    assert ulps.max() <= 4
    cdf, w = O._sampling_tables(A, which, I.C, I.M, "f32", False, {which: ref_cdf})
    np.testing.assert_allclose(w, g[f"steps_{kernel}_weight"], rtol=4e-7)
    alpha, _, _ = O.get_norms(A)
    z, v = O.generate_zv(A, alpha, O.alpha_squared(alpha))
    zero = np.zeros(I.M, np.float32)
    for i in range(I.NSTEPS):
        idx, st = O.sample_sorted(cdf, st, I.C)
        assert np.array_equal(idx, g[f"steps_{kernel}_sorted"][i]), f"step {i}"
        if kernel == "previousAMM":
            tmp, y = O.previous_amm(A, x, zero, zero, idx, w)
        else:
            tmp, y = O.proposed_amm(A, alpha, x, zero, zero, idx, w, z, v)
        assert np.linalg.norm(y - g[f"steps_{kernel}_y"][i]) <= 1e-5 * np.linalg.norm(y)
        np.testing.assert_allclose(tmp, g[f"steps_{kernel}_tmp"][i], rtol=1e-3,
                                   atol=1e-5 * np.abs(tmp).max())
        lam, _, _, x = O.dot_product_and_generate_x(x, y)
        assert abs(lam - g[f"steps_{kernel}_eigs"][i]) <= 2e-5 * abs(lam)
    assert np.array_equal(st[:I.C], g[f"steps_{kernel}_states"][:I.C])


@pytest.mark.parametrize("kernel", ["previousAMM", "proposedAMM"])
def test_sanity_known_answer(g, kernel):
    A = I.symmetric_matrix()
    tr = O.power_method(A, I.start_vector(), method="exact", step=3)
    np.testing.assert_allclose(g[f"sanity_{kernel}_eigs"], tr.eigs, rtol=2e-5)


RUNS = {
    "exact": ("exact", dict()),
    "previousAMM": ("previous", dict(vr_period=I.VR)),
    "proposedAMM": ("proposed", dict(vr_period=I.VR)),
    "proposedAMM_v2": ("proposed_v2", dict(vr_period=I.VR)),
    "previousAMM_adaptive": ("previous", dict(vr_adaptive_threshold=1e-3)),
}


@pytest.mark.parametrize("name", list(RUNS))
def test_power_method_runs(g, name):
    """The reference's own drivers: λ per step, err per step, advanced states."""
    method, kw = RUNS[name]
    A = I.symmetric_matrix()
    st = I.states()
    x0 = g["x0_seed_1276"]
    vstar = I.top_eigenvector(A)
    over = {}
    if method in ("previous",):
        over["norm"] = g[f"run_{name}_cdf"]
    elif method == "proposed":
        over["normp"] = g[f"run_{name}_cdf"]
    elif method == "proposed_v2":
        over["normp"] = g[f"run_{name}_cdf"]
    tr = O.power_method(A, x0, method=method, step=I.STEPS, c=I.C, states=st, vstar=vstar,
                        cdf_precision="f32", cdf_override=over, **kw)
    ref = g[f"run_{name}_eigs"]
    np.testing.assert_allclose(tr.eigs, ref, rtol=1e-4)
    np.testing.assert_allclose(tr.errs, g[f"run_{name}_errs"], atol=1e-4)
    assert np.array_equal(tr.states[:I.C], g[f"run_{name}_states"][:I.C])
    # the reference reports sqrt(λ) - offset with offset 0 in the harness
    assert np.all(np.isfinite(O.reported_eigenvalue(ref)))
