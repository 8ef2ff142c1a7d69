"""CPU checks of the oracle (oracle/amm_oracle.py) itself: known answers, properties and the
reference's own -sanity mode.  The golden-vector pins live in test_golden.py."""
import numpy as np
import pytest

import amm_oracle as O


def _py_xorshift(y):
    y ^= (y << 13) & 0xFFFFFFFF
    y ^= (y >> 17)
    y ^= (y << 5) & 0xFFFFFFFF
    return y & 0xFFFFFFFF


def test_xorshift_matches_scalar_restatement():
    rng = np.random.default_rng(0)
    st = rng.integers(0, 2**32, size=1000, dtype=np.uint64).astype(np.uint32)
    st[:3] = [0, 1, 0xFFFFFFFF]
    new, u = O.xorshift32(st)
    for k in range(len(st)):
        y = _py_xorshift(int(st[k]))
        assert int(new[k]) == y
        mant = y & 0x7FFFFF
        assert float(u[k]) == float(np.float32(mant / 2.0**23))
    assert int(new[0]) == 0            # the zero state is a fixed point
    assert np.all((u >= 0) & (u < 1))


def _linear_pick(cdf, target):
    for i in range(len(cdf)):
        if cdf[i] > target:
            return i
    return len(cdf) - 1


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_pick_index_equals_first_greater(dtype):
    rng = np.random.default_rng(1)
    for n in (1, 2, 7, 33, 100):
        w = rng.exponential(size=n).astype(np.float32)
        w[rng.random(n) < 0.3] = 0.0          # zero-weight columns are never picked
        if w.sum() == 0:
            w[0] = 1.0
        cdf = O.cdf_f32(w) if dtype == np.float32 else O.cdf_f64(w)
        st = rng.integers(1, 2**32, size=50, dtype=np.uint64).astype(np.uint32)
        idx, new = O.pick_index(cdf, st, 50)
        _, u = O.xorshift32(st)
        for k in range(50):
            if dtype == np.float32:
                target = np.float32(cdf[-1]) * u[k]
            else:
                target = np.float64(cdf[-1]) * np.float64(u[k])
            assert idx[k] == _linear_pick(cdf, target)
            assert w[idx[k]] > 0
        assert np.array_equal(new[:50], O.xorshift32(st)[0])


def test_pick_index_clamps_when_target_reaches_total():
    cdf = np.array([0.0, 0.0, 0.0], dtype=np.float32)      # total 0: no cdf[i] > 0
    idx, _ = O.pick_index(cdf, np.array([12345], np.uint32), 1)
    assert idx[0] == 2


def test_sanity_mode_equals_exact():
    """The reference's -sanity known answer (host_memory.h:103-106, device_memory.h:500-551):
    with c == n, weights 1 and indices 0..n-1 every AMM step is the exact product."""
    rng = np.random.default_rng(2)
    m, n = 32, 48
    A = (rng.standard_normal((m, n)) * rng.lognormal(0, 1, n)).astype(np.float32)
    x0 = rng.standard_normal(m).astype(np.float32)
    ex = O.power_method(A, x0, method="exact", step=6)
    for method in ("previous", "proposed"):
        tr = O.power_method(A, x0, method=method, step=6, c=n, sanity=True)
        np.testing.assert_allclose(tr.eigs, ex.eigs, rtol=2e-6)


def test_proposed_decomposition_is_exact_with_all_columns():
    rng = np.random.default_rng(3)
    m, n = 24, 40
    A = (rng.standard_normal((m, n)) + 0.7).astype(np.float32)
    alpha, norm, normp = O.get_norms(A)
    z, v = O.generate_zv(A, alpha, O.alpha_squared(alpha))
    x = O.normalize(rng.standard_normal(m).astype(np.float32))
    xm = O.normalize(rng.standard_normal(m).astype(np.float32))
    ym = rng.standard_normal(m).astype(np.float32)
    idx = np.arange(n, dtype=np.uint32)
    w = np.ones(n, np.float32)
    _, y = O.proposed_amm(A, alpha, x, xm, ym, idx, w, z, v)
    expect = ym.astype(np.float64) + A.astype(np.float64) @ (A.astype(np.float64).T @ (x - xm).astype(np.float64))
    np.testing.assert_allclose(y, expect, rtol=1e-4, atol=1e-4 * np.abs(expect).max())


@pytest.mark.parametrize("which", ["previous", "proposed"])
def test_amm_products_are_unbiased(which):
    rng = np.random.default_rng(4)
    m, n, c = 16, 64, 16
    A = (rng.standard_normal((m, n)) * rng.lognormal(0, 0.5, n) + 0.3).astype(np.float32)
    alpha, norm, normp = O.get_norms(A)
    z, v = O.generate_zv(A, alpha, O.alpha_squared(alpha))
    x = O.normalize(rng.standard_normal(m).astype(np.float32))
    zero = np.zeros(m, np.float32)
    cdf, w = O._sampling_tables(A, "norm" if which == "previous" else "normp", c, n, "f64", False, None)
    st = rng.integers(1, 2**32, size=c, dtype=np.uint64).astype(np.uint32)
    acc = np.zeros(m)
    reps = 3000
    for _ in range(reps):
        idx, st = O.sample_sorted(cdf, st, c)
        if which == "previous":
            _, y = O.previous_amm(A, x, zero, zero, idx, w)
        else:
            _, y = O.proposed_amm(A, alpha, x, zero, zero, idx, w, z, v)
        acc += y
    exact = O.exact_product(A, x).astype(np.float64)
    err = np.linalg.norm(acc / reps - exact) / np.linalg.norm(exact)
    assert err < 0.03


def test_exact_power_method_converges_to_eigvalsh():
    rng = np.random.default_rng(5)
    m, n = 64, 256
    A = (rng.standard_normal((m, n)) * rng.lognormal(0, 1, n)).astype(np.float32)
    x0 = rng.standard_normal(m).astype(np.float32)
    tr = O.power_method(A, x0, method="exact", step=200)
    lam = O.lambda_max_f64(A)
    assert abs(tr.eigs[-1] - lam) / lam < 1e-5


def test_variance_reduction_schedule():
    """VR steps land where the reference's drivers put them."""
    rng = np.random.default_rng(6)
    m, n, c = 16, 64, 16
    A = rng.standard_normal((m, n)).astype(np.float32)
    x0 = rng.standard_normal(m).astype(np.float32)
    st = rng.integers(1, 2**32, size=c, dtype=np.uint64).astype(np.uint32)
    tr = O.power_method(A, x0, method="previous", step=9, c=c, states=st, vr_period=3)
    assert [i for i, k in enumerate(tr.modes) if k == "exact"] == [2, 5, 8]
    tr = O.power_method(A, x0, method="proposed", step=9, c=c, states=st, vr_period=2)
    # i=1 is skipped (needs i > last_exact + 1 = 1); then 3, 5, 7
    assert [i for i, k in enumerate(tr.modes) if k == "exact"] == [3, 5, 7]
    tr = O.power_method(A, x0, method="proposed_v2", step=10, c=c, states=st, vr_period=4)
    assert tr.modes[:4] == ["previous"] * 3 + ["exact_nomemo"]
    assert tr.modes[7] == "exact" and tr.modes[4:7] == ["proposed"] * 3
    with pytest.raises(ValueError):
        O.power_method(A, x0, method="proposed_v2", step=3, c=c, states=st, vr_period=4)


def test_states_advance_once_per_amm_sample():
    rng = np.random.default_rng(7)
    m, n, c = 8, 32, 8
    A = rng.standard_normal((m, n)).astype(np.float32)
    x0 = rng.standard_normal(m).astype(np.float32)
    st = rng.integers(1, 2**32, size=c, dtype=np.uint64).astype(np.uint32)
    tr = O.power_method(A, x0, method="previous", step=5, c=c, states=st, vr_period=5)
    expect = st.copy()
    for _ in range(4):                     # 4 AMM steps, one VR step
        expect, _ = O.xorshift32(expect)
    assert np.array_equal(tr.states, expect)


def test_grad_lambda_matches_finite_differences():
    rng = np.random.default_rng(8)
    m, n = 12, 30
    A = rng.standard_normal((m, n)) * rng.lognormal(0, 0.5, n)
    w, V = np.linalg.eigh(A @ A.T)
    g = O.grad_lambda(A, V[:, -1])
    h = 1e-6
    for (i, j) in [(0, 0), (3, 7), (11, 29), (5, 12)]:
        Ap, Am = A.copy(), A.copy()
        Ap[i, j] += h
        Am[i, j] -= h
        fd = (O.lambda_max_f64(Ap) - O.lambda_max_f64(Am)) / (2 * h)
        assert abs(fd - g[i, j]) <= 1e-5 * max(1.0, abs(fd))
