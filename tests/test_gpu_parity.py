"""GPU parity of libamm (called through the C ABI) against the oracle on seeded inputs.

Integer work (xorshift states, sampled indices) must match bit for bit; floating-point results
must match within the FP32 tolerances stated in helpers.py.
"""
import numpy as np
import pytest
import torch

import amm_oracle as O
from helpers import RTOL_LAMBDA_F32, RTOL_VEC_F32, rel, scaled_gaussian, states, vec_rel

pytestmark = pytest.mark.gpu


def ctx_for(A, c=0, step=10, dtype="f32", cdf="f64", **kw):
    from eigenvaluecomputation_by_amm_b200 import AMMContext, column_major
    m, n = A.shape
    ctx = AMMContext(m, n, c=c, step=step, dtype=dtype, cdf_precision=cdf, **kw)
    tA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    if dtype == "bf16":
        tA = tA.to(torch.bfloat16)
    ctx.set_matrix(column_major(tA))
    return ctx


def t32(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def tu32(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()


def np_u32(t):
    return t.cpu().numpy().view(np.uint32)


SHAPES = [(64, 256), (512, 2048), (1024, 4096), (4096, 1024)]


@pytest.mark.parametrize("m,n", SHAPES)
def test_column_stats(m, n):
    A = scaled_gaussian(m, n, seed=m + n, shift=0.2)
    ctx = ctx_for(A)
    st = ctx.column_stats()
    alpha, norm, normp = O.get_norms(A)
    np.testing.assert_allclose(st["alpha"].cpu().numpy(), alpha, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(st["norm"].cpu().numpy(), norm, rtol=1e-6)
    np.testing.assert_allclose(st["normp"].cpu().numpy(), normp, rtol=1e-5)
    a2 = O.alpha_squared(alpha)
    assert abs(st["alpha2"] - a2) <= 1e-6 * a2  # FP32 α_j, accumulated in FP64
    z, v = O.generate_zv(A, alpha, a2)
    assert vec_rel(st["z"].cpu().numpy(), z) < 1e-5
    assert vec_rel(st["v"].cpu().numpy(), v) < 1e-5


@pytest.mark.parametrize("cdf", ["f64", "f32"])
def test_cdf_and_weights(cdf):
    A = scaled_gaussian(256, 3000, seed=3, shift=0.1)
    c = 200
    ctx = ctx_for(A, c=c, cdf=cdf)
    # the tables are a function of the library's own column norms (checked against the oracle
    # in test_column_stats); FP32 norms may differ from the oracle's in the last bit
    stats = ctx.column_stats()
    norm, normp = stats["norm"].cpu().numpy(), stats["normp"].cpu().numpy()
    for which, base in ((0, norm), (1, normp)):
        gcdf, gw = ctx.sampling_tables(which)
        gcdf = gcdf.cpu().numpy()
        weight = O.set_weights(base)
        if cdf == "f64":
            ocdf = O.cdf_f64(base.astype(np.float64) ** 2)
            np.testing.assert_allclose(gcdf, ocdf, rtol=1e-11)
            ow = O.update_weights(base.astype(np.float64) ** 2, ocdf[-1], c, "f64")
        else:
            ocdf = O.cdf_f32(weight)
            ulps = np.abs(gcdf.view(np.int32).astype(np.int64) - ocdf.view(np.int32).astype(np.int64))
            assert ulps.max() <= 1
            ow = O.update_weights(weight, gcdf[-1], c, "f32")
        np.testing.assert_allclose(gw.cpu().numpy(), ow, rtol=2e-7)


@pytest.mark.parametrize("cdf", ["f64", "f32"])
@pytest.mark.parametrize("n", [1, 31, 32, 1000, 65536, 100003])
def test_sampler_bit_exact(cdf, n):
    """pick_index (device_memory.h:516-545): same CDF + same states -> same indices and states."""
    rng = np.random.default_rng(n)
    m = 64
    A = scaled_gaussian(m, n, seed=n, sigma=2.0)
    A[:, rng.random(n) < 0.05] = 0.0               # zero columns: never picked
    if not A.any():
        A[0, 0] = 1.0
    c = 4096
    ctx = ctx_for(A, c=c, cdf=cdf)
    st = states(c, seed=n + 1)
    ctx.set_rng_state(tu32(st))
    for which in (0, 1):
        gcdf, _ = ctx.sampling_tables(which)
        gcdf = gcdf.cpu().numpy()
        got = np_u32(ctx.sample_indices(which))
        want, _ = O.pick_index(gcdf, st, c)
        assert np.array_equal(got, want)
        assert np.all(np.any(A[:, got] != 0, axis=0))


def test_sampler_with_imported_cdf_and_ties():
    """An imported FP32 CDF with flat runs (zero weights) and a duplicated total."""
    n, c = 5000, 2048
    rng = np.random.default_rng(9)
    w = rng.lognormal(0, 2, n).astype(np.float32)
    w[rng.random(n) < 0.3] = 0
    w[-50:] = 0
    cdf32 = np.cumsum(w.astype(np.float64)).astype(np.float32)
    A = scaled_gaussian(64, n, seed=1)
    ctx = ctx_for(A, c=c, cdf="f32")
    ctx.set_cdf(0, torch.from_numpy(cdf32))
    st = states(c, 10)
    ctx.set_rng_state(tu32(st))
    got = np_u32(ctx.sample_indices(0))
    want, _ = O.pick_index(cdf32, st, c)
    assert np.array_equal(got, want)


def _oracle_tables(A, c, cdf):
    return {w: O._sampling_tables(A, w, c, A.shape[1], cdf, False, None) for w in ("norm", "normp")}


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
@pytest.mark.parametrize("method", ["previous", "proposed"])
def test_single_product(method, dtype):
    m, n, c = 512, 4096, 700
    A = scaled_gaussian(m, n, seed=21, shift=0.3)
    if dtype == "bf16":
        A = torch.from_numpy(A).to(torch.bfloat16).float().numpy()
    ctx = ctx_for(A, c=c, dtype=dtype)
    st = states(c, 22)
    ctx.set_rng_state(tu32(st))
    rng = np.random.default_rng(23)
    x = O.normalize(rng.standard_normal(m).astype(np.float32))
    xm = O.normalize(rng.standard_normal(m).astype(np.float32))
    ym = (rng.standard_normal(m) * 100).astype(np.float32)
    which = "norm" if method == "previous" else "normp"
    ocdf, ow = _oracle_tables(A, c, "f64")[which]
    oidx, ost = O.sample_sorted(ocdf, st, c)
    if method == "previous":
        y, idx = ctx.core_previousAMM(t32(x), t32(xm), t32(ym))
        _, oy = O.previous_amm(A, x, xm, ym, oidx, ow)
    else:
        y, idx = ctx.core_proposedAMM(t32(x), t32(xm), t32(ym))
        alpha, _, _ = O.get_norms(A)
        z, v = O.generate_zv(A, alpha, O.alpha_squared(alpha))
        _, oy = O.proposed_amm(A, alpha, x, xm, ym, oidx, ow, z, v)
    assert np.array_equal(np_u32(idx), oidx)
    assert vec_rel(y.cpu().numpy(), oy) < RTOL_VEC_F32
    assert np.array_equal(np_u32(ctx.get_rng_state(c)), ost[:c])


@pytest.mark.parametrize("m,n", [(64, 256), (1024, 4096), (16384, 512)])
def test_exact_product(m, n):
    A = scaled_gaussian(m, n, seed=31)
    ctx = ctx_for(A)
    x = np.random.default_rng(32).standard_normal(m).astype(np.float32)
    y = ctx.exact_product(t32(x)).cpu().numpy()
    assert vec_rel(y, O.exact_product(A, x)) < RTOL_VEC_F32


RUNS = [
    ("exact", dict()),
    ("previous", dict()),
    ("previous", dict(vr_period=4)),
    ("proposed", dict(vr_period=3)),
    ("proposed", dict()),
    ("proposed_v2", dict(vr_period=5)),
    ("proposed_v2", dict(vr_period=1)),
]


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("method,kw", RUNS)
def test_power_method_trace(method, kw, use_graph):
    m, n, c, step = 512, 2048, 256, 16
    A = scaled_gaussian(m, n, seed=41, shift=0.05)
    ctx = ctx_for(A, c=c, step=step, use_graph=use_graph, **kw)
    st = states(c, 42)
    ctx.set_rng_state(tu32(st))
    x0 = np.random.default_rng(43).standard_normal(m).astype(np.float32)
    vstar = np.linalg.eigh(A.astype(np.float64) @ A.astype(np.float64).T)[1][:, -1]
    ctx.set_eigenvector(torch.from_numpy(vstar))
    ctx.power_method(method, t32(x0))
    tr = ctx.trace()
    ref = O.power_method(A, x0, method=method, step=step, c=c, states=st, vstar=vstar, **kw)
    assert tr["steps_run"] == step
    assert tr["kinds"] == ref.modes
    assert np.all(rel(tr["eigs"], ref.eigs) < RTOL_LAMBDA_F32), (tr["eigs"], ref.eigs)
    assert np.all(np.abs(tr["errs"] - ref.errs) < 1e-4)
    assert np.all(np.abs(tr["coss"] - ref.coss) < 1e-5)
    assert np.array_equal(np_u32(ctx.get_rng_state(c)), ref.states[:c])
    x, y = ctx.vectors()
    assert vec_rel(x.cpu().numpy(), ref.x) < 1e-4


@pytest.mark.parametrize("method,kw", [("previous", dict(vr_period=4)),
                                       ("proposed", dict(vr_period=7)),
                                       ("proposed", dict(vr_adaptive_threshold=1e-2)),
                                       ("proposed_v2", dict(vr_period=5))])
def test_power_method_trace_many_windows(method, kw):
    """40 steps: the work lists are drawn 16 AMM steps at a time, so the call refills its list
    window twice and reuses every slot; the trace, kinds and final states still follow the
    oracle step for step."""
    m, n, c, step = 512, 2048, 256, 40
    A = scaled_gaussian(m, n, seed=51, shift=0.05)
    ctx = ctx_for(A, c=c, step=step, **kw)
    st = states(c, 52)
    ctx.set_rng_state(tu32(st))
    x0 = np.random.default_rng(53).standard_normal(m).astype(np.float32)
    vstar = np.linalg.eigh(A.astype(np.float64) @ A.astype(np.float64).T)[1][:, -1]
    ctx.set_eigenvector(torch.from_numpy(vstar))
    ctx.power_method(method, t32(x0))
    tr = ctx.trace()
    ref = O.power_method(A, x0, method=method, step=step, c=c, states=st, vstar=vstar, **kw)
    thr = kw.get("vr_adaptive_threshold", 0.0)
    if thr and np.min(np.abs(ref.coss - (1 - thr))) < 1e-6:
        pytest.skip("a cos lies within FP32 noise of the threshold")
    assert tr["steps_run"] == step
    assert tr["kinds"] == ref.modes
    assert sum(k != "exact" for k in ref.modes) > 16
    assert np.all(rel(tr["eigs"], ref.eigs) < RTOL_LAMBDA_F32), (tr["eigs"], ref.eigs)
    assert np.array_equal(np_u32(ctx.get_rng_state(c)), ref.states[:c])


EDGE_SHAPES = [(4, 1, 1), (8, 3, 5), (12, 37, 37), (1028, 513, 64), (16, 100003, 4096)]


@pytest.mark.parametrize("m,n,c", EDGE_SHAPES)
@pytest.mark.parametrize("method,kw", [("exact", dict()), ("previous", dict(vr_period=2)),
                                       ("proposed", dict(vr_period=3)),
                                       ("proposed_v2", dict(vr_period=2))])
def test_power_method_edge_shapes(m, n, c, method, kw):
    """One column, more picks than columns, ragged row and column counts, many short columns:
    the trace (λ, kinds), the advanced states and the final vector against the oracle."""
    step = 6
    A = scaled_gaussian(m, n, seed=m * 7 + n, shift=0.05)
    ctx = ctx_for(A, c=c, step=step, **kw)
    st = states(c, m + n + c)
    ctx.set_rng_state(tu32(st))
    x0 = np.random.default_rng(m + 3).standard_normal(m).astype(np.float32)
    ctx.power_method(method, t32(x0))
    tr = ctx.trace()
    ref = O.power_method(A, x0, method=method, step=step, c=c, states=st, **kw)
    assert tr["steps_run"] == step
    assert tr["kinds"] == ref.modes
    assert np.all(rel(tr["eigs"], ref.eigs) < RTOL_LAMBDA_F32), (tr["eigs"], ref.eigs)
    assert np.array_equal(np_u32(ctx.get_rng_state(c)), ref.states[:c])
    x, _ = ctx.vectors()
    assert vec_rel(x.cpu().numpy(), ref.x) < 1e-4
    ctx.close()


def test_adaptive_variance_reduction():
    m, n, c, step, thr = 512, 2048, 256, 24, 2e-3
    A = scaled_gaussian(m, n, seed=51)
    x0 = np.random.default_rng(52).standard_normal(m).astype(np.float32)
    st = states(c, 53)
    ref = O.power_method(A, x0, method="previous", step=step, c=c, states=st,
                         vr_adaptive_threshold=thr)
    margin = np.min(np.abs(ref.coss - (1 - thr)))
    if margin < 1e-6:
        pytest.skip("a cos lies within FP32 noise of the threshold")
    ctx = ctx_for(A, c=c, step=step, vr_adaptive_threshold=thr)
    ctx.set_rng_state(tu32(st))
    ctx.power_method("previous", t32(x0))
    tr = ctx.trace()
    assert tr["kinds"] == ref.modes
    assert "exact" in ref.modes
    assert np.all(rel(tr["eigs"], ref.eigs) < RTOL_LAMBDA_F32)


@pytest.mark.parametrize("method", ["previous", "proposed"])
def test_sanity_mode_known_answer(method):
    """-sanity with c == n: every AMM step is the exact product (host_memory.h:103-106)."""
    m, n, step = 256, 1024, 8
    A = scaled_gaussian(m, n, seed=61, shift=0.4)
    x0 = np.random.default_rng(62).standard_normal(m).astype(np.float32)
    ctx = ctx_for(A, c=n, step=step, sanity=True)
    ctx.power_method(method, t32(x0))
    tr = ctx.trace()
    ex = ctx_for(A, c=n, step=step)
    ex.power_method("exact", t32(x0))
    tex = ex.trace()
    assert np.all(rel(tr["eigs"], tex["eigs"]) < 1e-5)
    assert set(tr["distinct"]) == {n}


def test_bf16_storage_power_method():
    m, n, c, step = 1024, 8192, 512, 12
    A = scaled_gaussian(m, n, seed=71)
    Ab = torch.from_numpy(A).to(torch.bfloat16).float().numpy()
    ctx = ctx_for(A, c=c, step=step, dtype="bf16", vr_period=4)
    st = states(c, 72)
    ctx.set_rng_state(tu32(st))
    x0 = np.random.default_rng(73).standard_normal(m).astype(np.float32)
    ctx.power_method("proposed", t32(x0))
    tr = ctx.trace()
    ref = O.power_method(Ab, x0, method="proposed", step=step, c=c, states=st, vr_period=4)
    assert tr["kinds"] == ref.modes
    assert np.all(rel(tr["eigs"], ref.eigs) < RTOL_LAMBDA_F32)


def test_exact_fp32_lambda_matches_fp64_eigvalsh():
    """1024 x 4096, N(0,1) x lognormal(0,1) columns, seed 0; x0 ~ N(0,1) seed 1; 200 steps."""
    rng = np.random.default_rng(0)
    A = (rng.standard_normal((1024, 4096)) * rng.lognormal(0, 1, 4096)).astype(np.float32)
    x0 = np.random.default_rng(1).standard_normal(1024).astype(np.float32)
    ctx = ctx_for(A, step=200)
    ctx.power_method("exact", t32(x0))
    tr = ctx.trace()
    lam = O.lambda_max_f64(A)
    assert rel(tr["eigs"][-1], lam) < 1e-5


@pytest.mark.parametrize("use_graph", [True, False])
def test_runs_are_deterministic(use_graph):
    m, n, c, step = 512, 4096, 300, 10
    A = scaled_gaussian(m, n, seed=81)
    x0 = t32(np.random.default_rng(82).standard_normal(m))
    out = []
    for _ in range(2):
        ctx = ctx_for(A, c=c, step=step, vr_period=3, use_graph=use_graph)
        ctx.set_rng_state(tu32(states(c, 83)))
        ctx.power_method("proposed", x0)
        out.append(ctx.trace()["eigs"])
        ctx.power_method("proposed", x0)       # a second call continues the states
        out.append(ctx.trace()["eigs"])
    assert np.array_equal(out[0], out[2]) and np.array_equal(out[1], out[3])
    assert not np.array_equal(out[0], out[1])


@pytest.mark.parametrize("method", ["previous", "proposed", "proposed_v2"])
def test_every_call_starts_from_a_zero_memo(method):
    """Each call restarts like the reference (zero_clear): repeated calls on one context with
    the same states and start vector give the same trace, equal to the oracle's."""
    m, n, c, step = 512, 4096, 256, 9
    A = scaled_gaussian(m, n, seed=85)
    x0 = np.random.default_rng(86).standard_normal(m).astype(np.float32)
    st = states(c, 87)
    ctx = ctx_for(A, c=c, step=step, vr_period=3)
    traces = []
    for _ in range(4):
        ctx.set_rng_state(tu32(st))
        ctx.power_method(method, t32(x0))
        traces.append(ctx.trace()["eigs"])
    for tr in traces[1:]:
        assert np.array_equal(tr, traces[0])
    ref = O.power_method(A, x0, method=method, step=step, c=c, states=st, vr_period=3)
    assert np.all(rel(traces[0], ref.eigs) < RTOL_LAMBDA_F32)


def test_grad_lambda_kernel():
    m, n = 256, 1024
    A = scaled_gaussian(m, n, seed=91)
    ctx = ctx_for(A)
    v = np.linalg.eigh(A.astype(np.float64) @ A.astype(np.float64).T)[1][:, -1]
    g = ctx.grad_lambda(t32(v)).cpu().numpy()
    assert vec_rel(g, O.grad_lambda(A, v)) < 1e-5


def test_rayleigh_and_normalize_helpers():
    m, n = 512, 512
    A = scaled_gaussian(m, n, seed=95)
    ctx = ctx_for(A)
    rng = np.random.default_rng(96)
    x = rng.standard_normal(m).astype(np.float32)
    tx = t32(x)
    ctx.normalize(tx)
    xn = O.normalize(x)
    assert vec_rel(tx.cpu().numpy(), xn) < 1e-6
    y = O.exact_product(A, xn)
    lam, err, cos = ctx.rayleigh_normalize(tx, t32(y))
    olam, oerr, ocos, oxn = O.dot_product_and_generate_x(xn, y)
    assert rel(lam, olam) < 1e-6 and abs(cos - ocos) < 1e-6
    assert vec_rel(tx.cpu().numpy(), oxn) < 1e-6


def test_error_paths():
    from eigenvaluecomputation_by_amm_b200 import AMMContext, AmmError, _lib
    with pytest.raises(AmmError) as e:
        AMMContext(130, 64)                               # m*4 not a multiple of 16
    assert e.value.status == _lib.AMM_ERR_ALIGNMENT
    with pytest.raises(AmmError) as e:
        AMMContext(32768, 64)
    assert e.value.status == _lib.AMM_ERR_UNSUPPORTED
    ctx = AMMContext(64, 128, step=3, vr_period=4)
    with pytest.raises(AmmError) as e:
        ctx.power_method("exact", torch.ones(64, device="cuda"))
    assert e.value.status == _lib.AMM_ERR_NOT_READY
    base = torch.zeros(66 * 128 + 1, device="cuda")
    Amis = base[1:1 + 66 * 128].view(128, 66).t()[:64, :]    # ld 66 floats: misaligned
    rc = ctx.lib.amm_set_matrix(ctx._ctx, Amis.data_ptr(), 66, None)
    assert rc == _lib.AMM_ERR_ALIGNMENT
    ctx.set_matrix(torch.randn(128, 64, device="cuda").t())
    with pytest.raises(AmmError) as e:
        ctx.power_method("proposed_v2", torch.ones(64, device="cuda"))  # step < vr_period
    assert e.value.status == _lib.AMM_ERR_INVALID_ARGUMENT
    Z = torch.zeros(128, 64, device="cuda").t()
    ctx.set_matrix(Z)                                     # all-zero A: degenerate CDF
    ctx.power_method("exact", torch.ones(64, device="cuda"))
    with pytest.raises(AmmError) as e:
        ctx.trace()
    assert e.value.status == _lib.AMM_ERR_DEGENERATE


def test_bounded_waits_give_up_and_the_context_stays_usable():
    """The device-side waits are bounded: a kernel waiting on an mbarrier that nothing arrives
    on and on a grid barrier one CTA short gives up after the wait limit (2 s each), the host
    reads AMM_ERR_DEVICE_TIMEOUT, and the same context then solves as a fresh one does."""
    import ctypes as C
    from eigenvaluecomputation_by_amm_b200 import _lib
    A = scaled_gaussian(256, 1024, seed=77, shift=0.1)
    x0 = torch.from_numpy(np.random.default_rng(78).standard_normal(256).astype(np.float32)).cuda()
    ref = ctx_for(A, c=128, step=6, vr_period=3)
    ref.set_rng_state(tu32(states(128, 79)))
    ref.power_method("proposed", x0)
    want = ref.trace()["eigs"]
    ctx = ctx_for(A, c=128, step=6, vr_period=3)
    out = (C.c_uint32 * 3)()
    rc = ctx.lib.amm_probe_bounded_waits(ctx._ctx, out, None)
    assert rc == _lib.AMM_ERR_DEVICE_TIMEOUT
    assert out[0] == 0 and out[1] == 0
    assert 3.9e6 <= out[2] <= 30e6                      # two waits of 2 s, in µs
    ctx.set_rng_state(tu32(states(128, 79)))
    ctx.power_method("proposed", x0)
    assert np.array_equal(ctx.trace()["eigs"], want)   # deterministic, as from a fresh context
    ref.close()
    ctx.close()


_KNOB_SCRIPT = r"""
import json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
from helpers import scaled_gaussian, states
from eigenvaluecomputation_by_amm_b200 import AMMContext, column_major
A = scaled_gaussian(512, 2048, seed=91, shift=0.05)
ctx = AMMContext(512, 2048, c=256, step=9, vr_period=4)
ctx.set_matrix(column_major(torch.from_numpy(A).cuda()))
ctx.set_rng_state(torch.from_numpy(states(256, 92).view(np.int32)).cuda())
x0 = torch.from_numpy(np.random.default_rng(93).standard_normal(512).astype(np.float32)).cuda()
ctx.power_method("proposed", x0)
tr = ctx.trace()
print(json.dumps({"eigs": tr["eigs"].tolist(), "kinds": tr["kinds"],
                  "states": ctx.get_rng_state(256).cpu().numpy().view(np.uint32).tolist(),
                  "geometry": ctx.geometry()}))
"""


@pytest.mark.parametrize("env", [{}, {"AMM_PDL": "0"}, {"AMM_PANEL_GC": "4"},
                                 {"AMM_PANEL_STAGES": "4", "AMM_PDL": "0"},
                                 {"AMM_PANEL_CLUSTER": "2"}, {"AMM_PANEL_CLUSTER": "4"},
                                 {"AMM_PANEL_CLUSTER": "4", "AMM_PDL": "0"}])
def test_launch_knobs_agree(env):
    """The environment knobs (no programmatic dependent launch, 4 instead of 8 columns per stage,
    a shallower ring, thread-block clusters that pre-sum their partial y through distributed
    shared memory) change only the launch shape: the same picks and step kinds, λ within the
    FP32 tolerance of the default configuration (run in separate processes: the knobs are read
    once per process)."""
    import json
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parents[1])

    def run(extra):
        e = dict(os.environ)
        for k in ("AMM_PDL", "AMM_PANEL_GC", "AMM_PANEL_STAGES", "AMM_PANEL_CLUSTER"):
            e.pop(k, None)
        e.update(extra)
        r = subprocess.run([sys.executable, "-c", _KNOB_SCRIPT, root], env=e, capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        return json.loads(r.stdout.strip().splitlines()[-1])

    base, got = run({}), run(env)
    assert got["kinds"] == base["kinds"]
    assert got["states"] == base["states"]
    assert np.all(rel(got["eigs"], base["eigs"]) < RTOL_LAMBDA_F32)
    if "AMM_PANEL_GC" in env:
        assert got["geometry"]["cols_per_stage"] == int(env["AMM_PANEL_GC"])
    if "AMM_PANEL_STAGES" in env:
        assert got["geometry"]["stages"] == int(env["AMM_PANEL_STAGES"])
    if "AMM_PANEL_CLUSTER" in env:
        assert got["geometry"]["cluster"] == int(env["AMM_PANEL_CLUSTER"])
        assert got["geometry"]["clusters"] * got["geometry"]["cluster"] >= 74
