"""Batched λ_max (amm_batch_*) and its backward, called through the C ABI.

The solver stops at a residual ‖C·v − λ·v‖ <= 1e-6·λ.  λ and v are compared with FP64 LAPACK
(numpy eigh on C = A·Aᵀ): λ_max within rtol 1e-5 for the 4- and 8-vector blocks and 1e-4 for
the single vector; the gradient 2·v(vᵀA) within 1e-4 (relative,
Frobenius) of FP64 torch.linalg.eigvalsh autograd and within 1e-3·max|g| of central finite
differences (h = 1e-3, FP64) on 32 entries.
"""
import ctypes as C

import numpy as np
import pytest
import torch

SIZES = [(64, 256), (70, 300), (128, 512), (333, 1000), (512, 2048), (1000, 700), (2048, 256)]


def _mats(sizes, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    out = []
    for m, n in sizes:
        A = rng.standard_normal((m, n)) * np.exp(scale * rng.standard_normal(n))[None, :]
        out.append(A.astype(np.float32))
    return out


def _device_col_major(A):
    m, n = A.shape
    ld = (m + 3) // 4 * 4
    buf = torch.zeros(n, ld, dtype=torch.float32, device="cuda")
    buf[:, :m] = torch.from_numpy(A.T.copy()).cuda()
    return buf, buf.t()[:m]


def _eigh_top(A, k=1):
    Cm = A.astype(np.float64) @ A.astype(np.float64).T
    w, V = np.linalg.eigh(Cm)
    return w[::-1][:k], V[:, ::-1][:, :k]


def test_batch_config_validation(amm_lib):
    """Argument checks come before any device work."""
    from eigenvaluecomputation_by_amm_b200 import _lib
    cfg = _lib.amm_batch_config()
    amm_lib.amm_batch_config_default(C.byref(cfg))
    assert cfg.nvec == 8 and cfg.max_iter > 0 and cfg.rr_period == 1
    mats = (_lib.amm_batch_matrix * 1)()
    mats[0].A, mats[0].ld, mats[0].m, mats[0].n = 256, 64, 64, 100
    b = C.c_void_p()
    bad = _lib.amm_batch_config()
    amm_lib.amm_batch_config_default(C.byref(bad))
    bad.nvec = 3
    assert amm_lib.amm_batch_create(C.byref(b), mats, 1, C.byref(bad), 0) == _lib.AMM_ERR_UNSUPPORTED
    assert amm_lib.amm_batch_create(C.byref(b), mats, 0, C.byref(cfg), 0) == \
        _lib.AMM_ERR_INVALID_ARGUMENT
    bad.nvec, bad.max_iter = 8, 0
    assert amm_lib.amm_batch_create(C.byref(b), mats, 1, C.byref(bad), 0) == \
        _lib.AMM_ERR_INVALID_ARGUMENT
    bad.max_iter, bad.wide = 10, 2
    assert amm_lib.amm_batch_create(C.byref(b), mats, 1, C.byref(bad), 0) == \
        _lib.AMM_ERR_INVALID_ARGUMENT
    assert cfg.wide == 0


@pytest.mark.gpu
@pytest.mark.parametrize("nvec,rtol,vtol", [(8, 1e-5, 2e-5), (4, 1e-5, 2e-5), (1, 1e-4, 1e-3)])
def test_batch_lambda_and_vector_vs_fp64(amm_lib, nvec, rtol, vtol):
    """At a residual of 1e-6·λ the eigenvector error is about 1e-6·λ_1/(λ_1 − λ_2): the single
    vector (no Rayleigh–Ritz over a block) gets the looser bound on 1 − |v·v*|."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    host = _mats(SIZES, seed=5)
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=nvec, max_iter=3000, tol=1e-6)
    lam, vec, iters = bs.run()
    torch.cuda.synchronize()
    lam = lam.cpu().numpy()
    it = iters.cpu().numpy()
    for i, A in enumerate(host):
        w, V = _eigh_top(A)
        assert it[i] > 0
        assert abs(lam[i] - w[0]) <= rtol * w[0], (i, lam[i], w[0], it[i])
        v = bs.vector(i).cpu().numpy().astype(np.float64)
        assert abs(np.linalg.norm(v) - 1.0) < 1e-5
        assert abs(float(v @ V[:, 0])) > 1 - vtol, i
    bs.close()


@pytest.mark.gpu
def test_batch_ritz_values_and_one_launch_per_matrix(amm_lib):
    """The 8-vector block also returns the next Ritz values; the per-matrix launches give
    bit-identical results (same kernel, one CTA per matrix)."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    host = _mats(SIZES[:5], seed=9)
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=8, max_iter=3000, tol=1e-6)
    bs.run()
    lam1 = bs.lam.clone()
    vec1 = bs.vectors.clone()
    bs.run(each=True)
    torch.cuda.synchronize()
    assert torch.equal(lam1, bs.lam)
    assert torch.equal(vec1, bs.vectors)
    bs.run()  # graph replay: deterministic
    assert torch.equal(lam1, bs.lam)
    for i, A in enumerate(host):
        # the stop is on the top pair; the next Ritz values are converged less far
        w, _ = _eigh_top(A, 3)
        got = lam1[i, :3].cpu().numpy()
        assert abs(got[0] - w[0]) <= 1e-5 * w[0]
        np.testing.assert_allclose(got[1:], w[1:], rtol=2e-3)
    k, gc, cl = bs.tile_choice()
    assert k == 8 and gc in (1, 2, 4, 8) and cl in (1, 2, 4, 8)
    assert int(bs.iters.max()) < 3000  # stopped on the residual, not on max_iter
    bs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cluster", [1, 2])
def test_batch_tensor_core_product_vs_fp64(amm_lib, cluster):
    """The tensor-core product (8 columns per group, TF32 mma.sync with A, X and AᵀX split into
    hi + lo parts) reaches the accuracy of the CUDA-core product: λ within 1e-5 of FP64 at the
    1e-6 residual, |v·v*| > 1 - 2e-5; at a fixed 20 products its Ritz values agree with the
    CUDA-core product's within 1e-5 (relative to λ_max)."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    host = _mats(SIZES, seed=5)
    keep = [_device_col_major(A) for A in host]
    mats = [v for _, v in keep]
    tc = BatchSolver(mats, nvec=8, max_iter=3000, tol=1e-6, tile_gc=8, cluster=cluster)
    lam, _, iters = tc.run()
    torch.cuda.synchronize()
    assert tc.tile_choice() == (8, 8, cluster)
    lam = lam.cpu().numpy()
    it = iters.cpu().numpy()
    for i, A in enumerate(host):
        w, V = _eigh_top(A)
        assert 0 < it[i] < 3000
        assert abs(lam[i] - w[0]) <= 1e-5 * w[0], (i, lam[i], w[0], it[i])
        v = tc.vector(i).cpu().numpy().astype(np.float64)
        assert abs(float(v @ V[:, 0])) > 1 - 2e-5, i
    tc.close()
    fixed = {}
    for gc in (8, 4):
        bs = BatchSolver(mats, nvec=8, max_iter=20, tol=0.0, tile_gc=gc, cluster=cluster)
        bs.run()
        torch.cuda.synchronize()
        fixed[gc] = bs.lam.cpu().numpy()
        assert (bs.iters.cpu().numpy() == 20).all()
        bs.close()
    scale = fixed[4][:, :1]
    assert np.all(np.abs(fixed[8] - fixed[4]) <= 1e-5 * scale), np.abs(fixed[8] - fixed[4]).max()


@pytest.mark.gpu
def test_batch_tensor_core_small_and_padded_shapes(amm_lib):
    """The tensor-core product's TMA tile copies (boxes of 32 rows x 8 columns, zeros outside
    the matrix) on shapes that do not fill them: fewer rows than a box (m = 8, 13, 31), ragged
    last boxes and groups (m = 33, 100; n = 9, 300), and a leading dimension well past m (the
    rows between m and ld hold garbage that must not be read).  λ is within 1e-5 of FP64 at the
    1e-6 residual; at a fixed 20 products the Ritz values are within 1e-5 (of λ_max) of the
    CUDA-core product's; and rebinding to other matrices of the same shapes, which re-encodes
    the tensor maps, gives bit for bit what a new solver on them gives."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    sizes = [(8, 8), (13, 9), (31, 300), (33, 40), (100, 9), (100, 300)]
    pads = [0, 12, 4, 20, 0, 28]  # extra rows of leading dimension past m rounded up to 4

    def device(host):
        keep = []
        for A, pad in zip(host, pads):
            m, n = A.shape
            ld = (m + 3) // 4 * 4 + pad
            buf = torch.full((n, ld), float("nan"), dtype=torch.float32, device="cuda")
            buf[:, :m] = torch.from_numpy(A.T.copy()).cuda()
            keep.append((buf, buf.t()[:m]))
        return keep

    host = _mats(sizes, seed=41)
    keep = device(host)
    mats = [v for _, v in keep]
    tc = BatchSolver(mats, nvec=8, max_iter=3000, tol=1e-6, tile_gc=8, cluster=1)
    lam, _, iters = tc.run()
    torch.cuda.synchronize()
    assert tc.tile_choice() == (8, 8, 1)
    lam, it = lam.cpu().numpy(), iters.cpu().numpy()
    for i, A in enumerate(host):
        w, _ = _eigh_top(A)
        assert 0 < it[i] < 3000, (i, it[i])
        assert abs(lam[i] - w[0]) <= 1e-5 * w[0], (i, lam[i], w[0], it[i])
    tc.close()
    fixed = {}
    for gc in (8, 4):
        bs = BatchSolver(mats, nvec=8, max_iter=20, tol=0.0, tile_gc=gc, cluster=1)
        bs.run()
        torch.cuda.synchronize()
        fixed[gc] = bs.lam.cpu().numpy()
        if gc == 8:
            host2 = _mats(sizes, seed=43)
            keep2 = device(host2)
            bs.set_matrices([v for _, v in keep2])
            bs.run()
            torch.cuda.synchronize()
            rebound = bs.lam.cpu().numpy()
            fresh = BatchSolver([v for _, v in keep2], nvec=8, max_iter=20, tol=0.0, tile_gc=8,
                                cluster=1)
            fresh.run()
            torch.cuda.synchronize()
            assert np.array_equal(rebound, fresh.lam.cpu().numpy())
            fresh.close()
        bs.close()
    assert np.all(np.isfinite(fixed[8]))
    scale = fixed[4][:, :1]
    assert np.all(np.abs(fixed[8] - fixed[4]) <= 1e-5 * scale), np.abs(fixed[8] - fixed[4]).max()


@pytest.mark.gpu
def test_batch_tensor_core_product_long_passes(amm_lib):
    """Long passes (up to 8192 columns, 1024 groups of 8 in one CTA): the tensor core's own
    accumulation is not rounded to nearest, so the product keeps every chain of tensor-core
    products short and sums them in FP32.  λ after 20 products stays within 1e-6 of FP64 (a
    single accumulator through the whole pass drifted to 6e-6 .. 4e-5 on these matrices)."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    sizes = [(1024, 8192), (2048, 4096), (300, 6000)]
    rng = np.random.default_rng(11)
    host = [(rng.standard_normal((m, n)) * np.exp(rng.standard_normal(n))[None, :]).astype(np.float32)
            for m, n in sizes]
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=8, max_iter=20, tol=0.0, tile_gc=8, cluster=1)
    bs.run()
    torch.cuda.synchronize()
    lam = bs.lam[:, 0].cpu().numpy()
    for i, A in enumerate(host):
        w, _ = _eigh_top(A)
        assert abs(lam[i] - w[0]) <= 1e-6 * w[0], (i, lam[i], w[0])
    bs.close()


@pytest.mark.gpu
def test_batch_tensor_core_product_is_exact_mode_only(amm_lib):
    """AMM batches have no tensor-core product: asking for it is UNSUPPORTED at the first run."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver, _lib
    host = _mats(SIZES[:2], seed=1)
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=8, max_iter=4, tol=0.0, c_divisor=8, tile_gc=8)
    with pytest.raises(_lib.AmmError) as err:
        bs.run()
    assert err.value.status == _lib.AMM_ERR_UNSUPPORTED
    bs.close()


@pytest.mark.gpu
def test_lambda_max_gradient_vs_eigvalsh_and_finite_differences():
    from eigenvaluecomputation_by_amm_b200 import lambda_max
    rng = np.random.default_rng(3)
    B, m, n = 3, 64, 256
    A = (rng.standard_normal((B, m, n)) * np.exp(0.5 * rng.standard_normal((B, 1, n))))
    A = A.astype(np.float32)
    tA = torch.from_numpy(A).cuda().requires_grad_(True)
    lam = lambda_max(tA, max_iter=3000, tol=1e-9)
    lam.sum().backward()
    g = tA.grad.double().cpu()
    # FP64 eigvalsh autograd
    A64 = torch.from_numpy(A.astype(np.float64)).requires_grad_(True)
    w = torch.linalg.eigvalsh(A64 @ A64.transpose(1, 2))[:, -1]
    w.sum().backward()
    np.testing.assert_allclose(lam.detach().cpu().numpy(), w.detach().numpy(), rtol=1e-5)
    rel = (g - A64.grad).norm() / A64.grad.norm()
    assert rel < 1e-4, float(rel)
    # central finite differences on 32 entries (FP64)
    h = 1e-3
    picks = [(int(rng.integers(B)), int(rng.integers(m)), int(rng.integers(n))) for _ in range(32)]
    A64n = A.astype(np.float64)
    gmax = float(g.abs().max())
    for b, i, j in picks:
        Ap, Am = A64n[b].copy(), A64n[b].copy()
        Ap[i, j] += h
        Am[i, j] -= h
        fd = (np.linalg.eigvalsh(Ap @ Ap.T)[-1] - np.linalg.eigvalsh(Am @ Am.T)[-1]) / (2 * h)
        assert abs(float(g[b, i, j]) - fd) <= 1e-3 * gmax, (b, i, j, float(g[b, i, j]), fd)


@pytest.mark.gpu
def test_batch_gradient_scale_and_layout(amm_lib):
    """grad_b = scale_b·2·v(vᵀA) written with its own leading dimension."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    host = _mats([(96, 300), (200, 150)], seed=11)
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=8, max_iter=2000, tol=1e-6)
    bs.run()
    grads, stores = [], []
    for A in host:
        m, n = A.shape
        gb = torch.full((n, m + 8), 7.0, device="cuda")   # ld = m + 8: rows m.. stay untouched
        stores.append(gb)
        grads.append(gb.t()[:m])
    scale = torch.tensor([2.0, -0.5], device="cuda")
    bs.grad(grads, scale=scale)
    for i, A in enumerate(host):
        v = bs.vector(i).double().cpu().numpy()
        want = scale[i].item() * 2.0 * np.outer(v, v @ A.astype(np.float64))
        got = grads[i].double().cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5 * np.abs(want).max())
        assert torch.all(stores[i][:, A.shape[0]:] == 7.0)
    bs.close()


@pytest.mark.gpu
def test_batch_gradient_many_small_matrices_unaligned(amm_lib):
    """The backward on more matrices than its column prefix keeps in shared memory (4200 > 4096:
    the search runs in global memory), with m not a multiple of 4 (the last chunk of a column)
    and gradient columns that do not start 16-byte aligned (leading dimension m + 1: the 4-byte
    stores): every gradient equals scale_b·2·v(vᵀA) within FP32 rounding, and the rows past m
    are not written."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    rng = np.random.default_rng(17)
    count = 4200
    ms = rng.choice([8, 9, 10, 13], size=count)
    ns = rng.choice([8, 11, 16], size=count)
    host = [rng.standard_normal((int(m), int(n))).astype(np.float32) for m, n in zip(ms, ns)]
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=8, max_iter=50, tol=1e-6)
    bs.run()
    grads, stores = [], []
    for A in host:
        m, n = A.shape
        gb = torch.full((n, m + 1), 7.0, device="cuda")
        stores.append(gb)
        grads.append(gb.t()[:m])
    scale = torch.from_numpy(rng.uniform(-2.0, 2.0, count).astype(np.float32)).cuda()
    bs.grad(grads, scale=scale)
    torch.cuda.synchronize()
    vecs = bs.vectors.double().cpu().numpy()
    sc = scale.double().cpu().numpy()
    for i, A in enumerate(host):
        v = vecs[int(bs.offsets[i]):int(bs.offsets[i]) + A.shape[0]]
        want = sc[i] * 2.0 * np.outer(v, v @ A.astype(np.float64))
        got = grads[i].double().cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5 * np.abs(want).max() + 1e-30)
        assert torch.all(stores[i][:, A.shape[0]:] == 7.0)
    bs.close()


@pytest.mark.gpu
def test_batch_amm_mode_spiked_matrices(amm_lib):
    """Previous-AMM products (c = n/8) in the batch: reproducible from the seed, identical with
    one launch per matrix, and within 2% of λ_max where a spike shared by every column dominates
    (then every sampled column carries the top direction)."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    rng = np.random.default_rng(21)
    host = []
    for m, n in [(64, 256), (200, 1600), (517, 4096), (1024, 8192)]:
        u = rng.standard_normal(m)
        u /= np.linalg.norm(u)
        A = 0.05 * rng.standard_normal((m, n)) + u[:, None] * rng.uniform(0.5, 1.5, n)[None, :]
        host.append(A.astype(np.float32))
    keep = [_device_col_major(A) for A in host]
    bs = BatchSolver([v for _, v in keep], nvec=8, max_iter=12, tol=0.0, c_divisor=8)
    bs.run()
    lam1 = bs.lam.clone()
    bs.run()
    assert torch.equal(lam1, bs.lam)
    bs.run(each=True)
    torch.cuda.synchronize()
    assert torch.equal(lam1, bs.lam)
    for i, A in enumerate(host):
        w, _ = _eigh_top(A)
        assert abs(lam1[i, 0].item() - w[0]) <= 0.02 * w[0], (i, lam1[i, 0].item(), w[0])
    assert int(bs.iters.min()) == 12
    bs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cluster", [1, 2, 4, 8])
def test_batch_every_cluster_size_agrees(amm_lib, cluster):
    """A matrix shared by a cluster of 2, 4 or 8 CTAs (columns split, partial products summed
    through distributed shared memory) gives λ within 1e-5 of the single-CTA result, in exact
    and AMM mode; the AMM picks are the same for every cluster size (one state stream)."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    host = _mats([(64, 256), (333, 1000), (1024, 4096), (2048, 300)], seed=31)
    keep = [_device_col_major(A) for A in host]
    ref = BatchSolver([v for _, v in keep], nvec=8, max_iter=3000, tol=1e-6, cluster=1)
    ref.run()
    got = BatchSolver([v for _, v in keep], nvec=8, max_iter=3000, tol=1e-6, cluster=cluster)
    got.run()
    torch.cuda.synchronize()
    assert got.tile_choice()[2] == cluster
    np.testing.assert_allclose(got.lam[:, 0].cpu().numpy(), ref.lam[:, 0].cpu().numpy(), rtol=1e-5)
    for A_i, (i, A) in zip(host, enumerate(host)):
        w, _ = _eigh_top(A)
        assert abs(got.lam[i, 0].item() - w[0]) <= 1e-5 * w[0]
    ra = BatchSolver([v for _, v in keep], nvec=8, max_iter=6, tol=0.0, c_divisor=8, cluster=1)
    ga = BatchSolver([v for _, v in keep], nvec=8, max_iter=6, tol=0.0, c_divisor=8, cluster=cluster)
    ra.run()
    ga.run()
    torch.cuda.synchronize()
    np.testing.assert_allclose(ga.lam[:, 0].cpu().numpy(), ra.lam[:, 0].cpu().numpy(), rtol=1e-4)
    for s in (ref, got, ra, ga):
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_wide_plan_agrees(amm_lib, use_graph):
    """An uneven batch (one matrix holding most of the work) run as two launches — the heavy
    matrix first on a wide cluster, the rest shared with a programmatic dependent launch queued
    behind it — gives the λ of one launch per run (within 1e-5, exact mode; 1e-4 in AMM mode,
    the same picks) and of FP64 LAPACK; the plan is reported by amm_batch_wide_plan."""
    from eigenvaluecomputation_by_amm_b200 import BatchSolver
    sizes = [(1536, 4096)] + [(64 + 16 * k, 256 + 32 * k) for k in range(40)]
    host = _mats(sizes, seed=41)
    keep = [_device_col_major(A) for A in host]
    mats = [v for _, v in keep]
    one = BatchSolver(mats, nvec=8, max_iter=3000, tol=1e-6, tile_gc=4, cluster=2, wide=-1,
                      use_graph=use_graph)
    two = BatchSolver(mats, nvec=8, max_iter=3000, tol=1e-6, tile_gc=4, cluster=2, wide=1,
                      use_graph=use_graph)
    one.run()
    two.run()
    torch.cuda.synchronize()
    assert one.wide_plan()["count"] == 0
    plan = two.wide_plan()
    assert plan["count"] >= 1 and plan["cluster"] > 2 and plan["ctas"] % plan["cluster"] == 0
    np.testing.assert_allclose(two.lam[:, 0].cpu().numpy(), one.lam[:, 0].cpu().numpy(),
                               rtol=1e-5)
    assert (two.iters.cpu().numpy() > 0).all()
    for i in (0, 1, 20, 40):
        w, _ = _eigh_top(host[i])
        assert abs(two.lam[i, 0].item() - w[0]) <= 1e-5 * w[0]
    # a second run of the same context (queues and states reset by the run's prologue)
    two.run()
    torch.cuda.synchronize()
    np.testing.assert_allclose(two.lam[:, 0].cpu().numpy(), one.lam[:, 0].cpu().numpy(),
                               rtol=1e-5)
    ra = BatchSolver(mats, nvec=8, max_iter=6, tol=0.0, c_divisor=8, tile_gc=4, cluster=2,
                     wide=-1, use_graph=use_graph)
    ga = BatchSolver(mats, nvec=8, max_iter=6, tol=0.0, c_divisor=8, tile_gc=4, cluster=2,
                     wide=1, use_graph=use_graph)
    ra.run()
    ga.run()
    torch.cuda.synchronize()
    assert ga.wide_plan()["count"] >= 1
    np.testing.assert_allclose(ga.lam[:, 0].cpu().numpy(), ra.lam[:, 0].cpu().numpy(), rtol=1e-4)
    for s in (one, two, ra, ga):
        s.close()
