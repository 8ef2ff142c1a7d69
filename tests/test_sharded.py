"""Column-sharded previous AMM (eigenvaluecomputation_by_amm_b200.sharded).

CPU: the host logic — the shard bounds, the global CDF assembled from the ranks' CDFs by
all-gather, the replicated state, one all-reduce of the partial products per step — run as
world-size-2 gloo process groups, each rank multiplying with the oracle's arithmetic (the
backend below is test infrastructure); the λ trace must equal the one-process restatement
``oracle.sharded_previous`` on the same shards (FP32 partial sums added in rank order: the same
numbers), and the picks are integer work.

GPU (one device): libamm's ``amm_shard_product`` for one shard holding every column and for 3
shards multiplied in turn on the same GPU (each with its own copy of the replicated states):
the states bit-exact against the oracle given the library's global CDF, λ within the FP32
tolerance of the tests.  Runs on several GPUs (NCCL) are not measured here: a call on this
pool gets one GPU.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import amm_oracle as O
from helpers import RTOL_LAMBDA_F32, scaled_gaussian, states

ROOT = Path(__file__).resolve().parents[1]


class OracleShard:
    """A shard whose products use the oracle's arithmetic on CPU tensors (test backend)."""

    def __init__(self, A_shard, c):
        self.A = np.asarray(A_shard, np.float32)
        self.c = c

    def local_cdf(self):
        return torch.from_numpy(O.shard_cdf(self.A))

    def exact(self, x):
        return torch.from_numpy(O.exact_product(self.A, x.numpy()))

    def sampled(self, cdf, col0, st, x, x_memo, y_memo):
        s = st.numpy().view(np.uint32)
        idx, s_new = O.pick_index(cdf.numpy(), s, self.c)
        s[:] = s_new
        cols, w = O.sharded_weights(cdf.numpy(), idx)
        n = self.A.shape[1]
        sel = (cols >= col0) & (cols < col0 + n)
        xm = np.zeros_like(self.A[:, 0]) if x_memo is None else x_memo.numpy()
        dx = (x.numpy() - xm).astype(np.float64)
        As = self.A[:, cols[sel] - col0].astype(np.float64)
        tmp = ((As.T @ dx).astype(np.float32) * w[sel]).astype(np.float32)
        base = 0.0 if y_memo is None else y_memo.numpy().astype(np.float64)
        return torch.from_numpy((base + As @ tmp.astype(np.float64)).astype(np.float32))

    def normalize(self, x):
        x.copy_(torch.from_numpy(O.normalize(x.numpy())))
        return x

    def rayleigh(self, x, y):
        lam, err, cosv, xn = O.dot_product_and_generate_x(x.numpy(), y.numpy())
        x.copy_(torch.from_numpy(xn))
        return lam, err, cosv


def _problem():
    m, n, c = 96, 1500, 256
    A = scaled_gaussian(m, n, seed=41, sigma=1.0)
    x0 = np.random.default_rng(42).standard_normal(m).astype(np.float32)
    st = states(c, seed=43)
    return A, x0, st, c


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    for p in (ROOT, ROOT / "oracle", ROOT / "tests"):
        sys.path.insert(0, str(p))
    from eigenvaluecomputation_by_amm_b200.sharded import ShardedPowerMethod, shard_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        A, x0, st, c = _problem()
        a, b = shard_bounds(A.shape[1], world, rank)
        pm = ShardedPowerMethod(OracleShard(A[:, a:b], c), a, A.shape[1], c, step=12, vr_period=4)
        stt = torch.from_numpy(st.view(np.int32).copy())
        tr = pm.run(torch.from_numpy(x0), stt)
        out[rank] = {"eigs": tr["eigs"], "kinds": tr["kinds"], "cdf": pm.cdf.numpy().tolist(),
                     "states": stt.numpy().view(np.uint32).tolist()}
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_the_columns():
    from eigenvaluecomputation_by_amm_b200.sharded import shard_bounds
    for n, w in [(10, 3), (65536, 8), (7, 7), (1000, 4)]:
        got = [shard_bounds(n, w, r) for r in range(w)]
        assert got[0][0] == 0 and got[-1][1] == n
        assert all(got[r][1] == got[r + 1][0] for r in range(w - 1))
        assert max(b - a for a, b in got) - min(b - a for a, b in got) <= 1


def test_oracle_sharding_leaves_picks_and_lambda_unchanged():
    """The restatement itself: 1, 2 or 3 shards draw the same picks from the same global CDF
    and give λ to FP32 rounding of the partial sums."""
    A, x0, st, c = _problem()
    n = A.shape[1]
    e1, k1, s1, cdf1, p1 = O.sharded_previous(A, [(0, n)], c=c, states=st, step=12,
                                              vr_period=4, x0=x0)
    for bounds in ([(0, 750), (750, n)], [(0, 400), (400, 1111), (1111, n)]):
        e, k, s, cdf, p = O.sharded_previous(A, bounds, c=c, states=st, step=12, vr_period=4,
                                             x0=x0, cdf=cdf1)
        assert k == k1 and np.array_equal(s, s1)
        assert all(np.array_equal(a, b) for a, b in zip(p, p1))
        assert np.all(np.abs(e - e1) <= RTOL_LAMBDA_F32 * np.abs(e1))


def test_two_gloo_ranks_match_the_restatement():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    A, x0, st, c = _problem()
    from eigenvaluecomputation_by_amm_b200.sharded import shard_bounds
    bounds = [shard_bounds(A.shape[1], world, r) for r in range(world)]
    e, k, s, cdf, _ = O.sharded_previous(A, bounds, c=c, states=st, step=12, vr_period=4, x0=x0)
    for r in range(world):
        got = out[r]
        assert got["kinds"] == k
        assert np.array_equal(np.array(got["cdf"]), cdf)
        assert np.array_equal(np.array(got["states"], np.uint32), s)
        np.testing.assert_array_equal(np.array(got["eigs"]), e)
    assert out[0]["eigs"] == out[1]["eigs"]


@pytest.mark.gpu
@pytest.mark.parametrize("nshards", [1, 3])
def test_shard_products_on_one_gpu_match_the_oracle(amm_lib, nshards):
    """amm_shard_product for each shard of the columns in turn (one GPU), partial products
    summed in rank order, against the restatement given the library's global CDF."""
    from eigenvaluecomputation_by_amm_b200 import column_major
    from eigenvaluecomputation_by_amm_b200.sharded import LibammShard, shard_bounds
    A, x0, st, c = _problem()
    n = A.shape[1]
    bounds = [shard_bounds(n, nshards, r) for r in range(nshards)]
    shards = [LibammShard(column_major(torch.from_numpy(A[:, a:b]).cuda()), c)
              for a, b in bounds]
    parts, off = [], 0.0
    for sh in shards:
        cg = sh.local_cdf().double()
        parts.append(cg + off)
        off += float(cg[-1].item())
    cdf = torch.cat(parts).contiguous()
    e_ref, k_ref, s_ref, _, _ = O.sharded_previous(A, bounds, c=c, states=st, step=12,
                                                   vr_period=4, x0=x0, cdf=cdf.cpu().numpy())
    sts = [torch.from_numpy(st.view(np.int32).copy()).cuda() for _ in shards]
    x = torch.from_numpy(x0).cuda()
    shards[0].normalize(x)
    xm = ym = None
    eigs = []
    for i in range(12):
        if (i + 1) % 4 == 0:
            y = sum(sh.exact(x) for sh in shards)
            xm, ym = x.clone(), y.clone()
        else:
            y = None
            for r, (sh, (a, b)) in enumerate(zip(shards, bounds)):
                p = sh.sampled(cdf, a, sts[r], x, xm, ym if r == 0 else None)
                y = p if y is None else y + p
        lam, _, _ = shards[0].rayleigh(x, y)
        eigs.append(lam)
    for s_ in sts:
        assert np.array_equal(s_.cpu().numpy().view(np.uint32), s_ref)
    assert np.all(np.abs(np.array(eigs) - e_ref) <= RTOL_LAMBDA_F32 * np.abs(e_ref))
    for sh in shards:
        sh.close()


@pytest.mark.gpu
def test_sharded_driver_on_one_rank(amm_lib):
    """The driver without a process group (one rank holding every column) on the GPU."""
    from eigenvaluecomputation_by_amm_b200 import column_major
    from eigenvaluecomputation_by_amm_b200.sharded import LibammShard, ShardedPowerMethod
    A, x0, st, c = _problem()
    sh = LibammShard(column_major(torch.from_numpy(A).cuda()), c)
    pm = ShardedPowerMethod(sh, 0, A.shape[1], c, step=12, vr_period=4)
    stt = torch.from_numpy(st.view(np.int32).copy()).cuda()
    tr = pm.run(torch.from_numpy(x0).cuda(), stt)
    e_ref, k_ref, s_ref, _, _ = O.sharded_previous(A, [(0, A.shape[1])], c=c, states=st, step=12,
                                                   vr_period=4, x0=x0, cdf=pm.cdf.cpu().numpy())
    assert tr["kinds"] == k_ref
    assert np.array_equal(stt.cpu().numpy().view(np.uint32), s_ref)
    assert np.all(np.abs(np.array(tr["eigs"]) - e_ref) <= RTOL_LAMBDA_F32 * np.abs(e_ref))
    sh.close()


@pytest.mark.gpu
def test_list_product_matches_the_oracle(amm_lib):
    """amm_core_list_product on a given work list (previous and proposed forms), and an index
    outside the matrix is reported instead of read."""
    from eigenvaluecomputation_by_amm_b200 import AMMContext, _lib, column_major
    m, n, c = 128, 700, 200
    A = scaled_gaussian(m, n, seed=51, shift=0.1)
    rng = np.random.default_rng(52)
    cols = np.unique(rng.integers(0, n, 150)).astype(np.int32)
    wm = rng.uniform(0.5, 2.0, cols.size).astype(np.float32)
    x = O.normalize(rng.standard_normal(m).astype(np.float32))
    xm = O.normalize(rng.standard_normal(m).astype(np.float32))
    ym = rng.standard_normal(m).astype(np.float32)
    ctx = AMMContext(m, n, c=c, step=1)
    ctx.set_matrix(column_major(torch.from_numpy(A).cuda()))
    w_full = np.zeros(n, np.float32)
    w_full[cols] = wm
    y = ctx.core_list_product("previous", torch.from_numpy(cols), torch.from_numpy(wm),
                              torch.from_numpy(x), torch.from_numpy(xm), torch.from_numpy(ym))
    _, want = O.previous_amm(A, x, xm, ym, cols, w_full)
    assert np.linalg.norm(y.cpu().numpy() - want) <= 1e-4 * np.linalg.norm(want)
    alpha, _, _ = O.get_norms(A)
    z, v = O.generate_zv(A, alpha, O.alpha_squared(alpha))
    y = ctx.core_list_product("proposed", torch.from_numpy(cols), torch.from_numpy(wm),
                              torch.from_numpy(x), torch.from_numpy(xm), torch.from_numpy(ym))
    _, want = O.proposed_amm(A, alpha, x, xm, ym, cols, w_full, z, v)
    assert np.linalg.norm(y.cpu().numpy() - want) <= 1e-4 * np.linalg.norm(want)
    bad = cols.copy()
    bad[3] = n + 5
    ctx.core_list_product("previous", torch.from_numpy(bad), torch.from_numpy(wm),
                          torch.from_numpy(x))
    with pytest.raises(_lib.AmmError) as ei:
        ctx.trace()
    assert ei.value.status == _lib.AMM_ERR_INVALID_ARGUMENT
    ctx.close()
