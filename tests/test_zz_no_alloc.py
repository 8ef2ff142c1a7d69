"""amm_pick_sorted_noalloc: the allocation-free draw + sort, called through the C ABI.

Compared with the context sampler (amm_sample_indices, the existing entry point) and with the
oracle's pick_index + sort on the same CDF and states, for two calls in a row (the second
starts from the states the first returned, and runs after the first has left its static
scratch behind).  Integer results: bit-exact.  Also: the largest n the static array takes and a
ragged last tile, an all-zero CDF (every pick falls back to column n-1, as in the reference's
pick_index), and the device's free memory unchanged across repeated calls.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import amm_oracle as O
from helpers import scaled_gaussian, states


def _noalloc(lib, st_in, st_out, cdf, n, prec, out, dcount, stream=0):
    return lib.amm_pick_sorted_noalloc(st_in.data_ptr(), st_out.data_ptr(), st_in.numel(),
                                       cdf.data_ptr(), prec, n, out.data_ptr(),
                                       dcount.data_ptr(), stream)


def test_rejects_sizes_beyond_the_static_scratch(amm_lib):
    """Argument checks happen before any device work (no GPU needed)."""
    from eigenvaluecomputation_by_amm_b200 import _lib
    p = C.c_void_p(16)  # never dereferenced: the size check fails first
    rc = amm_lib.amm_pick_sorted_noalloc(p, p, 8, p, _lib.AMM_CDF_F64, (1 << 18) + 1, p, p, None)
    assert rc == _lib.AMM_ERR_UNSUPPORTED
    rc = amm_lib.amm_pick_sorted_noalloc(p, p, 0, p, _lib.AMM_CDF_F64, 100, p, p, None)
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT
    rc = amm_lib.amm_pick_sorted_noalloc(p, p, 8, p, 7, 100, p, p, None)
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT
    rc = amm_lib.amm_pick_sorted_noalloc(None, p, 8, p, _lib.AMM_CDF_F64, 100, p, p, None)
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("cdf", ["f64", "f32"])
@pytest.mark.parametrize("n", [1, 31, 3000, 65536])
def test_matches_the_context_sampler_twice_in_a_row(amm_lib, cdf, n):
    from eigenvaluecomputation_by_amm_b200 import AMMContext, _lib, column_major
    m, c = 64, 2048
    A = scaled_gaussian(m, n, seed=n + 5, sigma=2.0)
    A[:, np.random.default_rng(n).random(n) < 0.05] = 0.0  # zero columns are never picked
    if not A.any():
        A[0, 0] = 1.0
    ctx = AMMContext(m, n, c=c, step=2, cdf_precision=cdf)
    ctx.set_matrix(column_major(torch.from_numpy(A).cuda()))
    prec = _lib.AMM_CDF_F64 if cdf == "f64" else _lib.AMM_CDF_F32
    st0 = states(c, seed=n + 11)
    cur = torch.from_numpy(st0.view(np.int32).copy()).cuda()
    for which in (0, 1):
        table, _ = ctx.sampling_tables(which)
        for call in range(2):
            ctx.set_rng_state(cur)
            want = np.sort(ctx.sample_indices(which).cpu().numpy().view(np.uint32))
            nxt = torch.empty_like(cur)
            out = torch.full((c,), -1, dtype=torch.int32, device="cuda")
            dcount = torch.full((1,), -1, dtype=torch.int32, device="cuda")
            assert _noalloc(amm_lib, cur, nxt, table, n, prec, out, dcount) == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, want), (which, call)
            assert int(dcount.item()) == len(np.unique(want))
            expect_states, _ = O.xorshift32(cur.cpu().numpy().view(np.uint32))
            assert np.array_equal(nxt.cpu().numpy().view(np.uint32), expect_states)
            cur = nxt
    ctx.close()


@pytest.mark.gpu
def test_in_place_states_and_all_picks_on_one_column(amm_lib):
    """States may alias (in place); a CDF with one non-zero weight puts every pick on it."""
    from eigenvaluecomputation_by_amm_b200 import _lib
    n, c = 1000, 4096
    w = np.zeros(n)
    w[417] = 3.0
    cdf = torch.from_numpy(np.cumsum(w)).cuda()
    st = states(c, seed=3)
    cur = torch.from_numpy(st.view(np.int32).copy()).cuda()
    out = torch.empty(c, dtype=torch.int32, device="cuda")
    dcount = torch.empty(1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        before = cur.cpu().numpy().view(np.uint32).copy()
        assert _noalloc(amm_lib, cur, cur, cdf, n, _lib.AMM_CDF_F64, out, dcount) == 0
        torch.cuda.synchronize()
        assert np.all(out.cpu().numpy() == 417)
        assert int(dcount.item()) == 1
        assert np.array_equal(cur.cpu().numpy().view(np.uint32), O.xorshift32(before)[0])


def _host_cdf(n, seed, prec):
    """An inclusive prefix of random non-negative weights (some zero), FP64 or FP32."""
    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 1.5, n)
    w[rng.random(n) < 0.1] = 0.0
    cdf = np.cumsum(w)
    return cdf if prec == "f64" else cdf.astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("cdf_prec", ["f64", "f32"])
@pytest.mark.parametrize("n,c", [(200003, 6000), (1 << 18, 8192), (5000, 40000)])
def test_matches_the_oracle_at_the_size_limit_twice_in_a_row(amm_lib, cdf_prec, n, c):
    """n = 2^18 is the largest n the static array holds; 200003 leaves a ragged last tile; c
    larger than n puts many picks on each column."""
    from eigenvaluecomputation_by_amm_b200 import _lib
    prec = _lib.AMM_CDF_F64 if cdf_prec == "f64" else _lib.AMM_CDF_F32
    cdf_h = _host_cdf(n, seed=n + c, prec=cdf_prec)
    cdf = torch.from_numpy(cdf_h).cuda()
    cur_h = states(c, seed=c + 1)
    cur = torch.from_numpy(cur_h.view(np.int32).copy()).cuda()
    for call in range(2):
        want, want_states = O.sample_sorted(cdf_h, cur_h, c)
        nxt = torch.empty_like(cur)
        out = torch.full((c,), -1, dtype=torch.int32, device="cuda")
        dcount = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        assert _noalloc(amm_lib, cur, nxt, cdf, n, prec, out, dcount) == 0
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want), call
        assert int(dcount.item()) == len(np.unique(want))
        assert np.array_equal(nxt.cpu().numpy().view(np.uint32), want_states)
        cur, cur_h = nxt, want_states


@pytest.mark.gpu
@pytest.mark.parametrize("cdf_prec", ["f64", "f32"])
def test_all_zero_cdf_puts_every_pick_on_the_last_column(amm_lib, cdf_prec):
    from eigenvaluecomputation_by_amm_b200 import _lib
    prec = _lib.AMM_CDF_F64 if cdf_prec == "f64" else _lib.AMM_CDF_F32
    n, c = 3001, 2048
    cdf = torch.zeros(n, dtype=torch.float64 if cdf_prec == "f64" else torch.float32,
                      device="cuda")
    cur = torch.from_numpy(states(c, seed=9).view(np.int32).copy()).cuda()
    out = torch.empty(c, dtype=torch.int32, device="cuda")
    dcount = torch.empty(1, dtype=torch.int32, device="cuda")
    assert _noalloc(amm_lib, cur, cur, cdf, n, prec, out, dcount) == 0
    torch.cuda.synchronize()
    assert np.all(out.cpu().numpy() == n - 1)
    assert int(dcount.item()) == 1


@pytest.mark.gpu
def test_repeated_calls_leave_free_device_memory_unchanged(amm_lib):
    """The entry point allocates nothing: after a first call (which may load the library's
    device module), cudaMemGetInfo reports the same free memory around 20 further calls."""
    from eigenvaluecomputation_by_amm_b200 import _lib
    n, c = 1 << 18, 16384
    cdf = torch.from_numpy(_host_cdf(n, seed=5, prec="f64")).cuda()
    cur = torch.from_numpy(states(c, seed=6).view(np.int32).copy()).cuda()
    out = torch.empty(c, dtype=torch.int32, device="cuda")
    dcount = torch.empty(1, dtype=torch.int32, device="cuda")
    assert _noalloc(amm_lib, cur, cur, cdf, n, _lib.AMM_CDF_F64, out, dcount) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(20):
        assert _noalloc(amm_lib, cur, cur, cdf, n, _lib.AMM_CDF_F64, out, dcount) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
