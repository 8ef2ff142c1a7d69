"""amm_pick_sorted_noalloc: the allocation-free draw + sort, called through the C ABI.

Compared with the context sampler (amm_sample_indices, the existing entry point) on the same
CDF and states, for two calls in a row (the second starts from the states the first returned,
and runs after the first has left its static scratch behind).  Integer results: bit-exact.
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
