"""Matrix sources of the reference's driver: -filepath loader and -matrixType generators.

The loader is host code (checked on the CPU against the layout device_memory.h:369-401
defines); the generators are compared bit for bit with the reference's own generate_matrix
(run through the oracle harness) for the same seed.
"""
import struct

import numpy as np
import pytest


def _write(path, A):
    with open(path, "wb") as f:
        f.write(struct.pack("<I", A.shape[0]))
        f.write(np.ascontiguousarray(A, np.float32).tobytes())


def test_read_matrix_file_pads_and_keeps_the_reference_layout(tmp_path, amm_lib):
    from eigenvaluecomputation_by_amm_b200.api import read_matrix_file
    rng = np.random.default_rng(0)
    A = rng.standard_normal((200, 200)).astype(np.float32)
    p = tmp_path / "cov.bin"
    _write(p, A)
    H, n0 = read_matrix_file(p)
    assert n0 == 200 and H.shape == (256, 256)          # padded to a multiple of 128
    np.testing.assert_array_equal(H[:200, :200], A)     # file row y at h[y*size + x]
    assert not H[200:].any() and not H[:, 200:].any()
    H2, _ = read_matrix_file(p, size=200)
    np.testing.assert_array_equal(H2, A)


def test_read_matrix_file_rejects_bad_input(tmp_path, amm_lib):
    from eigenvaluecomputation_by_amm_b200 import _lib
    import ctypes as C
    p = tmp_path / "short.bin"
    with open(p, "wb") as f:
        f.write(struct.pack("<I", 10))
        f.write(np.zeros(50, np.float32).tobytes())   # 50 of 100 values
    buf = np.zeros((16, 16), np.float32)
    o = C.c_int64(0)
    rc = amm_lib.amm_read_matrix_file(str(p).encode(), buf.ctypes.data_as(C.c_void_p), 16,
                                      C.byref(o))
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT
    rc = amm_lib.amm_read_matrix_file(str(p).encode(), buf.ctypes.data_as(C.c_void_p), 8,
                                      C.byref(o))
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT       # buffer smaller than the matrix
    rc = amm_lib.amm_read_matrix_file(str(tmp_path / "none.bin").encode(), None, 0, C.byref(o))
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT


def test_generate_matrix_rejects_unknown_kinds(amm_lib):
    from eigenvaluecomputation_by_amm_b200 import _lib
    rc = amm_lib.amm_generate_matrix(b"cauchy_0_1", 128, 1, 16, None, None)
    assert rc == _lib.AMM_ERR_UNSUPPORTED
    rc = amm_lib.amm_generate_matrix(b"gaussian_0_1", 0, 1, 16, None, None)
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["gaussian_0.0_1.0", "lognormal_0.0_0.5", "uniform_-1.0_2.0"])
def test_generators_match_the_reference_bit_for_bit(kind):
    import ref_harness as R
    if not R.available():
        pytest.skip("reference harness not built")
    from eigenvaluecomputation_by_amm_b200.api import generate_matrix
    m, seed = 256, 77
    A, off = generate_matrix(kind, m, seed)
    want, woff = R.generate(kind, m, seed)
    got = A.cpu().numpy()          # column-major storage of a symmetric matrix
    assert off == woff
    np.testing.assert_array_equal(got.T, want.T)
    np.testing.assert_array_equal(got, got.T)
