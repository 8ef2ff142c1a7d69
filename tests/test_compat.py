"""The reference's driver and result files through include/amm_compat.hpp.

tests/compat_main.cpp is the reference's main (AMM.cu:7-95) over the compat header; it and the
reference's own AMM binary (built from its sources by oracle/Makefile) run with the same flags
on the same covariance file, and their result files (time, eig, err doubles per step,
device_memory.h:256-275) are compared: the file names must be identical, eig within rtol 1e-5
and err within 1e-5 (FP32 power method, different summation orders); the time column is not
compared.  A -matrixType run (no file) is compared the same way against our own generator.
"""
import os
import shutil
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "eigenvaluecomputation_by_amm_b200"
REF_BIN = ROOT / "oracle" / "_ref" / "amm_ref"


def _build(tmp):
    exe = tmp / "compat_main"
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include",
           str(ROOT / "tests" / "compat_main.cpp"), "-o", str(exe), f"-L{PKG}", "-lamm",
           "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_compat_driver_compiles(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    _build(tmp_path)


def _workdir(tmp, name, A, v):
    d = tmp / name
    (d / "data").mkdir(parents=True)
    (d / "result").mkdir()
    with open(d / "matrix.bin", "wb") as f:
        f.write(struct.pack("<I", A.shape[0]))
        f.write(np.ascontiguousarray(A, np.float32).tobytes())
    np.asarray(v, np.float64).tofile(d / "data" / "exact_eigenvector")
    return d


def _results(d):
    files = sorted((d / "result").iterdir())
    assert len(files) == 1
    return files[0].name, np.fromfile(files[0], np.float64).reshape(-1, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("args", [["-kernel", "exact", "-step", "12"],
                                  ["-kernel", "previousAMM", "-step", "6", "-c", "256",
                                   "-sanity"]])
def test_result_files_match_the_reference_driver(tmp_path, args):
    if not REF_BIN.exists():
        pytest.skip("reference driver not built (make -C oracle)")
    exe = _build(tmp_path)
    rng = np.random.default_rng(4)
    m = 256
    B = rng.standard_normal((m, 3 * m)) * np.exp(rng.standard_normal(3 * m))[None, :]
    A = (B @ B.T / (3 * m)).astype(np.float32)      # a covariance matrix (symmetric, PSD)
    w, V = np.linalg.eigh(A.astype(np.float64) @ A.astype(np.float64))
    v = V[:, -1]
    flags = ["-m", str(m), "-r", "2", "-seed", "9", "-filepath", "matrix.bin"] + args
    d_ref = _workdir(tmp_path, "ref", A, v)
    d_us = _workdir(tmp_path, "us", A, v)
    subprocess.run([str(REF_BIN)] + flags, cwd=d_ref, check=True, capture_output=True, timeout=120)
    subprocess.run([str(exe)] + flags, cwd=d_us, check=True, capture_output=True, timeout=120)
    n_ref, r_ref = _results(d_ref)
    n_us, r_us = _results(d_us)
    assert n_us == n_ref
    assert r_us.shape == r_ref.shape
    np.testing.assert_allclose(r_us[:, 1], r_ref[:, 1], rtol=1e-5)
    np.testing.assert_allclose(r_us[:, 2], r_ref[:, 2], atol=1e-5)


@pytest.mark.gpu
def test_generated_matrix_run_follows_the_reference_generator_sequence(tmp_path):
    """-matrixType without a file (the reference's own driver cannot run this case: its result
    file naming indexes the empty path, device_memory.h:256-259).  The reference draws the
    matrix (size² values), the states (m values) and then the start vectors from ONE cuRAND
    generator that re-seeding does not rewind; the driver's trace must equal a library run
    whose start vectors come from that position, and report sqrt(λ) − offset."""
    import ctypes as C
    import torch
    from eigenvaluecomputation_by_amm_b200 import AMMContext, _lib
    from eigenvaluecomputation_by_amm_b200.api import generate_matrix
    exe = _build(tmp_path)
    m, seed, steps = 256, 13, 20
    d = tmp_path / "gen"
    (d / "data").mkdir(parents=True)
    (d / "result").mkdir()
    np.zeros(m, np.float64).tofile(d / "data" / "exact_eigenvector")
    subprocess.run([str(exe), "-m", str(m), "-r", "1", "-seed", str(seed), "-kernel", "exact",
                    "-step", str(steps), "-matrixType", "gaussian_0.0_1.0"], cwd=d, check=True,
                   capture_output=True, timeout=120)
    _, r = _results(d)
    A, off = generate_matrix("gaussian_0.0_1.0", m, seed)
    ctx = AMMContext(m, m, step=steps)
    ctx.set_matrix(A.t())  # symmetric: the transpose view is the column-major layout
    lib = _lib.load()
    assert lib.amm_seed_start_vectors_at(ctx._ctx, 1234 + seed, m * m + m) == 0
    x0 = torch.empty(m, device="cuda")
    for _ in range(2):  # the driver's warm-up draw, then the measured one
        assert lib.amm_draw_start_vector(ctx._ctx, x0.data_ptr(), None) == 0
        ctx.power_method("exact", x0)
    lam = ctx.trace()["eigs"]
    want = np.maximum(0.0, np.sqrt(np.maximum(0.0, lam)) - off)
    np.testing.assert_allclose(r[:, 1], want, rtol=1e-12)
    ctx.close()
