"""ctypes wrapper of oracle/_ref/libamm_ref.so — the reference's own kernels and drivers
compiled for sm_100a (see ref_harness.cu and the Makefile beside it).

TEST INFRASTRUCTURE ONLY: used by the reference-parity GPU tests and by the script that
generates tests/golden/.  It needs a CUDA device; it never reads the reference sources at run
time (only the prebuilt library).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libamm_ref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle REF=<reference checkout>)")
        _lib = C.CDLL(str(LIB))
        P = C.c_void_p
        _lib.ref_draw_x0.argtypes = [C.c_int64, C.c_uint64, P]
        _lib.ref_seed_states.argtypes = [C.c_int64, C.c_uint64, P]
        _lib.ref_power_method.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                          C.c_double, C.c_int, P, C.c_uint64, P, P] + [P] * 12
        _lib.ref_amm_steps.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                       P, P, P] + [P] * 7
        _lib.ref_pick_index.argtypes = [C.c_int64, C.c_int64, P, P, P, P]
        _lib.ref_generate.argtypes = [C.c_char_p, C.c_int64, C.c_uint32, P, P]
        for f in (_lib.ref_draw_x0, _lib.ref_seed_states, _lib.ref_power_method,
                  _lib.ref_amm_steps, _lib.ref_pick_index, _lib.ref_generate):
            f.restype = C.c_int
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with {rc}")


def generate(matrix_type: str, m: int, seed: int):
    """The reference's generate_matrix (device_memory.h:360-433): (A column-major m x m with the
    diagonal offset added, offset)."""
    out = np.zeros(m * m, np.float32)
    off = np.zeros(1, np.float32)
    _check(load().ref_generate(matrix_type.encode(), m, seed, _p(out), _p(off)), "ref_generate")
    return out.reshape(m, m).T, float(off[0])   # element (r, c) at out[r + c*m]


def draw_x0(m: int, x0_seed: int) -> np.ndarray:
    out = np.zeros(m, np.float32)
    _check(load().ref_draw_x0(m, x0_seed, _p(out)), "ref_draw_x0")
    return out


def seed_states(m: int, seed: int) -> np.ndarray:
    out = np.zeros(m, np.uint32)
    _check(load().ref_seed_states(m, seed, _p(out)), "ref_seed_states")
    return out


def pick_index(cdf: np.ndarray, states: np.ndarray):
    cdf = np.ascontiguousarray(cdf, np.float32)
    st = np.ascontiguousarray(states, np.uint32)
    idx = np.zeros(len(st), np.uint32)
    st_out = np.zeros(len(st), np.uint32)
    _check(load().ref_pick_index(len(cdf), len(st), _p(cdf), _p(st), _p(idx), _p(st_out)),
           "ref_pick_index")
    return idx, st_out


def power_method(kernel: str, A: np.ndarray, x0_seed: int, states: np.ndarray, *, c: int,
                 step: int, vr_period: int = 0, vr_thr: float = 0.0, sanity: bool = False,
                 vstar=None) -> dict:
    """One powerMethod_by_<kernel> call; A is square (m, m) and used column-major."""
    m = A.shape[0]
    Acm = np.asfortranarray(A, dtype=np.float32).ravel(order="F")
    st = np.ascontiguousarray(states, np.uint32)
    vs = None if vstar is None else np.ascontiguousarray(vstar, np.float64)
    out = dict(eigs=np.zeros(step), errs=np.zeros(step), x=np.zeros(m, np.float32),
               y=np.zeros(m, np.float32), alpha=np.zeros(m, np.float32),
               norm=np.zeros(m, np.float32), normp=np.zeros(m, np.float32),
               cdf=np.zeros(m, np.float32), weight=np.zeros(m, np.float32),
               sorted=np.zeros(c, np.uint32), states=np.zeros(m, np.uint32),
               time_ms=np.zeros(1, np.float32))
    rc = load().ref_power_method(kernel.encode(), m, c, step, vr_period, vr_thr, int(sanity),
                                 _p(Acm), x0_seed, _p(st), _p(vs), _p(out["eigs"]),
                                 _p(out["errs"]), _p(out["x"]), _p(out["y"]), _p(out["alpha"]),
                                 _p(out["norm"]), _p(out["normp"]), _p(out["cdf"]),
                                 _p(out["weight"]), _p(out["sorted"]), _p(out["states"]),
                                 _p(out["time_ms"]))
    _check(rc, f"ref_power_method({kernel})")
    return out


def amm_steps(kernel: str, A: np.ndarray, x0: np.ndarray, states: np.ndarray, *, c: int,
              nsteps: int, sanity: bool = False) -> dict:
    m = A.shape[0]
    Acm = np.asfortranarray(A, dtype=np.float32).ravel(order="F")
    x0 = np.ascontiguousarray(x0, np.float32)
    st = np.ascontiguousarray(states, np.uint32)
    out = dict(sorted=np.zeros((nsteps, c), np.uint32), tmp=np.zeros((nsteps, c), np.float32),
               y=np.zeros((nsteps, m), np.float32), eigs=np.zeros(nsteps),
               cdf=np.zeros(m, np.float32), weight=np.zeros(m, np.float32),
               states=np.zeros(m, np.uint32))
    rc = load().ref_amm_steps(kernel.encode(), m, c, nsteps, int(sanity), _p(Acm), _p(x0), _p(st),
                              _p(out["sorted"]), _p(out["tmp"]), _p(out["y"]), _p(out["eigs"]),
                              _p(out["cdf"]), _p(out["weight"]), _p(out["states"]))
    _check(rc, f"ref_amm_steps({kernel})")
    return out
