"""ctypes binding of libamm.so (include/amm.h).  No torch types cross this boundary: every
entry point takes plain integers (device addresses, sizes, streams)."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libamm.so"

# status codes (enum amm_status)
AMM_OK = 0
AMM_ERR_INVALID_ARGUMENT = 1
AMM_ERR_ALIGNMENT = 2
AMM_ERR_UNSUPPORTED = 3
AMM_ERR_NOT_READY = 4
AMM_ERR_DEGENERATE = 5
AMM_ERR_CUDA = 6
AMM_ERR_DEVICE_TIMEOUT = 7
AMM_ERR_OUT_OF_MEMORY = 8
AMM_ERR_NO_DEVICE = 9

AMM_F32, AMM_BF16 = 0, 1
AMM_CDF_F64, AMM_CDF_F32 = 0, 1
METHODS = {"exact": 0, "previous": 1, "proposed": 2, "proposed_v2": 3}
STEP_KINDS = {0: "exact", 1: "exact_nomemo", 2: "previous", 3: "proposed"}


class amm_config(C.Structure):
    _fields_ = [
        ("m", C.c_int64),
        ("n", C.c_int64),
        ("c", C.c_int64),
        ("step", C.c_int64),
        ("vr_period", C.c_int64),
        ("vr_adaptive_threshold", C.c_double),
        ("tol", C.c_double),
        ("dtype", C.c_int32),
        ("cdf_precision", C.c_int32),
        ("sanity", C.c_int32),
        ("use_graph", C.c_int32),
    ]


class amm_batch_matrix(C.Structure):
    _fields_ = [("A", C.c_void_p), ("ld", C.c_int64), ("m", C.c_int64), ("n", C.c_int64)]


class amm_batch_config(C.Structure):
    _fields_ = [
        ("nvec", C.c_int32),
        ("rr_period", C.c_int32),
        ("max_iter", C.c_int64),
        ("tol", C.c_double),
        ("seed", C.c_uint64),
        ("use_graph", C.c_int32),
        ("tile_gc", C.c_int32),
        ("c_divisor", C.c_int32),
        ("cluster", C.c_int32),
        ("wide", C.c_int32),
        ("vr_period", C.c_int32),
    ]


class AmmError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = f"{where}: {status_string(status)}"
        if status == AMM_ERR_CUDA:
            msg += f" ({last_cuda_error()})"
        super().__init__(msg)


_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32

# name -> argtypes (all return int status unless listed in _RET)
_SIGS = {
    "amm_config_default": [C.POINTER(amm_config)],
    "amm_create": [C.POINTER(_P), C.POINTER(amm_config), C.c_int],
    "amm_destroy": [_P],
    "amm_set_matrix": [_P, _P, _I64, _P],
    "amm_set_rng_state": [_P, _P, _I64, _P],
    "amm_get_rng_state": [_P, _P, _I64, _P],
    "amm_seed_rng": [_P, C.c_uint64, _I64, _P],
    "amm_seed_start_vectors": [_P, C.c_uint64],
    "amm_seed_rng_at": [_P, C.c_uint64, C.c_uint64, _I64, _P],
    "amm_seed_start_vectors_at": [_P, C.c_uint64, C.c_uint64],
    "amm_draw_start_vector": [_P, _P, _P],
    "amm_set_cdf": [_P, C.c_int, _P, _P],
    "amm_set_eigenvector": [_P, _P, _P],
    "amm_power_method": [_P, C.c_int, _P, _P],
    "amm_power_exact": [_P, _P, _P],
    "amm_power_previous": [_P, _P, _P],
    "amm_power_proposed": [_P, _P, _P],
    "amm_power_proposed_v2": [_P, _P, _P],
    "amm_get_trace": [_P, _P, _P, _P, _P, _P, _P, _P, _P],
    "amm_get_vectors": [_P, _P, _P, _P],
    "amm_device_clock": [_P, _P],
    "amm_get_step_clocks": [_P, _P, C.c_int64, _P, _P],
    "amm_core_previousAMM": [_P, _P, _P, _P, _P, _P, _P],
    "amm_core_proposedAMM": [_P, _P, _P, _P, _P, _P, _P],
    "amm_exact_product": [_P, _P, _P, _P],
    "amm_core_list_product": [_P, C.c_int, _P, _P, _I64, _P, _P, _P, _P, _P],
    "amm_shard_product": [_P, _P, _I64, _I64, _P, _P, _P, _P, _P, _P, _P],
    "amm_rayleigh_normalize": [_P, _P, _P, _P, _P],
    "amm_normalize": [_P, _P, _P],
    "amm_get_column_stats": [_P, _P, _P, _P, _P, _P, _P, _P],
    "amm_get_sampling_tables": [_P, C.c_int, _P, _P, _P],
    "amm_sample_indices": [_P, C.c_int, _P, _P],
    "amm_pick_sorted_noalloc": [_P, _P, _I64, _P, C.c_int, _I64, _P, _P, _P],
    "amm_generate_matrix": [C.c_char_p, _I64, C.c_uint64, _P, _P, _P],
    "amm_read_matrix_file": [C.c_char_p, _P, _I64, _P],
    "amm_batch_config_default": [C.POINTER(amm_batch_config)],
    "amm_batch_create": [C.POINTER(_P), C.POINTER(amm_batch_matrix), _I64,
                         C.POINTER(amm_batch_config), C.c_int],
    "amm_batch_destroy": [_P],
    "amm_batch_vector_offsets": [_P, _P],
    "amm_batch_run": [_P, _P, _P, _P, _P],
    "amm_batch_run_each": [_P, _P, _P, _P, _P],
    "amm_batch_grad": [_P, _P, _P, _P, _P, _P],
    "amm_batch_tile_choice": [_P, _P, _P, _P],
    "amm_batch_record": [_P, _P, _P, _I64],
    "amm_batch_set_matrices": [_P, C.POINTER(amm_batch_matrix), _I64, _P],
    "amm_batch_wide_plan": [_P, _P, _P, _P, _P],
    "amm_probe_bounded_waits": [_P, _P, _P],
    "amm_benchmark_product": [_P, C.c_int, C.c_int, _P, _P, _P],
    "amm_grad_lambda": [_P, _P, _P, _I64, _P],
    "amm_get_geometry": [_P, _P],
    "amm_status_string": [C.c_int],
    "amm_last_cuda_error": [],
    "amm_kernel_launch_count": [],
}
_RET = {
    "amm_config_default": None,
    "amm_batch_config_default": None,
    "amm_status_string": C.c_char_p,
    "amm_last_cuda_error": C.c_char_p,
    "amm_kernel_launch_count": C.c_int64,
}

_lib = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load libamm.so (raises ImportError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python -m eigenvaluecomputation_by_amm_b200.build` "
            "(nvcc, sm_100a); there is no CPU fallback")
    lib = C.CDLL(str(p))
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RET.get(name, C.c_int)
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


def status_string(status: int) -> str:
    return load().amm_status_string(int(status)).decode()


def last_cuda_error() -> str:
    return load().amm_last_cuda_error().decode()


def check(status: int, where: str) -> None:
    if status != AMM_OK:
        raise AmmError(status, where)


def launch_count() -> int:
    return int(load().amm_kernel_launch_count())
