"""CPU checks of the C ABI boundary: libamm.so loads, exports every function include/amm.h
declares, and rejects bad input on the host without touching a device."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    txt = (ROOT / "include" / "amm.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(amm_[a-zA-Z0-9_]+)\s*\(", txt)))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for want in ("amm_power_exact", "amm_power_previous", "amm_power_proposed",
                 "amm_power_proposed_v2", "amm_core_previousAMM", "amm_core_proposedAMM",
                 "amm_rayleigh_normalize", "amm_normalize", "amm_set_matrix", "amm_create",
                 "amm_destroy", "amm_grad_lambda"):
        assert want in names


def test_library_exports_every_declared_symbol(amm_lib):
    missing = [n for n in declared_functions() if not hasattr(amm_lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    from eigenvaluecomputation_by_amm_b200 import _lib
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_status_strings(amm_lib):
    from eigenvaluecomputation_by_amm_b200 import _lib
    for code in range(10):
        s = _lib.status_string(code)
        assert s and s != "unknown status"
    assert _lib.status_string(99) == "unknown status"


def test_config_defaults_mirror_host_memory(amm_lib):
    from eigenvaluecomputation_by_amm_b200._lib import amm_config
    cfg = amm_config()
    amm_lib.amm_config_default(C.byref(cfg))
    # host_memory.h:26-50: m 128, c 0 (-> m), step 10, no VR, not sanity
    assert (cfg.m, cfg.c, cfg.step, cfg.vr_period, cfg.sanity) == (128, 0, 10, 0, 0)
    assert cfg.vr_adaptive_threshold == 0.0 and cfg.use_graph == 1


def _cfg(amm_lib, **kw):
    from eigenvaluecomputation_by_amm_b200._lib import amm_config
    cfg = amm_config()
    amm_lib.amm_config_default(C.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


@pytest.mark.parametrize("kw", [dict(m=0), dict(n=0), dict(step=0), dict(c=-1), dict(dtype=7),
                                dict(cdf_precision=3), dict(vr_period=-1),
                                dict(vr_adaptive_threshold=-0.5)])
def test_create_rejects_bad_config(amm_lib, kw):
    from eigenvaluecomputation_by_amm_b200 import _lib
    ctx = C.c_void_p()
    rc = amm_lib.amm_create(C.byref(ctx), C.byref(_cfg(amm_lib, **kw)), 0)
    assert rc == _lib.AMM_ERR_INVALID_ARGUMENT
    assert not ctx.value


def test_null_arguments_are_rejected(amm_lib):
    from eigenvaluecomputation_by_amm_b200 import _lib
    assert amm_lib.amm_create(None, None, 0) == _lib.AMM_ERR_INVALID_ARGUMENT
    assert amm_lib.amm_destroy(None) == _lib.AMM_ERR_INVALID_ARGUMENT
    assert amm_lib.amm_set_matrix(None, None, 0, None) == _lib.AMM_ERR_INVALID_ARGUMENT
    assert amm_lib.amm_power_method(None, 0, None, None) == _lib.AMM_ERR_INVALID_ARGUMENT
    assert amm_lib.amm_get_trace(None, *([None] * 8)) == _lib.AMM_ERR_INVALID_ARGUMENT


def test_create_without_device_reports_no_device(amm_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from eigenvaluecomputation_by_amm_b200 import _lib
    ctx = C.c_void_p()
    rc = amm_lib.amm_create(C.byref(ctx), C.byref(_cfg(amm_lib, m=1024, n=4096)), 0)
    assert rc == _lib.AMM_ERR_NO_DEVICE


def test_python_api_fails_loudly_without_library(tmp_path, monkeypatch):
    from eigenvaluecomputation_by_amm_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.load(tmp_path / "libamm.so")
