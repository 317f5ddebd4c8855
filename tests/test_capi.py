"""The C ABI library loads and exports every symbol include/trench_b200.h declares.

CPU only: no compute call is made; tb_create on a machine without a GPU must
fail with TB_ERR_DEVICE and a message, never crash.
"""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from trench_b200 import _capi, build

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "trench_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(tb_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _capi.lib()


def test_header_declares_the_boundary():
    names = header_functions()
    for required in ("tb_create", "tb_destroy", "tb_last_error", "tb_set_fields", "tb_trace", "tb_check"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_capi.SIGNATURES) >= set(header_functions())


def test_trace_args_layout_matches_header():
    # 8-byte aligned struct; the n field first and write_state last, as declared.
    assert _capi.TraceArgs.n.offset == 0
    assert _capi.TraceArgs.d_x.offset == 8
    assert ctypes.sizeof(_capi.TraceArgs) % 8 == 0


def test_create_without_device_reports_error(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    vac = np.ones((4, 5), dtype=np.uint8)
    h = ctypes.c_void_p()
    code = lib.tb_create(ctypes.byref(h), 0, 4, 5, 1e-9, vac.ctypes.data_as(ctypes.c_void_p))
    assert code == _capi.TB_ERR_DEVICE
    assert b"not available" in lib.tb_last_error(None)
    assert not h.value


def test_invalid_grid_is_rejected_before_touching_a_device(lib):
    vac = np.ones((4, 5), dtype=np.uint8)
    h = ctypes.c_void_p()
    code = lib.tb_create(ctypes.byref(h), 0, 0, 5, 1e-9, vac.ctypes.data_as(ctypes.c_void_p))
    assert code == _capi.TB_ERR_ARG
    assert b"invalid grid" in lib.tb_last_error(None)


def test_tracer_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from trench_b200.tracer import B200Tracer
    with pytest.raises(RuntimeError):
        B200Tracer(np.ones((4, 5), bool))


def test_entry_points_reject_a_missing_context(lib):
    """Every call taking a context returns TB_ERR_ARG for a null one, without touching a device."""
    null = None
    assert lib.tb_set_rf_fields(null, null, null, null, null, null, 0, null) == _capi.TB_ERR_ARG
    assert lib.tb_set_tuning(null, 1024, 1) == _capi.TB_ERR_ARG
    assert lib.tb_set_claim_order(null, 0) == _capi.TB_ERR_ARG
    assert lib.tb_reserve_claim_order(null, 10) == _capi.TB_ERR_ARG
    assert lib.tb_batch_reset(null, null, null, 0, null, 0, null, 0, null) == _capi.TB_ERR_ARG
    assert lib.tb_trace(null, null, 1, null) == _capi.TB_ERR_ARG
    assert lib.tb_check(null, null) == _capi.TB_ERR_ARG
    assert lib.tb_inject(null, null, null) == _capi.TB_ERR_ARG
    assert lib.tb_pack_trace(null, 1, null) == _capi.TB_ERR_ARG
