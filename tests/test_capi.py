"""The C-ABI library loads and exports every symbol include/msgpu.h declares.

No compute call is made here (no GPU needed)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "msgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(msgpu_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert "msgpu_register_batch" in syms and "msgpu_warp_mean" in syms
    assert len(syms) >= 15


def test_library_builds_and_exports_all_symbols():
    import msgpu
    from msgpu import build
    build.build()
    lib = ctypes.CDLL(msgpu.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(msgpu.EXPORTS) <= set(declared_symbols())


def test_params_defaults_and_version():
    import msgpu
    p = msgpu.default_params()
    assert (p.precision_level, p.start_level, p.stop_level, p.max_gd_iterations) == (9, 5, 9, 30)
    assert p.lambda_ == pytest.approx(0.1) and p.lambda_factor == 1.0 and p.saturation_percent == pytest.approx(0.15)
    assert msgpu.lib().msgpu_abi_version() == 8


def test_errors_are_reported_not_swallowed():
    import msgpu
    L = msgpu.lib()
    # no context: invalid argument, no crash
    assert L.msgpu_register_batch(None, None, None, None, 0, None, None, None, None) == 1
    assert L.msgpu_last_error(None) == b"no context"
    h = ctypes.c_void_p()
    st = L.msgpu_create(0, ctypes.byref(h))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert st == 3 and not h.value  # CUDA error, loudly
    else:
        assert st == 0
        L.msgpu_destroy(h)
