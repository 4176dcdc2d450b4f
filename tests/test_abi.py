"""CPU tests of the C-ABI library: it loads, exports every symbol that
include/gila_b200.h declares, and fails cleanly (no abort) without a GPU."""
from __future__ import annotations

import ctypes as ct
import os
import re

import pytest

from conftest import ROOT, has_gpu, load_pkg


def _declared():
    src = open(os.path.join(ROOT, "include", "gila_b200.h")).read()
    return sorted(set(re.findall(r"\b(gila_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    gila = load_pkg()
    h = gila._lib.lib()
    missing = [n for n in _declared() if not hasattr(h, n)]
    assert not missing, missing
    # the binding covers every declared entry point
    assert set(_declared()) <= set(gila._lib.exported_symbols())


def test_status_strings_and_version():
    gila = load_pkg()
    h = gila._lib.lib()
    assert h.gila_version().decode().count(".") == 2
    for s in range(13):
        assert h.gila_status_string(s)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_is_an_error_not_an_abort():
    gila = load_pkg()
    h = gila._lib.lib()
    c = ct.c_void_p()
    st = h.gila_ctx_create(0, ct.byref(c))
    assert st == gila._lib.GILA_ERR_NODEV
    assert "CUDA is not functional" in gila._lib.last_error()


def test_null_arguments_rejected():
    gila = load_pkg()
    h = gila._lib.lib()
    assert h.gila_opr_apply(None, 1, None, 0, None, 0, 1, None) == gila._lib.GILA_ERR_ARG
    assert h.gila_opr_sizes(None, (ct.c_int64 * 4)(), (ct.c_int64 * 4)()) == gila._lib.GILA_ERR_ARG
