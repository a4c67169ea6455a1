"""The C-ABI library: loads, exports every declared symbol, and its host-side
element tables (C++, no GPU) match the reference's golden tables."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "maple_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(maple_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_api():
    names = declared_functions()
    assert "maple_ctx_create" in names and "maple_oc_step" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in maple_b200.h but not exported"


def test_binding_covers_header(lib):
    from maple_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES), "ctypes binding misses a declared entry point"


@pytest.mark.parametrize("r", [8, 16, 32])
def test_host_element_tables_match_reference(lib, golden, r):
    from maple_b200.core import element_matrices
    g = golden("element_tables.npz")
    mine = element_matrices(r)
    for name, m in zip(("Ke3", "Fe3", "X03", "Ke1", "Fe1", "X01"), mine):
        ref = g[f"r{r}_{name}"]
        assert np.abs(m - ref).max() / np.abs(ref).max() < 1e-12, name


def test_error_reporting_without_gpu(lib):
    from maple_b200 import _lib
    st = lib.maple_box_filter(8, 1, 2, None, None, None)
    assert st == _lib.MAPLE_OK + 1  # MAPLE_E_BADARG
    msg = lib.maple_last_error_string().decode()
    assert "NULL" in msg or "odd" in msg
    with pytest.raises(_lib.MapleError):
        _lib.check(st)


def test_element_matrices_rejects_bad_resolution(lib):
    buf = np.zeros(576)
    p = buf.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.maple_element_matrices(0, 1.0, 0.3, 1.0, p, None, None, None, None, None) != 0
