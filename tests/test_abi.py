"""The C-ABI library loads on a machine without a GPU and exports exactly the
entry points include/evxg.h declares (no compute calls here)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "evxg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(evxg_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_expected_api():
    import chicago_b200 as cb
    assert declared() == sorted(cb.EXPORTS)


def test_library_exports_every_declared_symbol():
    import chicago_b200 as cb
    if not os.path.exists(cb.LIB_PATH):
        pytest.skip("libevxg.so not built")
    lib = C.CDLL(cb.LIB_PATH)
    assert [s for s in declared() if not hasattr(lib, s)] == []


def test_lambda_host_formula(oracle):
    import chicago_b200 as cb
    if not os.path.exists(cb.LIB_PATH):
        pytest.skip("libevxg.so not built")
    for q in range(1, 64):
        assert cb.lam(q) == oracle.lib.orc_lambda(q)


def test_import_fails_loudly_without_library(tmp_path):
    import chicago_b200 as cb
    with pytest.raises(ImportError):
        cb._load(str(tmp_path / "missing.so"))
