"""The C-ABI library loads and exports every symbol include/umagnus_b200.h
declares (no device work: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT
from umagnus_b200 import _lib

HEADER = os.path.join(ROOT, "include", "umagnus_b200.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(umag_\w+)\s*\(", src, re.M)))


def test_header_declares_functions():
    names = header_functions()
    assert len(names) >= 45
    assert "umag_demag_exec" in names and "umag_sim_steps" in names


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")
def test_library_exports_every_header_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(_lib.exported_names()) == header_functions()


@pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="library not built")
def test_calls_before_init_fail_loudly():
    L = _lib.load()
    if _lib._initialised is not None:
        pytest.skip("already initialised in this process")
    rc = L.umag_sync()
    assert rc == 5  # UMAG_E_NOT_INIT
    assert b"umag_init" in L.umag_last_error()
