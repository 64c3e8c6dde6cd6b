"""The C-ABI library loads without a GPU and exports every entry point include/rbmpp.h declares."""
import ctypes
import os
import re

from rbm_pp_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "rbmpp.h")).read()
    return sorted(set(re.findall(r"\b(rbmpp_[a-z0-9_]+)\s*\(", src)))


def test_header_matches_binding_list():
    assert declared_symbols() == sorted(capi.EXPORTS)


def test_library_exports_all_symbols():
    build.build()
    lib = ctypes.CDLL(capi.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name
