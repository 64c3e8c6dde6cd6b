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


def test_unsupported_dimensions_are_refused_without_a_gpu():
    """rbmpp_create checks the sizes before touching a device: a negative unit count, an odd site count and a
    lattice beyond the supported size come back as RBMPP_E_ARG with a message."""
    build.build()
    lib = capi.lib()
    cases = [(dict(L=4, alphac=-1), "bad dimensions"), (dict(L=5), "unsupported L"), (dict(L=24), "unsupported L")]
    for kw, msg in cases:
        d = capi.Dims(kw.get("L", 4), 1, kw.get("alphac", 0), 1, 16, 1, 1, 1, 1.0, 0.5, 0, 0)
        h = ctypes.c_void_p()
        rc = lib.rbmpp_create(ctypes.byref(d), ctypes.byref(h))
        try:
            assert rc == 1, (kw, rc)
            assert msg in lib.rbmpp_last_error(h).decode(), kw
        finally:
            lib.rbmpp_destroy(h)
