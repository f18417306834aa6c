"""The C-ABI library loads without a GPU and exports every declared entry point."""
import os
import re

from next_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(next_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("next_create", "next_upload", "next_step", "next_accel", "next_adaptive_dt",
                     "next_download", "next_destroy", "next_last_error"):
        assert required in names


def test_every_declared_symbol_is_exported():
    lib = native.load()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert declared_functions() <= set(native.SIGNATURES)


def test_status_strings_without_gpu():
    lib = native.load()
    assert lib.next_status_string(0) == b"ok"
    assert lib.next_status_string(5) == b"device error"


def test_invalid_params_rejected_without_gpu():
    import ctypes as C
    lib = native.load()
    p = native.Params()
    assert lib.next_params_default(C.byref(p), 1, 1) == 0
    assert p.leaf_cap == 16 and p.reuse_forces == 1
    bad = native.Params()
    lib.next_params_default(C.byref(bad), 0, 1)      # mixed precision needs accurate physics
    h = C.c_void_p()
    assert lib.next_create(C.byref(bad), C.byref(h)) == 1
    bad.physics = 1
    bad.group_cap = 64                               # groups are at most one warp wide
    assert lib.next_create(C.byref(bad), C.byref(h)) == 1
