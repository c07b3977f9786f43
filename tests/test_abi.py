"""CPU checks of the drop-in boundary: the CUDA library loads without a GPU
and exports exactly the entry points include/ckks_b200.h declares."""
import ctypes
import os
import re

import ckks_b200 as cb


def declared_symbols():
    text = open(cb.HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ckks_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = cb.lib()
    names = declared_symbols()
    assert len(names) >= 9
    for name in names:
        assert hasattr(lib, name), name


def test_binding_covers_header():
    assert set(declared_symbols()) <= set(cb._SIGS)


def test_error_string_without_gpu():
    lib = cb.lib()
    assert lib.ckks_version().startswith(b"ckks_b200")
    h = ctypes.c_void_p()
    rc = lib.ckks_ctx_create(1, None, 0, None, 0, ctypes.byref(h))
    assert rc == -1
    assert b"log_n" in lib.ckks_last_error_string()
