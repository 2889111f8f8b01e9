"""CPU checks of the C ABI boundary: the library builds, loads and exports
every entry point include/fibrenet.h declares; without a GPU it refuses to
create a context instead of falling back to anything."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def declared():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        names |= set(re.findall(r"FN_\w*API\s+[\w\s\*]+?\b(fn_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    assert "fn_create" in names and "fn_step" in names and "fn_upload" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from fibrenet_b200 import build, native
    build.build()
    lib = C.CDLL(native.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    # and the binding knows every one of them
    assert not [n for n in declared() if n not in native.SIGNATURES]


def test_no_device_means_error_not_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fibrenet_b200 import native
    lib = native.load()
    cfg = native.FnConfig(0, 64, 64, 1, 0, 0, 0)
    h = C.c_void_p()
    rc = lib.fn_create(C.byref(cfg), C.byref(h))
    assert rc == 2  # FN_ERR_CUDA
    assert not h.value


def test_detmath_acos_close_to_libm(oracle_built):
    """The device arc cosine (IEEE ops only, shared with the mirror checker)
    stays within 2 ulp of the C library's acos over [-1, 1]."""
    import math

    import numpy as np
    lib = C.CDLL(oracle_built.ORACLE_SO)
    lib.fo_detmath_acos.restype = C.c_double
    lib.fo_detmath_acos.argtypes = [C.c_double]
    xs = np.concatenate([np.linspace(-1, 1, 20001), 1 - np.logspace(-16, 0, 400),
                         -1 + np.logspace(-16, 0, 400)])
    worst = 0.0
    for x in xs:
        a = lib.fo_detmath_acos(float(x))
        b = math.acos(float(x))
        ulp = math.ulp(b) if b != 0 else 5e-324
        worst = max(worst, abs(a - b) / ulp)
    assert worst <= 2.0, worst
