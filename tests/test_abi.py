"""CPU: the C-ABI library loads and exports every entry point that
include/cj_b200.h declares; host-only calls work without a device."""
import ctypes as C
import os
import re

import numpy as np

from calamarijoins_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cj_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cj_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(_lib._SIGS), set(declared_functions()) ^ set(_lib._SIGS)


def test_version_and_no_device_behaviour():
    lib = _lib.lib()
    assert lib.cj_version().startswith(b"cj_b200")
    h = C.c_void_p()
    rc = lib.cj_context_create(-1, C.byref(h))
    if rc == 0:  # running on a GPU host
        lib.cj_context_destroy(h.value)
    else:
        assert rc == 8  # CJ_ERR_NO_DEVICE, with a message
        assert lib.cj_last_error()


def test_null_arguments_are_rejected():
    lib = _lib.lib()
    assert lib.cj_context_create(0, None) == 1
    assert lib.cj_execute(None, None, 0, None, None, None) == 1
    n = C.c_uint64()
    assert lib.cj_encode_num_pages(9, None, None, None, 0, C.byref(n)) == 1


def test_encoder_page_counts():
    lib = _lib.lib()
    n = C.c_uint64()
    vals = np.arange(1984 * 3, dtype=np.int32)
    assert lib.cj_encode_num_pages(0, vals.ctypes.data, None, None, len(vals), C.byref(n)) == 0
    assert n.value == 3  # 1984 INT32 rows per page
    vals = np.arange(1007 * 2 + 1, dtype=np.int64)
    assert lib.cj_encode_num_pages(1, vals.ctypes.data, None, None, len(vals), C.byref(n)) == 0
    assert n.value == 3  # 1007 INT64 rows per page
