"""CPU checks of the C-ABI: the library loads, exports every function the public header
declares, and fails cleanly (status codes, no exit) without a device or with bad input."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu


def header_functions():
    txt = open(os.path.join(ROOT, "include", "gems_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gems_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from gems_b200 import _lib
    lib = _lib.gems()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_strings():
    from gems_b200 import _lib
    lib = _lib.gems()
    assert b"sm_100a" in lib.gems_version()
    assert isinstance(lib.gems_last_error(), bytes)


def test_bad_descriptor_rejected():
    from gems_b200.api import SessionDesc
    from gems_b200 import _lib
    lib = _lib.gems()
    h = ctypes.c_void_p()
    for d in (SessionDesc(2, 10, 4, 4, 1, 0, 0, 0),      # too few taxa
              SessionDesc(8, 10, 5, 4, 6, 0, 0, 0),      # unsupported state count
              SessionDesc(8, 10, 4, 0, 6, 0, 0, 0),      # no categories
              SessionDesc(8, 10, 4, 4, 6, 3, 0, 0)):     # unknown precision
        assert lib.gems_session_create(ctypes.byref(d), ctypes.byref(h)) == 5
        assert not h.value


def test_footprint_admission_numbers():
    from gems_b200.api import Session
    # 512 taxa x 600k patterns, FP64, one slot per internal node: ~39 GB of partials
    b = Session.footprint(512, 600_000, 4, 4, 510)
    assert 38e9 < b < 41e9
    bm = Session.footprint(512, 600_000, 4, 4, 510, precision="mixed")
    assert bm < 0.55 * b


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_status():
    from gems_b200.api import SessionDesc
    from gems_b200 import _lib
    lib = _lib.gems()
    h = ctypes.c_void_p()
    d = SessionDesc(8, 100, 4, 4, 6, 0, 0, 0)
    assert lib.gems_session_create(ctypes.byref(d), ctypes.byref(h)) == 8
    n = ctypes.c_int(-1)
    lib.gems_device_count(ctypes.byref(n))
    assert n.value == 0


def test_tree_rejects_non_binary():
    from gems_b200 import _lib
    lib = _lib.gems()
    eu = np.array([4, 4, 4, 4], np.int32)  # star with 4 leaves: degree-4 node
    ev = np.array([0, 1, 2, 3], np.int32)
    ln = np.full(4, 0.1)
    h = ctypes.c_void_p()
    st = lib.gems_tree_create(None, 4, eu.ctypes.data_as(ctypes.c_void_p),
                              ev.ctypes.data_as(ctypes.c_void_p),
                              ln.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h))
    assert st == 5
