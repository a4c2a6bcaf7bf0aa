"""ctypes loading of the in-tree native libraries (no fallback: a missing library raises)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_synth = None
_gems = None


def synth():
    global _synth
    if _synth is None:
        path = os.path.join(HERE, "libgems_synth.so")
        if not os.path.exists(path):
            from . import build
            build.build_synth()
        lib = ctypes.CDLL(path)
        lib.gems_synth_tree.restype = ctypes.c_int
        lib.gems_synth_simulate.restype = ctypes.c_int
        lib.gems_synth_compress.restype = ctypes.c_longlong
        _synth = lib
    return _synth


def gems():
    """The CUDA library.  Raises OSError when it has not been built."""
    global _gems
    if _gems is None:
        path = os.path.join(HERE, "libgems_b200.so")
        if not os.path.exists(path):
            raise OSError(f"{path} is missing: run `python -m gems_b200.build`")
        _gems = ctypes.CDLL(path)
        _gems.gems_version.restype = ctypes.c_char_p
        _gems.gems_last_error.restype = ctypes.c_char_p
    return _gems
