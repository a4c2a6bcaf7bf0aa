"""The allocation-free entry point, gems_lnl_from_theta_noalloc.

It exists for callers that cannot allocate device memory when they evaluate a likelihood:
code running under a CUDA stream capture, hosts whose memory pool owns the whole device, or
a loop that must stay off the allocator.  Its scratch is a fixed device array of the library
instead of a cudaMalloc'd buffer.  Here it is called through the C-ABI on a theta buffer the
test owns (allocated by torch, as such a caller would own it), twice in a row at two branch
lengths, and must give what the session entry point gems_lnl_from_buffer gives on the same
theta.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from gems_b200 import PhyloTree, synth
from gems_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_session_entry_point(gpu):
    import torch
    tree, model, aln = synth.config_dna16(seed=21, nsites=4000)
    gt = PhyloTree.from_case(tree, model, aln)
    s = gt.session
    u, v = int(tree.eu[2]), int(tree.ev[2])
    gt.computeLikelihoodDerv(v, u)  # builds theta for branch (u, v) in the session
    theta, scale_all = s.get_theta()
    dev = torch.device("cuda:0")
    d_theta = torch.tensor(theta, dtype=torch.float64, device=dev).contiguous()
    d_scale = torch.tensor(scale_all, dtype=torch.float64, device=dev)
    d_freq = torch.tensor(aln.weights, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    lib = _lib.gems()
    ev = np.ascontiguousarray(model.eval, np.float64)
    rt = np.ascontiguousarray(model.rates, np.float64)
    pr = np.ascontiguousarray(model.props, np.float64)
    for length in (float(tree.length[2]), 0.37):
        ref = s.lnl_from_buffer(length)
        out = ctypes.c_double()
        st = lib.gems_lnl_from_theta_noalloc(
            _ptr(d_theta), _ptr(d_scale), _ptr(d_freq), None, aln.npat, 4, model.ncat,
            ev.ctypes.data_as(ctypes.c_void_p), rt.ctypes.data_as(ctypes.c_void_p),
            pr.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(length), None,
            ctypes.byref(out))
        assert st == 0, lib.gems_last_error()
        assert abs(out.value - ref) <= RTOL * abs(ref), (out.value, ref)


def test_noalloc_rejects_oversize(gpu):
    lib = _lib.gems()
    dummy = ctypes.c_void_p(16)
    one = np.ones(4)
    out = ctypes.c_double()
    # 4 categories: at most 1,048,576 patterns fit the fixed scratch
    st = lib.gems_lnl_from_theta_noalloc(
        dummy, dummy, dummy, None, 2_000_000, 4, 4, one.ctypes.data_as(ctypes.c_void_p),
        one.ctypes.data_as(ctypes.c_void_p), one.ctypes.data_as(ctypes.c_void_p),
        ctypes.c_double(0.1), None, ctypes.byref(out))
    assert st == 5
    assert b"scratch" in lib.gems_last_error()
