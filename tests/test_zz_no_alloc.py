"""The allocation-free entry point, gems_lnl_from_theta_noalloc.

It exists for callers that cannot allocate device memory when they evaluate a likelihood: a
host whose own memory pool has reserved the device, an embedding that accounts every device
byte itself, or a loop that must not hit cudaMalloc/cudaFree (both synchronise the device).
Its scratch is a fixed device array of the library instead of a cudaMalloc'd buffer.

Here it is called through the C-ABI on a theta buffer the test owns (allocated by torch, as
such a caller would own it), twice in a row at two branch lengths, and must give what the
session entry point gems_lnl_from_buffer gives on the same theta (to 1e-12) and what the
oracle's computeLikelihoodFromBuffer gives (to the FP64 bar, 1e-9).  Cases cover 4, 20 and 61
states; 1, 3, 4 and 8 categories (3 leaves idle lanes in a power-of-two lane group); NORM and
SAFE theta; with and without +I; the default stream and a caller's stream.  The free device
memory is the same before and after the second call.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import ptn_invar
from gems_b200 import PhyloTree, synth
from gems_b200 import _lib
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

RTOL = 1e-12        # against the session entry point (same theta, same device sums)
RTOL_ORACLE = 1e-9  # against the FP64 oracle

# (states, categories, scaling, p_invar, caller stream)
CASES = [
    (4, 1, "norm", 0.0, False),
    (4, 3, "norm", 0.2, False),
    (4, 4, "safe", 0.0, True),
    (4, 8, "norm", 0.0, False),
    (20, 4, "norm", 0.15, True),
    (61, 4, "safe", 0.0, False),
]
IDS = [f"n{n}-c{c}-{sc}-{'inv' if p else 'noinv'}-{'stream' if st else 'default'}"
       for n, c, sc, p, st in CASES]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _model(n, ncat, seed):
    rng = np.random.default_rng(seed)
    if n == 4:
        return synth.dna_gtr(rng, ncat, 0.6)
    if n == 20:
        return synth.protein(rng, ncat, 0.8)
    return synth.codon_gy(rng, ncat, 0.5)


def _call(lib, d_theta, d_scale, d_freq, d_invar, npat, n, model, length, stream):
    ev = np.ascontiguousarray(model.eval, np.float64)
    rt = np.ascontiguousarray(model.rates, np.float64)
    pr = np.ascontiguousarray(model.props, np.float64)
    out = ctypes.c_double()
    st = lib.gems_lnl_from_theta_noalloc(
        _ptr(d_theta), _ptr(d_scale), _ptr(d_freq),
        _ptr(d_invar) if d_invar is not None else None, npat, n, model.ncat,
        ev.ctypes.data_as(ctypes.c_void_p), rt.ctypes.data_as(ctypes.c_void_p),
        pr.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(length), stream,
        ctypes.byref(out))
    assert st == 0, lib.gems_last_error()
    return out.value


@pytest.mark.parametrize("n,ncat,scaling,pinv,use_stream", CASES, ids=IDS)
def test_noalloc_matches_session_and_oracle(gpu, n, ncat, scaling, pinv, use_stream):
    import torch
    model = _model(n, ncat, 100 + n + ncat)
    model.p_invar = pinv
    tree = synth.random_tree(10, 0.12, 200 + n + ncat)
    aln = synth.simulate(tree, model, 600 if n == 61 else 2000, 300 + n + ncat)
    safe = scaling == "safe"
    invar = ptn_invar(model, aln)
    gt = PhyloTree.from_case(tree, model, aln, scaling=scaling, invar=invar)
    ot = orc.OracleTree(tree, model, aln, safe=safe, const_char=aln.const_char())
    s = gt.session
    e = 4
    u, v = int(tree.eu[e]), int(tree.ev[e])
    gt.computeLikelihoodDerv(v, u)  # builds theta for branch (u, v) in the session
    theta, scale_all = s.get_theta()
    dev = torch.device("cuda:0")
    d_theta = torch.tensor(theta, dtype=torch.float64, device=dev).contiguous()
    d_scale = torch.tensor(scale_all, dtype=torch.float64, device=dev)
    d_freq = torch.tensor(aln.weights, dtype=torch.float64, device=dev)
    d_invar = torch.tensor(invar, dtype=torch.float64, device=dev) if pinv > 0 else None
    torch.cuda.synchronize()
    lib = _lib.gems()
    stream = torch.cuda.Stream() if use_stream else None
    handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    for k, length in enumerate((float(tree.length[e]), 0.37)):
        free_before = torch.cuda.mem_get_info()[0]
        got = _call(lib, d_theta, d_scale, d_freq, d_invar, aln.npat, n, model, length, handle)
        if k == 1:  # the first call may load the kernels' module; the second allocates nothing
            assert torch.cuda.mem_get_info()[0] == free_before
        ref = s.lnl_from_buffer(length)
        assert abs(got - ref) <= RTOL * abs(ref), (got, ref)
        # the oracle's lnL from buffer is taken at the branch computeFuncDerv made current
        ot.computeFuncDerv(u, v, length, new_branch=(k == 0))
        lo = ot.computeLikelihoodFromBuffer()
        assert abs(got - lo) <= RTOL_ORACLE * abs(lo), (got, lo)


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
