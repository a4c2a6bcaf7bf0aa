import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def golden_opt_files():
    """Golden cases that carry the program's optimised branch lengths."""
    return [p for p in golden_files() if "ref_lnl_opt" in np.load(p).files]


def load_golden(path):
    """Inputs of a golden case as (tree, model, aln, z) with the oracle's eigensystem."""
    from gems_b200 import synth
    from oracle import oracle as orc
    z = np.load(path)
    n = int(z["nstates"])
    tree = synth.Tree(int(z["ntaxa"]), z["eu"], z["ev"], z["length"])
    ev, v, iv = orc.eigensystem(z["exch_upper"], z["freq"])
    model = synth.Model(n, z["exch_upper"], z["freq"], z["rates"], z["props"], ev, v, iv,
                        p_invar=float(z["p_invar"]), gamma_shape=float(z["alpha"]))
    aln = synth.Alignment(int(z["ntaxa"]), n, int(z["weights"].sum()), z["patterns"],
                          z["weights"])
    return tree, model, aln, z


def ptn_invar(model, aln):
    """ptn_invar as computePtnInvar forms it (phylotreesse.cpp:549-612), for the GPU upload."""
    p = model.p_invar
    out = np.zeros(aln.npat)
    if p == 0:
        return out
    from gems_b200.synth import state_unknown
    cc = aln.const_char()
    unk = state_unknown(model.nstates)
    freq = np.asarray(model.freq) / np.sum(model.freq)
    for i, c in enumerate(cc):
        if c > unk:
            continue
        if c == unk:
            out[i] = p
        elif c < model.nstates:
            out[i] = p * freq[c]
        elif model.nstates == 4:
            bm = c - 3
            out[i] = p * sum(freq[x] for x in range(4) if bm & (1 << x))
    return out


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from gems_b200 import _lib
    _lib.gems()
    return True
