"""4-state traversal kernels (two patterns per lane group) for every category count 1..8: lane
groups with idle lanes (C = 3, 5, 6, 7) and pattern counts that leave the last block partly
filled, NORM and SAFE, against the FP64 oracle.  FP64: lnL and pattern lnL to 1e-9, partials to
1e-10 of their pattern's largest value, scale counters exact.  Mixed: lnL to 1e-6."""
import numpy as np
import pytest

from gems_b200 import GemsError, PhyloTree, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def case(ncat, seed):
    rng = np.random.default_rng(seed)
    model = synth.dna_gtr(rng, ncat, 0.5)
    tree = synth.random_tree(30, 0.1, seed + 1)
    aln = synth.simulate(tree, model, 3001, seed + 2, gap_frac=0.05)
    return tree, model, aln


def internal_branches(tree):
    out = []
    for u, v in zip(tree.eu, tree.ev):
        u, v = int(u), int(v)
        if v >= tree.ntaxa:
            out.append((v, u))
        if u >= tree.ntaxa:
            out.append((u, v))
    return out


@pytest.mark.parametrize("ncat", [1, 2, 3, 5, 6, 7, 8])
@pytest.mark.parametrize("safe", [False, True], ids=["norm", "safe"])
def test_fp64_partials_and_lnl(gpu, ncat, safe):
    tree, model, aln = case(ncat, 70 + ncat)
    ot = orc.OracleTree(tree, model, aln, safe=safe)
    gt = PhyloTree.from_case(tree, model, aln, precision="fp64",
                             scaling="safe" if safe else "norm")
    lo, plo = ot.computeLikelihood(pattern_lh=True)
    lg, plg = gt.computeLikelihood(pattern_lh=True)
    assert abs(lg - lo) <= 1e-9 * abs(lo), (lg, lo)
    assert np.allclose(plg, plo, rtol=1e-9, atol=1e-12)
    checked = 0
    for node, dad in internal_branches(tree):
        try:
            po, so = ot.getPartial(node, dad)
        except AssertionError:
            continue
        try:
            pg, sg = gt.getPartial(node, dad)
        except GemsError:
            continue
        np.testing.assert_array_equal(sg, so)
        scale = np.abs(po).max(axis=(1, 2), keepdims=True) + 1e-300
        assert np.max(np.abs(pg - po) / scale) < 1e-10
        checked += 1
    assert checked >= tree.ntaxa - 2
    gt.close()
    gt.session.close()


@pytest.mark.parametrize("ncat", [1, 2, 3, 5, 6, 7, 8])
@pytest.mark.parametrize("safe", [False, True], ids=["norm", "safe"])
def test_mixed_lnl(gpu, ncat, safe):
    tree, model, aln = case(ncat, 90 + ncat)
    lo = orc.OracleTree(tree, model, aln, safe=safe).computeLikelihood()
    gt = PhyloTree.from_case(tree, model, aln, precision="mixed",
                             scaling="safe" if safe else "norm")
    lg = gt.computeLikelihood()
    assert abs(lg - lo) <= 1e-6 * abs(lo), (lg, lo)
    gt.close()
    gt.session.close()
