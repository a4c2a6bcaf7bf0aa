"""The 20-state tcgen05 traversal at two CTAs per SM in half-steps (GEMS_OPT_TC20_HALVES) gives
the same values as the one-CTA form, bit for bit: lnL, pattern lnL, every internal partial and
every scale counter, NORM and SAFE, 1 to 4 categories, pattern counts that leave a ragged last
tile, and a deep tree whose rows underflow (NORM scaling decided after the last half-step, the
first half-step's rows rescaled afterwards)."""
import numpy as np
import pytest

from gems_b200 import PhyloTree, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def run(tree, model, aln, scaling, halves):
    gt = PhyloTree.from_case(tree, model, aln, precision="mixed", scaling=scaling)
    gt.session.set_tc20_halves(halves)
    lnl, plh = gt.computeLikelihood(pattern_lh=True)
    parts = []
    for u, v in zip(tree.eu.tolist(), tree.ev.tolist()):
        for node, dad in ((u, v), (v, u)):
            if node >= tree.ntaxa:
                try:
                    parts.append(gt.getPartial(node, dad))
                except Exception:
                    pass  # not resident in this orientation
    gt.close()
    gt.session.close()
    return lnl, plh, parts


@pytest.mark.parametrize("ncat", [1, 2, 3, 4])
@pytest.mark.parametrize("scaling", ["norm", "safe"])
def test_halves_same_bits(gpu, ncat, scaling):
    rng = np.random.default_rng(100 + ncat)
    model = synth.protein(rng, ncat, 0.7)
    tree = synth.random_tree(26, 0.15, 101 + ncat)
    aln = synth.simulate(tree, model, 900, 102 + ncat, gap_frac=0.03)
    a = run(tree, model, aln, scaling, False)
    b = run(tree, model, aln, scaling, True)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    assert len(a[2]) == len(b[2]) > 0
    for (pa, sa), (pb, sb) in zip(a[2], b[2]):
        np.testing.assert_array_equal(pa, pb)
        np.testing.assert_array_equal(sa, sb)
    ot = orc.OracleTree(tree, model, aln, safe=scaling == "safe")
    lo = ot.computeLikelihood()
    assert abs(b[0] - lo) <= 1e-6 * abs(lo)


@pytest.mark.parametrize("scaling", ["norm", "safe"])
def test_halves_with_underflow(gpu, scaling):
    rng = np.random.default_rng(7)
    model = synth.protein(rng, 4, 0.6)
    tree = synth.random_tree(150, 0.9, 8)     # long branches: deep rows underflow
    aln = synth.simulate(tree, model, 500, 9)
    a = run(tree, model, aln, scaling, False)
    b = run(tree, model, aln, scaling, True)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    scaled = sum(int(np.count_nonzero(s)) for _, s in b[2])
    assert scaled > 0, "the case must exercise the scaling path"
    for (pa, sa), (pb, sb) in zip(a[2], b[2]):
        np.testing.assert_array_equal(pa, pb)
        np.testing.assert_array_equal(sa, sb)
