"""SPR moves on the device tree against the oracle doing the same moves: the subtree pruned and
regrafted as assessSPRMove does (tree/phylotree.cpp:4822-4880), then Newton on the four branches
swapSPR optimises (tree/phylotree.cpp:4764-4768) and the lnL from the buffers.  After every move
the edge lists agree, the lnL matches the oracle's at the form's bar and every branch length
matches; for all three slot modes (one slot per internal node, per directed branch, and the
LM_MEM_SAVE pool), FP64 and mixed."""
import numpy as np
import pytest

from gems_b200 import GemsError, PhyloTree, synth
from gems_b200.serve import spr4, spr_regraft_branches, tree_move
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def case(n, ntaxa, nsites, seed, ncat=4):
    rng = np.random.default_rng(seed)
    model = synth.dna_gtr(rng, ncat) if n == 4 else synth.protein(rng, ncat)
    tree = synth.random_tree(ntaxa, 0.1, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2)
    return tree, model, aln


def run_pair(tree, model, aln, precision, slots, nreq, move=spr4, tc=None):
    ot = orc.OracleTree(tree, model, aln)
    gt = PhyloTree.from_case(tree, model, aln, precision=precision, slots=slots)
    if tc is not None:
        gt.session.set_tensor_cores(tc)
    ot.computeLikelihood()
    gt.computeLikelihood()
    out = []
    for k in range(nreq):
        lo, _ = move(ot, tree.ntaxa, np.random.default_rng((13, k)))
        lg, _ = move(gt, tree.ntaxa, np.random.default_rng((13, k)))
        np.testing.assert_array_equal(gt.eu, ot.eu)
        np.testing.assert_array_equal(gt.ev, ot.ev)
        out.append((lg, lo, gt.getBranchLengths(), ot.getBranchLengths()))
    gt.close()
    gt.session.close()
    return out


@pytest.mark.parametrize("slots", ["node", "branch", "pool"])
@pytest.mark.parametrize("n", [4, 20])
def test_spr4_fp64(gpu, n, slots):
    tree, model, aln = case(n, 32, 3000, 51 + n)
    for lg, lo, bg, bo in run_pair(tree, model, aln, "fp64", slots, 8):
        assert abs(lg - lo) <= 1e-9 * abs(lo), (lg, lo)
        np.testing.assert_allclose(bg, bo, rtol=1e-7, atol=1e-10)


@pytest.mark.parametrize("n,tc", [(4, None), (20, False), (20, True)])
def test_spr4_mixed(gpu, n, tc):
    tree, model, aln = case(n, 32, 3000, 61 + n)
    for lg, lo, bg, bo in run_pair(tree, model, aln, "mixed", "node", 8, tc=tc):
        assert abs(lg - lo) <= 1e-6 * abs(lo), (lg, lo)
        np.testing.assert_allclose(bg, bo, rtol=2e-4, atol=1e-7)


@pytest.mark.parametrize("slots", ["node", "pool"])
def test_mixed_nni_and_spr_requests(gpu, slots):
    """The serving request mix (NNI and SPR drawn per request) on one session."""
    tree, model, aln = case(4, 40, 2000, 71)
    for lg, lo, bg, bo in run_pair(tree, model, aln, "fp64", slots, 12, move=tree_move):
        assert abs(lg - lo) <= 1e-9 * abs(lo), (lg, lo)
        np.testing.assert_allclose(bg, bo, rtol=1e-7, atol=1e-10)


@pytest.mark.parametrize("slots", ["node", "branch", "pool"])
def test_every_regraft_of_one_prune(gpu, slots):
    """Every regraft branch of one pruned subtree (those next to the joint included), each on a
    fresh tree: the lnL computed after the move equals the oracle's after the same move."""
    tree, model, aln = case(4, 16, 1500, 81)
    base = orc.OracleTree(tree, model, aln)
    node, dad = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                     if a >= tree.ntaxa and b >= tree.ntaxa)
    _, _, cand = spr_regraft_branches(base, node, dad, radius=20)
    assert len(cand) >= 6
    for node2, dad2 in cand:
        ot = orc.OracleTree(tree, model, aln)
        ot.computeLikelihood()
        ot.doSPR(node, dad, node2, dad2)
        lo = ot.computeLikelihood()
        g2 = PhyloTree.from_case(tree, model, aln, precision="fp64", slots=slots)
        g2.computeLikelihood()
        g2.doSPR(node, dad, node2, dad2)
        lg = g2.computeLikelihood()
        assert abs(lg - lo) <= 1e-9 * abs(lo), (node2, dad2, lg, lo)
        np.testing.assert_array_equal(g2.eu, ot.eu)
        g2.close()
        g2.session.close()


def test_bad_spr_refused_tree_unchanged(gpu):
    tree, model, aln = case(4, 12, 500, 91)
    gt = PhyloTree.from_case(tree, model, aln, precision="fp64")
    l0 = gt.computeLikelihood()
    eu, ev = gt.eu.copy(), gt.ev.copy()
    u, v = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa)
    inside = [x for x in gt.neighbors(u) if x != v][0]
    at_dad = [x for x in gt.neighbors(v) if x != u][0]
    for args in ((u, v, inside, u), (u, v, at_dad, v), (gt.neighbors(0)[0], 0, u, v)):
        with pytest.raises(GemsError) as e:
            gt.doSPR(*args)
        assert e.value.status == 5
    np.testing.assert_array_equal(gt.eu, eu)
    np.testing.assert_array_equal(gt.ev, ev)
    assert gt.computeLikelihood() == l0
    gt.close()
    gt.session.close()
