"""NNI moves on the device tree against the oracle: after each doNNI + Newton on the five
branches around the swapped branch, the lnL read from the buffers and every branch length
agree with the oracle doing the same (phylotree.cpp:4059 doNNI, :4176 NNI-5 evaluation)."""
import numpy as np
import pytest

from conftest import load_golden, golden_files, ptn_invar
from gems_b200 import PhyloTree, synth
from gems_b200.serve import nni5
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def case(n, ntaxa, nsites, seed, ncat=4):
    rng = np.random.default_rng(seed)
    model = synth.dna_gtr(rng, ncat) if n == 4 else synth.protein(rng, ncat)
    tree = synth.random_tree(ntaxa, 0.1, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2)
    return tree, model, aln


def run_pair(tree, model, aln, precision, slots, nreq, safe=False, tc=None, invar=None,
             const_char=None):
    ot = orc.OracleTree(tree, model, aln, safe=safe, const_char=const_char)
    gt = PhyloTree.from_case(tree, model, aln, precision=precision, slots=slots,
                             scaling="safe" if safe else "norm", invar=invar)
    if tc is not None:
        gt.session.set_tensor_cores(tc)
    ot.computeLikelihood()
    gt.computeLikelihood()
    out = []
    for k in range(nreq):
        lo, _ = nni5(ot, tree.ntaxa, np.random.default_rng((11, k)))
        lg, _ = nni5(gt, tree.ntaxa, np.random.default_rng((11, k)))
        np.testing.assert_array_equal(gt.eu, ot.eu)
        np.testing.assert_array_equal(gt.ev, ot.ev)
        out.append((lg, lo, gt.getBranchLengths(), ot.getBranchLengths()))
    return out


@pytest.mark.parametrize("slots", ["node", "branch", "pool"])
@pytest.mark.parametrize("n", [4, 20])
def test_nni5_fp64(gpu, n, slots):
    tree, model, aln = case(n, 24, 3000, 21 + n)
    for lg, lo, bg, bo in run_pair(tree, model, aln, "fp64", slots, 6):
        assert abs(lg - lo) <= 1e-9 * abs(lo), (lg, lo)
        np.testing.assert_allclose(bg, bo, rtol=1e-7, atol=1e-10)


@pytest.mark.parametrize("path", [p for p in golden_files() if "safe" in p or "inv" in p])
def test_nni5_fp64_golden(gpu, path):
    """SAFE scaling and invariant sites through NNI moves."""
    tree, model, aln, z = load_golden(path)
    safe = bool(z["safe"])
    res = run_pair(tree, model, aln, "fp64", "node", 4, safe=safe,
                   invar=ptn_invar(model, aln), const_char=z["const_char"])
    for lg, lo, bg, bo in res:
        assert abs(lg - lo) <= 1e-9 * abs(lo), (lg, lo)
        np.testing.assert_allclose(bg, bo, rtol=1e-7, atol=1e-10)


@pytest.mark.parametrize("tc", [False, True])
@pytest.mark.parametrize("n", [4, 20])
def test_nni5_mixed(gpu, n, tc):
    if n == 4 and tc:
        pytest.skip("tensor-core form is for 20 states")
    tree, model, aln = case(n, 24, 3000, 31 + n)
    for lg, lo, bg, bo in run_pair(tree, model, aln, "mixed", "node", 6, tc=tc):
        assert abs(lg - lo) <= 1e-6 * abs(lo), (lg, lo)
        np.testing.assert_allclose(bg, bo, rtol=2e-4, atol=1e-7)


def oracle_evaluate_nni(ot, u, v, max_nr=10):
    """getBestNNIForBran's NNI-5 evaluation done by hand on the oracle, in the canonical order
    gems_tree_nni_evaluate uses (u's smaller other neighbour a against each of v's other
    neighbours b in id order; u's outer branches, the central one, v's outer branches, outer
    ones in id order); the lengths carry over from the first move to the second and are put
    back at the end."""
    saved = ot.getBranchLengths().copy()
    eu, ev = ot.eu.copy(), ot.ev.copy()
    a = min(x for x in ot.neighbors(u) if x != v)
    out = []
    for b in sorted(y for y in ot.neighbors(v) if y != u):
        ot.doNNI(u, v, a, b)
        lens = [0.0] * 5
        i = 1
        for x in sorted(x for x in ot.neighbors(u) if x != v):
            ot.optimizeOneBranch(u, x, True, max_nr)
            lens[i] = ot.getBranchLength(u, x)
            i += 1
        ot.optimizeOneBranch(u, v, True, max_nr)
        lens[0] = ot.getBranchLength(u, v)
        for y in sorted(y for y in ot.neighbors(v) if y != u):
            ot.optimizeOneBranch(v, y, True, max_nr)
            lens[i] = ot.getBranchLength(v, y)
            i += 1
        out.append((a, b, ot.computeLikelihoodFromBuffer(), np.array(lens)))
        ot.doNNI(u, v, b, a)
    np.testing.assert_array_equal(ot.eu, eu)
    for (x, y), ln in zip(zip(ot.eu.tolist(), ot.ev.tolist()), saved):
        ot.setLength(x, y, float(ln))
    return out


@pytest.mark.parametrize("slots", ["node", "node+spare", "branch", "pool"])
def test_evaluate_nni_matches_oracle_and_leaves_tree(gpu, slots):
    """gems_tree_nni_evaluate on several internal branches: both moves' lnL and five lengths as
    the oracle doing the same sequence; the tree (edges, lengths, lnL) unchanged after."""
    tree, model, aln = case(4, 20, 2500, 91)
    ot = orc.OracleTree(tree, model, aln)
    gt = PhyloTree.from_case(tree, model, aln, precision="fp64", slots=slots)
    l0 = gt.computeLikelihood()
    ot.computeLikelihood()
    internal = [(int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa][:4]
    for u, v in internal:
        got = gt.evaluateNNI(u, v)
        ref = oracle_evaluate_nni(ot, u, v)
        for (ga, gb, gl, gL), (ra, rb, rl, rL) in zip(got, ref):
            assert (ga, gb) == (ra, rb)
            assert abs(gl - rl) <= 1e-9 * abs(rl), (u, v, gl, rl)
            np.testing.assert_allclose(gL, rL, rtol=1e-7, atol=1e-10)
        np.testing.assert_array_equal(gt.eu, tree.eu)
        np.testing.assert_array_equal(gt.getBranchLengths(), tree.length)
        assert gt.computeLikelihood() == l0
    gt.close()
    gt.session.close()


def test_evaluate_nni_with_spare_slots_keeps_the_partials(gpu):
    """With two spare slots the evaluation computes in them: the tree's partials stay valid, so
    the next lnL at the same branch recomputes nothing; without spares the central partials
    are recomputed."""
    tree, model, aln = case(4, 24, 2000, 93)
    u, v = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa)
    res = {}
    for slots in ("node+spare", "node"):
        gt = PhyloTree.from_case(tree, model, aln, precision="fp64", slots=slots)
        l0 = gt.computeLikelihoodBranch(u, v)
        gt.evaluateNNI(u, v)
        before = gt.stats()[0]
        assert gt.computeLikelihoodBranch(u, v) == l0
        res[slots] = gt.stats()[0] - before
        gt.close()
        gt.session.close()
    assert res["node+spare"] == 0
    assert res["node"] > 0


def test_evaluate_nni_mixed(gpu):
    tree, model, aln = case(20, 16, 1500, 95)
    ot = orc.OracleTree(tree, model, aln)
    gt = PhyloTree.from_case(tree, model, aln, precision="mixed", slots="node+spare")
    gt.computeLikelihood()
    ot.computeLikelihood()
    u, v = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa)
    for (ga, gb, gl, gL), (ra, rb, rl, rL) in zip(gt.evaluateNNI(u, v),
                                                  oracle_evaluate_nni(ot, u, v)):
        assert (ga, gb) == (ra, rb)
        assert abs(gl - rl) <= 1e-6 * abs(rl)
        np.testing.assert_allclose(gL, rL, rtol=2e-4, atol=1e-7)
    gt.close()
    gt.session.close()
