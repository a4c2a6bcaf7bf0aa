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
