"""LM_MEM_SAVE: a tree run in fewer partial slots than internal nodes (down to log2(ntaxa) + 1,
tree/phylotree.cpp:1026-1040, tree/memslot.cpp:28-229) gives the same lnL, pattern lnL,
derivatives on every branch, optimised branch lengths and NNI results, bit for bit, as one slot
per internal node and one per directed branch; it recomputes more partials to get there."""
import numpy as np
import pytest

from gems_b200 import GemsError, PhyloTree, Session, synth
from gems_b200.api import min_pool_slots
from gems_b200.serve import nni5

pytestmark = pytest.mark.gpu


def case(n, ntaxa, nsites, seed):
    rng = np.random.default_rng(seed)
    model = synth.dna_gtr(rng, 4, 0.5) if n == 4 else synth.protein(rng, 4, 0.8)
    tree = synth.random_tree(ntaxa, 0.1, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2, gap_frac=0.02)
    return tree, model, aln


def run(tree, model, aln, slots, precision, scaling):
    gt = PhyloTree.from_case(tree, model, aln, precision=precision, scaling=scaling,
                             slots=slots)
    out = {}
    out["lnl"], out["plh"] = gt.computeLikelihood(pattern_lh=True)
    derv = []
    for e in range(tree.nedges):
        u, v = int(tree.eu[e]), int(tree.ev[e])
        derv.append(gt.computeFuncDerv(u, v, float(tree.length[e]), new_branch=True))
    out["derv"] = np.array(derv)
    out["opt_lnl"] = gt.optimizeAllBranches(3, 0.001, 100)
    out["opt_len"] = gt.getBranchLengths()
    nni = []
    for k in range(4):
        lg, _ = nni5(gt, tree.ntaxa, np.random.default_rng((5, k)))
        nni.append(lg)
    out["nni"] = np.array(nni)
    out["ops"] = gt.stats()[0]
    gt.close()
    gt.session.close()
    return out


@pytest.mark.parametrize("n,precision,scaling", [(4, "fp64", "norm"), (4, "mixed", "safe"),
                                                 (20, "fp64", "safe"), (20, "mixed", "norm")])
def test_memory_modes_give_the_same_results(gpu, n, precision, scaling):
    tree, model, aln = case(n, 48, 2000, 60 + n)
    ref = run(tree, model, aln, "node", precision, scaling)
    for slots in ("branch", "pool", min_pool_slots(tree.ntaxa) + 4):
        got = run(tree, model, aln, slots, precision, scaling)
        assert got["lnl"] == ref["lnl"], slots
        np.testing.assert_array_equal(got["plh"], ref["plh"])
        np.testing.assert_array_equal(got["derv"], ref["derv"])
        assert got["opt_lnl"] == ref["opt_lnl"]
        np.testing.assert_array_equal(got["opt_len"], ref["opt_len"])
        np.testing.assert_array_equal(got["nni"], ref["nni"])
        if slots == "pool":
            assert got["ops"] > ref["ops"]  # evicted partials are recomputed


def test_too_few_slots_refused(gpu):
    tree, model, aln = case(4, 64, 500, 3)
    s = Session(tree.ntaxa, aln.npat, 4, 4, min_pool_slots(tree.ntaxa) - 1)
    s.upload_tips(aln.patterns)
    s.upload_patterns(aln.weights)
    s.set_model(model.eval, model.evec, model.inv_evec, model.rates, model.props)
    with pytest.raises(GemsError) as e:
        PhyloTree(s, tree.eu, tree.ev, tree.length)
    assert e.value.status == 2
    s.close()
