"""61-state (codon) mixed-precision form on the tensor cores: the tcgen05 kernel against the FP32
CUDA-core kernel and the FP64 oracle (SAFE scaling, +G4 / +R8 / one category, gaps, pattern
counts that are not a multiple of the 128-row tile), and the batched launch of many candidate
models on one alignment against each model evaluated alone."""
import numpy as np
import pytest

from gems_b200 import PhyloTree, Session, branch_lnl_batch, full_traversal, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
MIXED_RTOL = 1e-6


def codon_case(ncat, seed, ntaxa=30, nsites=700, gap=0.05):
    rng = np.random.default_rng(seed)
    model = synth.codon_gy(rng, ncat, 0.5, freerate=ncat == 8)
    tree = synth.random_tree(ntaxa, 0.1, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2, gap_frac=gap)
    return tree, model, aln


@pytest.mark.parametrize("ncat", [1, 4, 8])
def test_tc61_matches_cuda_cores_and_oracle(gpu, ncat):
    tree, model, aln = codon_case(ncat, 60 + ncat)
    assert aln.npat % 128 != 0
    ot = orc.OracleTree(tree, model, aln, safe=True)
    lo = ot.computeLikelihood()
    res = []
    for tc in (True, False):
        gt = PhyloTree.from_case(tree, model, aln, precision="mixed", scaling="safe")
        gt.session.set_tensor_cores(tc)
        lg, plg = gt.computeLikelihood(pattern_lh=True)
        assert abs(lg - lo) <= MIXED_RTOL * abs(lo), (tc, lg, lo)
        # every branch, from buffers the tensor-core traversal wrote
        for e in (0, len(tree.eu) // 2, len(tree.eu) - 1):
            u, v = int(tree.eu[e]), int(tree.ev[e])
            assert abs(gt.computeLikelihoodBranch(v, u) - lo) <= MIXED_RTOL * abs(lo)
        res.append(plg)
        gt.close()
        gt.session.close()
    assert np.max(np.abs(res[0] - res[1]) / (np.abs(res[1]) + 1)) < 1e-5


def test_tc61_deep_tree_scaling(gpu):
    """A deep tree forces the per-category 2^64 rescaling on many patterns."""
    rng = np.random.default_rng(71)
    model = synth.codon_gy(rng, 4, 0.5)
    tree = synth.random_tree(120, 0.3, 72)
    aln = synth.simulate(tree, model, 400, 73)
    ot = orc.OracleTree(tree, model, aln, safe=True)
    lo = ot.computeLikelihood()
    gt = PhyloTree.from_case(tree, model, aln, precision="mixed", scaling="safe")
    lg = gt.computeLikelihood()
    assert abs(lg - lo) <= MIXED_RTOL * abs(lo), (lg, lo)


def test_batched_models_match_each_alone(gpu):
    """Candidate codon models (different kappa/omega and rates) on one alignment and tree in
    one batched launch: every lnL equals the oracle's for that model, and the same session
    evaluated alone."""
    tree, model0, aln = codon_case(4, 81, ntaxa=40, nsites=900)
    rng = np.random.default_rng(82)
    models = [model0] + [synth.codon_gy(rng, 4, float(rng.uniform(0.3, 1.5))) for _ in range(5)]
    sessions = []
    for m in models:
        s = Session(tree.ntaxa, aln.npat, 61, 4, tree.ntaxa - 2, "mixed", "safe")
        s.upload_tips(aln.patterns)
        s.upload_patterns(aln.weights)
        s.set_model(m.eval, m.evec, m.inv_evec, m.rates, m.props)
        sessions.append(s)
    ops, br = full_traversal(tree)
    got = branch_lnl_batch(sessions, ops, br)
    for m, s, g in zip(models, sessions, got):
        lo = orc.OracleTree(tree, m, aln, safe=True).computeLikelihood()
        assert abs(g - lo) <= MIXED_RTOL * abs(lo), (g, lo)
        alone = s.branch_lnl(ops, br)
        assert abs(alone - g) <= 1e-12 * abs(g)
    for s in sessions:
        s.close()
