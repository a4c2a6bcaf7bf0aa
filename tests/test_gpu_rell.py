"""Bootstrap reweighting (UFBoot RELL) on device against the same sums formed from the FP64
oracle's per-pattern terms."""
import numpy as np
import pytest

from gems_b200 import PhyloTree, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def multinomial_weights(aln, R, seed):
    """R bootstrap replicates of the sites, as pattern counts (the reference draws sites with
    replacement and counts them per pattern)."""
    rng = np.random.default_rng(seed)
    nsites = int(aln.weights.sum())
    return rng.multinomial(nsites, aln.weights / nsites, size=R).astype(np.float32)


def test_reweighted_lnl_and_derivatives(gpu):
    tree, model, aln = synth.config_dna16(seed=8, nsites=5000)
    ot = orc.OracleTree(tree, model, aln)
    gt = PhyloTree.from_case(tree, model, aln)
    s = gt.session
    w = multinomial_weights(aln, 256, 3)
    s.upload_reweightings(w)
    lo, plo = ot.computeLikelihood(pattern_lh=True)
    gt.computeLikelihood()
    r = s.reweighted_lnl()
    ref64 = w.astype(np.float64) @ plo.astype(np.float32).astype(np.float64)
    assert np.allclose(r, ref64, rtol=1e-9, atol=0)
    # the reference's float dot product agrees to float precision
    ref32 = np.array([np.dot(wr, plo.astype(np.float32)) for wr in w], dtype=np.float64)
    assert np.allclose(r, ref32, rtol=2e-5)
    # the replicate with the original weights reproduces the tree lnL
    s.upload_reweightings(aln.weights[None, :].astype(np.float32))
    assert abs(s.reweighted_lnl()[0] - lo) < 1e-3  # pattern lnL taken in FP32 as in UFBoot
    # derivatives: the original weights give back df, ddf of the branch
    u, v = int(tree.eu[3]), int(tree.ev[3])
    ot.clearAllPartialLH()
    gt.clearAllPartialLH()
    dfo, ddfo = ot.computeLikelihoodDerv(v, u)
    gt.computeLikelihoodDerv(v, u)
    df, ddf = s.reweighted_derv()
    assert abs(df[0] - dfo) <= 1e-9 * max(1, abs(dfo))
    assert abs(ddf[0] - ddfo) <= 1e-9 * max(1, abs(ddfo))
    s.upload_reweightings(w)
    df, ddf = s.reweighted_derv()
    g = ot.dfFrac()
    assert np.allclose(df, w.astype(np.float64) @ g, rtol=1e-9, atol=1e-9)
