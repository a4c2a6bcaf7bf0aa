"""Parity at the shape of the scale configuration: 512 taxa, the generator of the FP64-vs-mixed
DNA workload (GTR+G4, lengths ~Exp(0.05), 5% gap cells) at 20,000 sites.

Every branch of the tree: first and second derivatives (computeFuncDerv with a new branch, as
optimizeOneBranch starts) and the lnL at that branch, FP64 plain form against the oracle at
the FP64 bar, mixed form against the oracle at the mixed bars (lnL 1e-6 relative; a derivative
error of at most 1e-6 of |ddf|, i.e. a Newton step moved by at most 1e-6 in branch-length
units)."""
import numpy as np
import pytest

from gems_b200 import PhyloTree, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case512():
    tree, model, aln = synth.config_dna512(seed=2, nsites=20_000, gap_frac=0.05)
    ot = orc.OracleTree(tree, model, aln, const_char=aln.const_char())
    ref = []
    for e in range(tree.nedges):
        u, v = int(tree.eu[e]), int(tree.ev[e])
        f, df = ot.computeFuncDerv(u, v, float(tree.length[e]), new_branch=True)
        ref.append((-f, -df, ot.computeLikelihoodFromBuffer()))
    return tree, model, aln, np.array(ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_branch_derivatives_512_taxa(gpu, case512, precision):
    tree, model, aln, ref = case512
    gt = PhyloTree.from_case(tree, model, aln, precision=precision)
    got = []
    for e in range(tree.nedges):
        u, v = int(tree.eu[e]), int(tree.ev[e])
        f, df = gt.computeFuncDerv(u, v, float(tree.length[e]), new_branch=True)
        got.append((-f, -df, gt.computeLikelihoodFromBuffer()))
    got = np.array(got)
    d1, d2, lnl = got.T
    r1, r2, rl = ref.T
    assert np.all(np.abs(lnl - rl) <= (1e-9 if precision == "fp64" else 1e-6) * np.abs(rl))
    if precision == "fp64":
        assert np.all(np.abs(d1 - r1) <= 1e-9 * np.maximum(1.0, np.abs(r1)))
        assert np.all(np.abs(d2 - r2) <= 1e-9 * np.maximum(1.0, np.abs(r2)))
    else:
        assert np.all(np.abs(d1 - r1) <= 1e-6 * np.abs(r2))
        assert np.all(np.abs(d2 - r2) <= 1e-6 * np.abs(r2))
