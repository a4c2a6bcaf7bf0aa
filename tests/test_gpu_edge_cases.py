"""Edge cases of the likelihood path against the FP64 oracle, for 4, 20 and 61 states, FP64 and
mixed: the smallest trees (3 and 4 taxa, one internal node or two), one or two patterns (a
block of idle lanes, P padded to 64), zero and very long branches, taxa that are all gaps and
columns of unknown states; and the sizes the session refuses (no patterns, fewer than 3 taxa)
return an error instead of running."""
import numpy as np
import pytest

from gems_b200 import GemsError, PhyloTree, Session, synth
from gems_b200.synth import state_unknown
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def model_of(n, rng):
    return {4: lambda: synth.dna_gtr(rng, 4, 0.5), 20: lambda: synth.protein(rng, 4, 0.8),
            61: lambda: synth.codon_gy(rng, 4, 0.5)}[n]()


def agree(tree, model, aln, precision):
    safe = model.nstates == 61
    lo, plo = orc.OracleTree(tree, model, aln, safe=safe).computeLikelihood(pattern_lh=True)
    gt = PhyloTree.from_case(tree, model, aln, precision=precision,
                             scaling="safe" if safe else "norm")
    lg, plg = gt.computeLikelihood(pattern_lh=True)
    tol = 1e-9 if precision == "fp64" else 1e-6
    assert abs(lg - lo) <= tol * max(1.0, abs(lo)), (lg, lo)
    if precision == "fp64":
        assert np.allclose(plg, plo, rtol=tol, atol=tol)
    else:  # the mixed form's pattern-level bar (FP32 sums of 61-state rows)
        assert np.max(np.abs(plg - plo) / (np.abs(plo) + 1.0)) < 1e-5
    # derivatives on every branch of the small tree
    ot = orc.OracleTree(tree, model, aln, safe=safe)
    ot.computeLikelihood()
    for u, v in zip(tree.eu, tree.ev):
        dfo, ddfo = ot.computeLikelihoodDerv(int(u), int(v))
        dfg, ddfg = gt.computeLikelihoodDerv(int(u), int(v))
        if precision == "fp64":
            assert abs(dfg - dfo) <= 1e-9 * max(1.0, abs(dfo), abs(lo)), (dfg, dfo)
            assert abs(ddfg - ddfo) <= 1e-9 * max(1.0, abs(ddfo), abs(lo)), (ddfg, ddfo)
        else:  # the bar of the mixed form's other derivative tests
            assert abs(dfg - dfo) <= 1e-5 * max(1.0, abs(dfo)) + 1e-6 * abs(lo), (dfg, dfo)
            assert abs(ddfg - ddfo) <= 1e-5 * max(1.0, abs(ddfo)) + 1e-6 * abs(lo), (ddfg, ddfo)
    gt.close()
    gt.session.close()


@pytest.mark.parametrize("n", [4, 20, 61])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("ntaxa,nsites", [(3, 1), (3, 5), (4, 1), (4, 2), (5, 40)])
def test_smallest_trees_and_pattern_counts(gpu, n, precision, ntaxa, nsites):
    rng = np.random.default_rng(ntaxa * 100 + nsites + n)
    model = model_of(n, rng)
    tree = synth.random_tree(ntaxa, 0.1, ntaxa + nsites)
    aln = synth.simulate(tree, model, nsites, n + nsites)
    agree(tree, model, aln, precision)


@pytest.mark.parametrize("n", [4, 20, 61])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zero_and_long_branches_gaps_and_unknown_columns(gpu, n, precision):
    rng = np.random.default_rng(500 + n)
    model = model_of(n, rng)
    tree = synth.random_tree(12, 0.1, 501)
    length = np.array(tree.length, dtype=np.float64)
    length[0] = 0.0
    length[3] = 0.0
    length[5] = 10.0
    tree.length = length
    aln = synth.simulate(tree, model, 400, 502)
    pat = aln.patterns.copy()
    unk = state_unknown(n)
    pat[2, :] = unk            # a taxon of gaps only
    pat[:, 0] = unk            # a column of unknown states
    aln = synth.Alignment(aln.ntaxa, n, aln.nsites, pat, aln.weights)
    agree(tree, model, aln, precision)


def test_refused_sizes(gpu):
    with pytest.raises(GemsError) as e:
        Session(8, 0, 4, 4, 6)
    assert e.value.status == 5
    with pytest.raises(GemsError) as e:
        Session(2, 10, 4, 4, 1)
    assert e.value.status == 5
