"""ModelFinder's candidate models on one alignment and tree, batched: 16 candidates' rate
matrices decomposed in one launch (gems_set_model_from_rates_batch) and their branch lengths
optimised together (gems_tree_optimize_all_branches_batch).  Each candidate must end exactly
where its own optimizeAllBranches ends (lnL and lengths, bit for bit); on the oracle's
eigensystems the batch ends within the FP64 bar of the oracle's optimizeAllBranches."""
import numpy as np
import pytest

from gems_b200 import PhyloTree, Session, optimize_all_branches_batch, set_models_from_rates, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def candidates(n, k, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        alpha = float(rng.uniform(0.3, 1.5))
        if n == 4:
            m = synth.dna_gtr(rng, 4, alpha)
        elif n == 20:
            m = synth.protein(rng, 4, alpha)
        else:
            m = synth.codon_gy(rng, 4, alpha)
        out.append(m)
    return out


def open_sessions(tree, aln, models, precision, scaling):
    ss = []
    for m in models:
        s = Session(tree.ntaxa, aln.npat, m.nstates, m.ncat, tree.ntaxa - 2, precision, scaling)
        s.upload_tips(aln.patterns)
        s.upload_patterns(aln.weights)
        ss.append(s)
    set_models_from_rates(ss, [m.exch_upper for m in models], [m.freq for m in models],
                          [m.rates for m in models], [m.props for m in models])
    return ss


@pytest.mark.parametrize("n,k,precision,scaling", [(4, 16, "fp64", "norm"),
                                                   (20, 8, "fp64", "norm"),
                                                   (61, 6, "fp64", "safe"),
                                                   (4, 16, "mixed", "norm")])
def test_batched_candidates_match_one_by_one_and_oracle(gpu, n, k, precision, scaling):
    truth = candidates(n, 1, 71 + n)[0]
    tree = synth.random_tree(16, 0.12, 72 + n)
    aln = synth.simulate(tree, truth, {4: 3000, 20: 1500, 61: 600}[n], 73 + n)
    models = candidates(n, k, 74 + n)
    # batched: one eigendecomposition launch, the optimisations overlapped
    ss = open_sessions(tree, aln, models, precision, scaling)
    trees = [PhyloTree(s, tree.eu, tree.ev, tree.length) for s in ss]
    lnl_b = optimize_all_branches_batch(trees, 100, 0.001, 100)
    # one by one, each on its own session with its own decomposition call
    for i, m in enumerate(models):
        s = Session(tree.ntaxa, aln.npat, n, m.ncat, tree.ntaxa - 2, precision, scaling)
        s.upload_tips(aln.patterns)
        s.upload_patterns(aln.weights)
        s.set_model_from_rates(m.exch_upper, m.freq, m.rates, m.props)
        one = PhyloTree(s, tree.eu, tree.ev, tree.length)
        lnl_1 = one.optimizeAllBranches(100, 0.001, 100)
        assert lnl_b[i] == lnl_1, (i, lnl_b[i], lnl_1)
        np.testing.assert_array_equal(trees[i].getBranchLengths(), one.getBranchLengths())
        one.close()
        s.close()
    for t, s in zip(trees, ss):
        t.close()
        s.close()


@pytest.mark.parametrize("n,k", [(4, 16), (20, 6)])
def test_batched_optimisation_matches_oracle(gpu, n, k):
    """Candidates on the oracle's own eigensystems: every batched optimisation ends within the
    FP64 bar of the oracle's optimizeAllBranches."""
    truth = candidates(n, 1, 81 + n)[0]
    tree = synth.random_tree(14, 0.1, 82 + n)
    aln = synth.simulate(tree, truth, 2000 if n == 4 else 1000, 83 + n)
    models = []
    for m in candidates(n, k, 84 + n):
        ev, v, iv = orc.eigensystem(m.exch_upper, m.freq)
        models.append(synth.Model(n, m.exch_upper, m.freq, m.rates, m.props, ev, v, iv))
    trees = [PhyloTree.from_case(tree, m, aln) for m in models]
    lnl_b = optimize_all_branches_batch(trees, 100, 0.001, 100)
    for i, m in enumerate(models):
        ot = orc.OracleTree(tree, m, aln)
        lo = ot.optimizeAllBranches(100, 0.001, 100)
        assert abs(lnl_b[i] - lo) <= 1e-9 * abs(lo)
        np.testing.assert_allclose(trees[i].getBranchLengths(), ot.getBranchLengths(),
                                   rtol=1e-7, atol=1e-9)
    for t in trees:
        t.close()
        t.session.close()


@pytest.mark.parametrize("n,k,precision,scaling", [(4, 12, "fp64", "norm"),
                                                   (4, 12, "mixed", "norm"),
                                                   (20, 6, "mixed", "norm"),
                                                   (61, 8, "mixed", "safe"),
                                                   (61, 4, "fp64", "safe")])
def test_gamma_shapes_batched_match_one_by_one_and_oracle(gpu, n, k, precision, scaling):
    """Every candidate re-evaluated at a new Gamma shape in one batched call (new rates, all
    partials cleared, lnL): equal bit for bit to each candidate's own computeLikelihood after
    the same change, and to the oracle at the form's bar.  The candidates' trees carry
    different branch lengths (each was optimised on its own), so every session evaluates its
    own op list."""
    from gems_b200 import evaluate_rates_batch
    truth = candidates(n, 1, 91 + n)[0]
    tree = synth.random_tree(14, 0.1, 92 + n)
    aln = synth.simulate(tree, truth, {4: 2000, 20: 1000, 61: 500}[n], 93 + n)
    models = candidates(n, k, 94 + n)
    rng = np.random.default_rng(95 + n)
    trees = [PhyloTree.from_case(tree, m, aln, precision=precision, scaling=scaling)
             for m in models]
    for t in trees:  # each candidate with its own lengths
        for e in rng.choice(tree.nedges, 3, replace=False):
            t.setLength(int(tree.eu[e]), int(tree.ev[e]), float(rng.uniform(0.01, 0.3)))
        t.computeLikelihood()
    alphas = rng.uniform(0.2, 2.0, k)
    rates = [synth.gamma_rates(a, models[i].ncat) for i, a in enumerate(alphas)]
    lnl_b = evaluate_rates_batch(trees, rates)
    bar = 1e-9 if precision == "fp64" else 1e-6
    for i, m in enumerate(models):
        one = PhyloTree.from_case(tree, m, aln, precision=precision, scaling=scaling)
        for (u, v), x in zip(zip(tree.eu, tree.ev), trees[i].getBranchLengths()):
            one.setLength(int(u), int(v), float(x))
        one.session.set_rates(rates[i], np.full(m.ncat, 1.0 / m.ncat))
        one.clearAllPartialLH()
        assert one.computeLikelihood() == lnl_b[i]
        one.close()
        one.session.close()
        mm = synth.Model(n, m.exch_upper, m.freq, rates[i], m.props, m.eval, m.evec, m.inv_evec)
        ot = orc.OracleTree(synth.Tree(tree.ntaxa, tree.eu, tree.ev, trees[i].getBranchLengths()),
                            mm, aln, safe=scaling == "safe")
        lo = ot.computeLikelihood()
        assert abs(lnl_b[i] - lo) <= bar * abs(lo), (i, lnl_b[i], lo)
    for t in trees:
        t.close()
        t.session.close()


def test_rate_and_batch_error_paths(gpu):
    """gems_set_rates before any model is a state error; a negative rate is refused; a batch of
    sessions of different shapes is refused before anything runs."""
    from gems_b200 import GemsError, compute_likelihood_batch
    m4 = candidates(4, 1, 5)[0]
    tree = synth.random_tree(10, 0.1, 6)
    aln = synth.simulate(tree, m4, 300, 7)
    s = Session(tree.ntaxa, aln.npat, 4, m4.ncat, tree.ntaxa - 2, "fp64", "norm")
    with pytest.raises(GemsError) as e:
        s.set_rates(m4.rates, m4.props)
    assert e.value.status == 7  # GEMS_ERR_STATE
    s.close()
    a = PhyloTree.from_case(tree, m4, aln)
    with pytest.raises(GemsError) as e:
        a.session.set_rates(-m4.rates, m4.props)
    assert e.value.status == 5  # GEMS_ERR_BAD_ARG
    m20 = candidates(20, 1, 8)[0]
    aln20 = synth.simulate(tree, m20, 300, 9)
    b = PhyloTree.from_case(tree, m20, aln20)
    with pytest.raises(GemsError) as e:
        compute_likelihood_batch([a, b])
    assert e.value.status == 5
    # the refused batch left no partial marked computed that was not: each tree still gives
    # its own lnL
    la = compute_likelihood_batch([a])[0]
    a.clearAllPartialLH()
    assert a.computeLikelihood() == la
    for t in (a, b):
        t.close()
        t.session.close()
