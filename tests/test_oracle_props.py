"""Size-independent properties of the oracle itself (it is the checker, so it is checked):
derivatives against finite differences, NORM vs SAFE, invariance to the evaluation branch,
Newton returning a stationary point."""
import numpy as np
import pytest

from gems_b200 import synth
from oracle import oracle as orc


def small_case(n=4, ntaxa=10, nsites=600, seed=3):
    rng = np.random.default_rng(seed)
    model = synth.dna_gtr(rng) if n == 4 else synth.protein(rng)
    tree = synth.random_tree(ntaxa, 0.12, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2)
    return tree, model, aln


@pytest.mark.parametrize("n", [4, 20])
def test_lnl_same_on_every_branch(n):
    tree, model, aln = small_case(n)
    ot = orc.OracleTree(tree, model, aln)
    vals = [ot.computeLikelihoodBranch(int(u), int(v)) for u, v in zip(tree.eu, tree.ev)]
    assert np.ptp(vals) < 1e-9 * abs(vals[0])


@pytest.mark.parametrize("n", [4, 20])
def test_derivatives_match_finite_differences(n):
    tree, model, aln = small_case(n)
    ot = orc.OracleTree(tree, model, aln)
    for e in (0, 3, len(tree.eu) - 1):
        u, v = int(tree.eu[e]), int(tree.ev[e])
        t0 = float(tree.length[e])
        h = 1e-5
        f = []
        for t in (t0 - h, t0, t0 + h):
            ot.setLength(u, v, t)
            f.append(ot.computeLikelihoodBranch(v, u))
        ot.setLength(u, v, t0)
        ot.clearAllPartialLH()
        df, ddf = ot.computeLikelihoodDerv(v, u)
        assert abs(df - (f[2] - f[0]) / (2 * h)) < 1e-4 * max(1, abs(df))
        assert abs(ddf - (f[2] - 2 * f[1] + f[0]) / h ** 2) < 1e-2 * max(1, abs(ddf))


def test_norm_and_safe_agree():
    tree, model, aln = small_case(4, ntaxa=120, nsites=300, seed=9)
    a = orc.OracleTree(tree, model, aln, safe=False).computeLikelihood()
    b = orc.OracleTree(tree, model, aln, safe=True).computeLikelihood()
    assert abs(a - b) < 1e-9 * abs(a)


def test_newton_reaches_stationary_point():
    tree, model, aln = small_case(4)
    ot = orc.OracleTree(tree, model, aln)
    u, v = int(tree.eu[2]), int(tree.ev[2])
    ot.optimizeOneBranch(u, v)
    ot.clearAllPartialLH()
    df, ddf = ot.computeLikelihoodDerv(v, u)
    assert abs(df) < 1e-3 and ddf < 0


@pytest.mark.parametrize("n", [4, 20])
def test_nni_incremental_equals_fresh_tree(n):
    """doNNI + NNI-5 branch optimisation keeps the partial buffers consistent: the lnL read
    from the buffers equals a from-scratch lnL of a new tree with the resulting topology."""
    from gems_b200.serve import nni5
    tree, model, aln = small_case(n, ntaxa=12)
    ot = orc.OracleTree(tree, model, aln)
    ot.computeLikelihood()
    for k in range(4):
        lnl, nbr = nni5(ot, tree.ntaxa, np.random.default_rng((7, k)))
        assert nbr == 5
        fresh = orc.OracleTree(synth.Tree(tree.ntaxa, ot.eu.copy(), ot.ev.copy(),
                                          ot.getBranchLengths()), model, aln)
        ref = fresh.computeLikelihood()
        assert abs(lnl - ref) <= 1e-9 * abs(ref), (k, lnl, ref)


def test_nni_changes_topology_and_back():
    """The same NNI applied twice restores the split set (doNNI is an involution up to the
    edge labels it rewrites)."""
    tree, model, aln = small_case(4, ntaxa=10)
    ot = orc.OracleTree(tree, model, aln)
    l0 = ot.computeLikelihood()
    u, v = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa)
    a = [x for x in ot.neighbors(u) if x != v][0]
    b = [x for x in ot.neighbors(v) if x != u][0]
    ot.doNNI(u, v, a, b)
    assert a in ot.neighbors(v) and b in ot.neighbors(u)
    l1 = ot.computeLikelihood()
    assert abs(l1 - l0) > 1e-6
    ot.doNNI(u, v, b, a)
    assert a in ot.neighbors(u) and b in ot.neighbors(v)
    l2 = ot.computeLikelihood()
    assert abs(l2 - l0) <= 1e-9 * abs(l0)


def _fresh_lnl(ot, tree, model, aln):
    fresh = orc.OracleTree(synth.Tree(tree.ntaxa, ot.eu.copy(), ot.ev.copy(),
                                      ot.getBranchLengths()), model, aln)
    return fresh.computeLikelihood()


@pytest.mark.parametrize("n", [4, 20])
def test_spr_incremental_equals_fresh_tree(n):
    """doSPR + the four-branch optimisation keeps the partial buffers consistent: the lnL read
    from the buffers equals a from-scratch lnL of a new tree with the resulting topology."""
    from gems_b200.serve import spr4
    tree, model, aln = small_case(n, ntaxa=14)
    ot = orc.OracleTree(tree, model, aln)
    ot.computeLikelihood()
    for k in range(6):
        lnl, nbr = spr4(ot, tree.ntaxa, np.random.default_rng((9, k)))
        assert nbr == 4
        ref = _fresh_lnl(ot, tree, model, aln)
        assert abs(lnl - ref) <= 1e-9 * abs(ref), (k, lnl, ref)


def test_spr_every_regraft_of_one_prune():
    """Every regraft branch within the radius of one pruned subtree, the moves next to the
    joint (dad2 or node2 a former neighbour of dad) included: after each move the lnL computed
    on the moved tree's buffers equals a fresh tree's, the edge list holds a binary tree with
    the same leaves, and the joined branch has the summed length."""
    from gems_b200.serve import spr_regraft_branches
    tree, model, aln = small_case(4, ntaxa=12)
    base = orc.OracleTree(tree, model, aln)
    u, v = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa)
    node, dad = u, v
    s1, s2, cand = spr_regraft_branches(base, node, dad, radius=10)
    assert any(s1 in c or s2 in c for c in cand)
    for node2, dad2 in cand:
        ot = orc.OracleTree(tree, model, aln)
        ot.computeLikelihood()
        l1 = ot.getBranchLength(dad, s1)
        l2 = ot.getBranchLength(dad, s2)
        l = ot.getBranchLength(node2, dad2)
        ot.doSPR(node, dad, node2, dad2)
        assert sorted(ot.neighbors(dad)) == sorted([node, node2, dad2])
        assert s2 in ot.neighbors(s1)
        assert ot.getBranchLength(s1, s2) == l1 + l2
        assert ot.getBranchLength(dad, node2) == l / 2 == ot.getBranchLength(dad, dad2)
        deg = np.bincount(np.concatenate([ot.eu, ot.ev]))
        assert np.all(deg[: tree.ntaxa] == 1) and np.all(deg[tree.ntaxa:] == 3)
        got = ot.computeLikelihood()
        ref = _fresh_lnl(ot, tree, model, aln)
        assert abs(got - ref) <= 1e-10 * abs(ref), (node2, dad2, got, ref)


def test_spr_refuses_bad_moves():
    tree, model, aln = small_case(4, ntaxa=10)
    ot = orc.OracleTree(tree, model, aln)
    u, v = next((int(a), int(b)) for a, b in zip(tree.eu, tree.ev)
                if a >= tree.ntaxa and b >= tree.ntaxa)
    inside = [x for x in ot.neighbors(u) if x != v][0]   # a branch inside the pruned subtree
    with pytest.raises(AssertionError):
        ot.doSPR(u, v, inside, u)
    with pytest.raises(AssertionError):                  # a branch at dad itself
        ot.doSPR(u, v, [x for x in ot.neighbors(v) if x != u][0], v)
    leaf = next(x for x in range(tree.ntaxa))
    with pytest.raises(AssertionError):                  # dad must be internal
        ot.doSPR(ot.neighbors(leaf)[0], leaf, u, v)
