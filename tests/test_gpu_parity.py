"""Parity of the CUDA path (through the C-ABI) with the FP64 oracle.

Bar (FP64 plain form): |dlnL| <= 1e-9 |lnL|, per-pattern lnL and partials to 1e-9 relative,
scale counters bit-exact (eigensystem injected from the oracle), derivatives to 1e-9,
Newton iterates and optimised lengths identical to 1e-9."""
import os

import numpy as np
import pytest

from conftest import golden_files, golden_opt_files, load_golden, ptn_invar
from gems_b200 import GemsError, PhyloTree, Session, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CASES = golden_files()
IDS = [os.path.basename(p)[:-4] for p in CASES]
RTOL = 1e-9


def gpu_tree(tree, model, aln, safe=False, slots="node", precision="fp64"):
    return PhyloTree.from_case(tree, model, aln, precision=precision,
                               scaling="safe" if safe else "norm", slots=slots,
                               invar=ptn_invar(model, aln))


def internal_branches(tree):
    out = []
    for u, v in zip(tree.eu, tree.ev):
        u, v = int(u), int(v)
        if v >= tree.ntaxa:
            out.append((v, u))
        if u >= tree.ntaxa:
            out.append((u, v))
    return out


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_lnl_partials_scale_counts(gpu, path):
    tree, model, aln, z = load_golden(path)
    safe = bool(z["safe"])
    ot = orc.OracleTree(tree, model, aln, safe=safe, const_char=z["const_char"])
    gt = gpu_tree(tree, model, aln, safe)
    lo, plo = ot.computeLikelihood(pattern_lh=True)
    lg, plg = gt.computeLikelihood(pattern_lh=True)
    assert abs(lg - lo) <= RTOL * abs(lo), (lg, lo)
    assert np.allclose(plg, plo, rtol=RTOL, atol=1e-12)
    # every partial the traversal produced: values and scale counters
    checked = 0
    for node, dad in internal_branches(tree):
        try:
            po, so = ot.getPartial(node, dad)
        except AssertionError:
            continue
        try:
            pg, sg = gt.getPartial(node, dad)
        except GemsError:
            continue
        np.testing.assert_array_equal(sg, so)
        scale = np.abs(po).max(axis=(1, 2), keepdims=True) + 1e-300
        assert np.max(np.abs(pg - po) / scale) < 1e-10
        checked += 1
    assert checked >= tree.ntaxa - 2


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_lnl_on_every_branch_and_derivatives(gpu, path):
    tree, model, aln, z = load_golden(path)
    safe = bool(z["safe"])
    ot = orc.OracleTree(tree, model, aln, safe=safe, const_char=z["const_char"])
    gt = gpu_tree(tree, model, aln, safe)
    for e in range(0, tree.nedges, max(1, tree.nedges // 12)):
        u, v = int(tree.eu[e]), int(tree.ev[e])
        lo = ot.computeLikelihoodBranch(v, u)
        lg = gt.computeLikelihoodBranch(v, u)
        assert abs(lg - lo) <= RTOL * abs(lo)
        ot.clearAllPartialLH()
        gt.clearAllPartialLH()
        dfo, ddfo = ot.computeLikelihoodDerv(v, u)
        dfg, ddfg = gt.computeLikelihoodDerv(v, u)
        assert abs(dfg - dfo) <= RTOL * max(1.0, abs(dfo))
        assert abs(ddfg - ddfo) <= RTOL * max(1.0, abs(ddfo))


OPT = golden_opt_files()


@pytest.mark.parametrize("path", OPT, ids=[os.path.basename(p)[:-4] for p in OPT])
def test_optimize_all_branches(gpu, path):
    tree, model, aln, z = load_golden(path)
    safe = bool(z["safe"])
    ot = orc.OracleTree(tree, model, aln, safe=safe, const_char=z["const_char"])
    gt = gpu_tree(tree, model, aln, safe)
    lo = ot.optimizeAllBranches(100, 0.001, 100)
    lg = gt.optimizeAllBranches(100, 0.001, 100)
    assert abs(lg - lo) <= RTOL * abs(lo)
    assert np.allclose(gt.getBranchLengths(), ot.getBranchLengths(), rtol=1e-7, atol=1e-9)
    assert abs(lg - float(z["ref_lnl_opt"])) < 5e-3


def test_one_newton_step_every_branch_config1(gpu):
    """Small FP64 configuration: 16 taxa, 10,000 sites; lnL, derivatives and one
    optimizeOneBranch on every branch (iterate counts equal)."""
    tree, model, aln = synth.config_dna16(seed=1)
    ot = orc.OracleTree(tree, model, aln)
    gt = gpu_tree(tree, model, aln)
    assert abs(gt.computeLikelihood() - ot.computeLikelihood()) <= RTOL * 8e4
    for u, v in zip(tree.eu, tree.ev):
        u, v = int(u), int(v)
        ot.optimizeOneBranch(u, v)
        gt.optimizeOneBranch(u, v)
        assert gt.stats()[1] == ot.lastNewtonEvals()
    assert np.allclose(gt.getBranchLengths(), ot.getBranchLengths(), rtol=1e-9, atol=1e-12)
    lo, lg = ot.computeLikelihoodFromBuffer(), gt.computeLikelihoodFromBuffer()
    assert abs(lg - lo) <= RTOL * abs(lo)


def test_per_branch_slots_same_as_per_node(gpu):
    tree, model, aln = synth.config_dna16(seed=5, nsites=3000)
    a = gpu_tree(tree, model, aln, slots="node")
    b = gpu_tree(tree, model, aln, slots="branch")
    la = [a.computeLikelihoodBranch(int(v), int(u)) for u, v in zip(tree.eu, tree.ev)]
    lb = [b.computeLikelihoodBranch(int(v), int(u)) for u, v in zip(tree.eu, tree.ev)]
    assert np.allclose(la, lb, rtol=1e-13, atol=0)


def test_codon_small(gpu):
    tree, model, aln = synth.config_codon200(seed=4, nsites=300)
    tree = synth.random_tree(20, 0.1, 99)
    aln = synth.simulate(tree, model, 300, 98)
    ot = orc.OracleTree(tree, model, aln, safe=True)
    gt = gpu_tree(tree, model, aln, safe=True)
    lo, lg = ot.computeLikelihood(), gt.computeLikelihood()
    assert abs(lg - lo) <= RTOL * abs(lo)


def test_gpu_eigensolver(gpu):
    rng = np.random.default_rng(11)
    for model in (synth.dna_gtr(rng), synth.protein(rng), synth.codon_gy(rng)):
        n = model.nstates
        s = Session(8, 64, n, model.ncat, 6)
        s.set_model_from_rates(model.exch_upper, model.freq, model.rates, model.props)
        ev, v, iv = s.eigensystem()
        assert np.allclose(np.sort(ev), np.sort(model.eval), atol=1e-10)
        q = v @ np.diag(ev) @ iv
        q_ref = model.evec @ np.diag(model.eval) @ model.inv_evec
        assert np.allclose(q, q_ref, atol=1e-10)
        s.close()


def test_lnl_with_gpu_eigensystem(gpu):
    tree, model, aln = synth.config_dna16(seed=2, nsites=2000)
    ot = orc.OracleTree(tree, model, aln)
    s = Session(tree.ntaxa, aln.npat, 4, 4, tree.ntaxa - 2)
    s.upload_tips(aln.patterns)
    s.upload_patterns(aln.weights)
    s.set_model_from_rates(model.exch_upper, model.freq, model.rates, model.props)
    gt = PhyloTree(s, tree.eu, tree.ev, tree.length)
    lo, lg = ot.computeLikelihood(), gt.computeLikelihood()
    assert abs(lg - lo) <= RTOL * abs(lo)


def test_kernel_set_errors(gpu):
    s = Session(5, 10, 4, 4, 3)
    from gems_b200.api import branch_struct
    with pytest.raises(GemsError) as e:
        s.branch_lnl([], branch_struct(0, 0, 1, 0.1))
    assert e.value.status == 7  # model not set
    s.set_model(np.zeros(4), np.eye(4), np.eye(4), np.ones(4), np.full(4, .25))
    with pytest.raises(GemsError) as e:
        s.traverse([(0, 0, 9, 0, 1, 0.1, 0.1)])  # taxon id out of range
    assert e.value.status == 5
    with pytest.raises(GemsError) as e:
        s.lnl_from_buffer(0.1)
    assert e.value.status == 7  # theta not computed
    with pytest.raises(GemsError) as e:
        s.upload_tips(np.full((5, 10), 99, np.uint8))  # state byte out of range
    assert e.value.status == 5
    with pytest.raises(GemsError) as e:  # tips are invalid until the next good upload
        s.traverse([(0, 0, 1, 0, 2, 0.1, 0.1)])
    assert e.value.status == 7
    s.upload_tips(np.zeros((5, 10), np.uint8))
    s.traverse([(0, 0, 1, 0, 2, 0.1, 0.1)])


# ---- mixed-precision form: FP32 real-space partials, FP64 theta / reductions / Newton ----
MIXED_RTOL = 1e-6  # |dlnL| <= 1e-6 |lnL|


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_mixed_lnl_within_1e6(gpu, path):
    tree, model, aln, z = load_golden(path)
    safe = bool(z["safe"])
    ot = orc.OracleTree(tree, model, aln, safe=safe, const_char=z["const_char"])
    gt = gpu_tree(tree, model, aln, safe, precision="mixed")
    lo, plo = ot.computeLikelihood(pattern_lh=True)
    lg, plg = gt.computeLikelihood(pattern_lh=True)
    assert abs(lg - lo) <= MIXED_RTOL * abs(lo), (lg, lo)
    assert np.max(np.abs(plg - plo) / (np.abs(plo) + 1.0)) < 1e-5
    u, v = int(tree.eu[1]), int(tree.ev[1])
    ot.clearAllPartialLH()
    gt.clearAllPartialLH()
    dfo, ddfo = ot.computeLikelihoodDerv(v, u)
    dfg, ddfg = gt.computeLikelihoodDerv(v, u)
    assert abs(dfg - dfo) <= 1e-5 * max(1.0, abs(dfo)) + 1e-6 * abs(lo)
    assert abs(ddfg - ddfo) <= 1e-5 * max(1.0, abs(ddfo)) + 1e-6 * abs(lo)


@pytest.mark.parametrize("n", [4, 20, 61])
def test_mixed_optimize_all(gpu, n):
    rng = np.random.default_rng(40 + n)
    model = {4: synth.dna_gtr, 20: synth.protein, 61: synth.codon_gy}[n](rng)
    tree = synth.random_tree(24, 0.1, 7 + n)
    aln = synth.simulate(tree, model, 1500, 9 + n)
    safe = n == 61
    ot = orc.OracleTree(tree, model, aln, safe=safe)
    gt = gpu_tree(tree, model, aln, safe, precision="mixed")
    lo = ot.optimizeAllBranches(100, 0.001, 100)
    lg = gt.optimizeAllBranches(100, 0.001, 100)
    assert abs(lg - lo) <= MIXED_RTOL * abs(lo)
    # the mixed lengths are re-evaluated in FP64 by the oracle at its own precision
    ot2 = orc.OracleTree(synth.Tree(tree.ntaxa, tree.eu, tree.ev, gt.getBranchLengths()),
                         model, aln, safe=safe)
    assert abs(ot2.computeLikelihood() - lo) <= MIXED_RTOL * abs(lo)


def test_tensor_core_path_matches_cuda_core_path(gpu):
    """20-state mixed traversal: tcgen05 split-TF32 products against the FP32 CUDA-core
    kernel and the FP64 oracle, NORM and SAFE, including tip-tip, tip-internal and
    internal-internal nodes and pattern counts that are not a multiple of the 128-row tile."""
    rng = np.random.default_rng(77)
    model = synth.protein(rng, 4, 0.8)
    for safe, ntaxa, nsites in ((False, 30, 700), (True, 45, 333)):
        tree = synth.random_tree(ntaxa, 0.15, ntaxa)
        aln = synth.simulate(tree, model, nsites, ntaxa + 1)
        ot = orc.OracleTree(tree, model, aln, safe=safe)
        lo = ot.computeLikelihood()
        res = []
        for tc in (True, False):
            gt = gpu_tree(tree, model, aln, safe, precision="mixed")
            gt.session.set_tensor_cores(tc)
            lg, plg = gt.computeLikelihood(pattern_lh=True)
            assert abs(lg - lo) <= MIXED_RTOL * abs(lo), (tc, lg, lo)
            res.append(plg)
        assert np.max(np.abs(res[0] - res[1]) / (np.abs(res[1]) + 1)) < 1e-5
