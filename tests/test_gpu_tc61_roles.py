"""The 61-state tcgen05 traversal with warp roles (split, MMA issue, epilogue and copies working
on consecutive steps at once; GEMS_OPT_TC61_ROLES, the default) gives the bits of the form in
which every warp runs the parts of a step in turn: one, four and eight categories, pattern
counts that are not a multiple of the 128-row tile, deep trees that rescale, LM_MEM_SAVE pools
(slots rewritten inside one op list) and batched candidate models."""
import numpy as np
import pytest

from gems_b200 import PhyloTree, Session, branch_lnl_batch, full_traversal, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
MIXED_RTOL = 1e-6


def codon_case(ncat, seed, ntaxa=30, nsites=700, blen=0.1):
    rng = np.random.default_rng(seed)
    model = synth.codon_gy(rng, ncat, 0.5, freerate=ncat == 8)
    tree = synth.random_tree(ntaxa, blen, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2, gap_frac=0.05)
    return tree, model, aln


def both_forms(tree, model, aln, slots="node"):
    out = []
    for roles in (True, False):
        gt = PhyloTree.from_case(tree, model, aln, precision="mixed", scaling="safe", slots=slots)
        gt.session.set_tc61_roles(roles)
        lnl, plh = gt.computeLikelihood(pattern_lh=True)
        u, v = int(tree.eu[len(tree.eu) // 2]), int(tree.ev[len(tree.eu) // 2])
        df, ddf = gt.computeLikelihoodDerv(v, u)
        out.append((lnl, np.array(plh), df, ddf))
        gt.close()
        gt.session.close()
    return out


@pytest.mark.parametrize("ncat", [1, 4, 8])
def test_roles_same_bits(gpu, ncat):
    tree, model, aln = codon_case(ncat, 160 + ncat)
    assert aln.npat % 128 != 0
    a, b = both_forms(tree, model, aln)
    assert a[0] == b[0] and np.array_equal(a[1], b[1]), (a[0], b[0])
    assert a[2] == b[2] and a[3] == b[3]
    lo = orc.OracleTree(tree, model, aln, safe=True).computeLikelihood()
    assert abs(a[0] - lo) <= MIXED_RTOL * abs(lo), (a[0], lo)


def test_roles_deep_tree_and_pool(gpu):
    """Long branches on 120 taxa rescale many rows; the LM_MEM_SAVE pool rewrites slots
    within one op list, so copies of recently stored rows wait for their stores."""
    tree, model, aln = codon_case(4, 171, ntaxa=120, nsites=400, blen=0.3)
    lo = orc.OracleTree(tree, model, aln, safe=True).computeLikelihood()
    for slots in ("node", "pool"):
        a, b = both_forms(tree, model, aln, slots=slots)
        assert a[0] == b[0] and np.array_equal(a[1], b[1]), (slots, a[0], b[0])
        assert abs(a[0] - lo) <= MIXED_RTOL * abs(lo), (slots, a[0], lo)


def test_roles_batched_models(gpu):
    tree, model0, aln = codon_case(4, 181, ntaxa=40, nsites=900)
    rng = np.random.default_rng(182)
    models = [model0] + [synth.codon_gy(rng, 4, float(rng.uniform(0.3, 1.5))) for _ in range(7)]
    ops, br = full_traversal(tree)
    res = []
    for roles in (True, False):
        sessions = []
        for m in models:
            s = Session(tree.ntaxa, aln.npat, 61, 4, tree.ntaxa - 2, "mixed", "safe")
            s.upload_tips(aln.patterns)
            s.upload_patterns(aln.weights)
            s.set_model(m.eval, m.evec, m.inv_evec, m.rates, m.props)
            s.set_tc61_roles(roles)
            sessions.append(s)
        res.append(list(branch_lnl_batch(sessions, ops, br)))
        for s in sessions:
            s.close()
    assert res[0] == res[1]
