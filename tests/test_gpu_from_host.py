"""Evaluation on new host data with the tip upload overlapped with the traversal
(gems_tree_compute_likelihood_from_host): the lnL and pattern lnL are bit-identical to loading
the tips, weights and +I terms first and evaluating after, for every chunk count and for the
forms that load first (tcgen05, 61 states); a bad tip byte fails the call and leaves the tips
invalid until a good load."""
import numpy as np
import pytest

from gems_b200 import GemsError, PhyloTree, synth
from gems_b200.synth import state_unknown

pytestmark = pytest.mark.gpu


def case(n, ncat, ntaxa=40, nsites=3000, seed=1):
    rng = np.random.default_rng(seed)
    if n == 4:
        model = synth.dna_gtr(rng, ncat, 0.5)
    elif n == 20:
        model = synth.protein(rng, ncat, 0.8)
    else:
        model = synth.codon_gy(rng, ncat, 0.5)
    tree = synth.random_tree(ntaxa, 0.1, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2)
    return tree, model, aln


def new_data(aln, n, seed, invar=True):
    """Other tip states of the same shape (ambiguity and gap codes included), weights and
    +I terms."""
    rng = np.random.default_rng(seed)
    st = aln.patterns.copy()
    mask = rng.random(st.shape) < 0.3
    st[mask] = rng.integers(0, state_unknown(n) + 1, size=int(mask.sum()))
    w = rng.integers(1, 5, size=aln.npat).astype(np.float64)
    iv = 0.02 * rng.random(aln.npat) * (rng.random(aln.npat) < 0.2) if invar else None
    return st, w, iv


def loaded_then_evaluated(gt, st, w, iv):
    gt.session.upload_tips(st)
    gt.session.upload_patterns(w, iv)
    gt.clearAllPartialLH()
    return gt.computeLikelihood(pattern_lh=True)


FORMS = [(4, 4, "fp64", True), (4, 4, "mixed", True), (4, 1, "mixed", True),
         (20, 4, "fp64", True), (20, 4, "mixed", False), (20, 4, "mixed", True),
         (61, 4, "mixed", True)]


@pytest.mark.parametrize("n,ncat,precision,tc", FORMS,
                         ids=[f"{n}s-C{c}-{p}{'' if t else '-cudacores'}" for n, c, p, t in FORMS])
def test_same_as_load_then_evaluate(gpu, n, ncat, precision, tc):
    tree, model, aln = case(n, ncat, nsites=3000 if n != 61 else 800)
    scaling = "safe" if n == 61 else "norm"
    gt = PhyloTree.from_case(tree, model, aln, precision=precision, scaling=scaling)
    gt.session.set_tensor_cores(tc)
    gt.computeLikelihood()
    for k, chunks in enumerate((1, 3, 8, 64)):
        st, w, iv = new_data(aln, n, 10 + k, invar=k % 2 == 0)
        got, plh = gt.computeLikelihoodFromHost(st, w, iv, chunks=chunks, pattern_lh=True)
        want, wplh = loaded_then_evaluated(gt, st, w, iv)
        assert got == want, (chunks, got, want)
        np.testing.assert_array_equal(plh, wplh)
    # back to the first data: the lnL of a fresh evaluation
    ref = PhyloTree.from_case(tree, model, aln, precision=precision, scaling=scaling)
    ref.session.set_tensor_cores(tc)
    assert gt.computeLikelihoodFromHost(aln.patterns, aln.weights, chunks=5) == \
        ref.computeLikelihood()
    for t in (gt, ref):
        t.close()
        t.session.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_many_chunks_ragged_pattern_count(gpu, precision):
    """Enough patterns for several chunks of whole waves, and a count that is not a multiple of
    the tiles (P padded to 64): every chunk bound and the padded tail."""
    rng = np.random.default_rng(5)
    model = synth.dna_gtr(rng, 4, 0.5)
    tree = synth.random_tree(40, 0.1, 6)
    aln = synth.simulate(tree, model, 300_001, 7, gap_frac=0.05)
    assert aln.npat > 200_000 and aln.npat % 64 != 0
    gt = PhyloTree.from_case(tree, model, aln, precision=precision)
    want = gt.computeLikelihood(pattern_lh=True)
    for chunks in (2, 3, 8, 64):
        got = gt.computeLikelihoodFromHost(aln.patterns, aln.weights, chunks=chunks,
                                           pattern_lh=True)
        assert got[0] == want[0], chunks
        np.testing.assert_array_equal(got[1], want[1])
    out = np.empty(aln.npat)
    assert gt.computeLikelihoodFromHost(aln.patterns, aln.weights, pattern_lh=out)[0] == want[0]
    np.testing.assert_array_equal(out, want[1])
    gt.close()
    gt.session.close()


def test_bad_tip_byte_rejected(gpu):
    tree, model, aln = case(4, 4, seed=7)
    gt = PhyloTree.from_case(tree, model, aln, precision="mixed")
    good = gt.computeLikelihood()
    bad = aln.patterns.copy()
    bad[3, aln.npat // 2] = 200
    with pytest.raises(GemsError) as e:
        gt.computeLikelihoodFromHost(bad, aln.weights, chunks=4)
    assert e.value.status == 5
    with pytest.raises(GemsError) as e:  # the tips stay invalid
        gt.clearAllPartialLH()
        gt.computeLikelihood()
    assert e.value.status == 7
    assert gt.computeLikelihoodFromHost(aln.patterns, aln.weights, chunks=4) == good
    gt.close()
    gt.session.close()
