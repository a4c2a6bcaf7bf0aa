"""Launch-shape tuning of the 4-state traversal: every shape gives the same lnL, pattern lnL and
partials bit for bit (FP64 and mixed), and a large enough traversal gets tuned."""
import numpy as np
import pytest

from gems_b200 import GemsError, PhyloTree, synth

pytestmark = pytest.mark.gpu


def case(seed, ntaxa, nsites):
    rng = np.random.default_rng(seed)
    model = synth.dna_gtr(rng, 4, 0.5)
    tree = synth.random_tree(ntaxa, 0.1, seed + 1)
    aln = synth.simulate(tree, model, nsites, seed + 2, gap_frac=0.05)
    return tree, model, aln


def computed_partials(gt, tree):
    out = {}
    for u, v in zip(tree.eu, tree.ev):
        for node, dad in ((int(u), int(v)), (int(v), int(u))):
            if node < tree.ntaxa:
                continue
            try:
                out[(node, dad)] = gt.getPartial(node, dad)
            except GemsError:
                pass
    return out


# shapes: the plan-driven kernels with staged inputs first (mixed: one thread per pattern, then
# two with a lane per category; FP64: two with a lane per category, then one thread per
# pattern), then the kernels that read every child and table from global memory
@pytest.mark.parametrize("scaling", ["norm", "safe"])
@pytest.mark.parametrize("precision,nshapes", [("fp64", 6), ("mixed", 7)])
def test_every_shape_gives_the_same_values(gpu, precision, nshapes, scaling):
    tree, model, aln = case(11, 40, 5001)
    ref = None
    seen = set()
    for k in range(nshapes):
        gt = PhyloTree.from_case(tree, model, aln, precision=precision, scaling=scaling)
        gt.session.set_autotune(force_shape=k)
        lnl, plh = gt.computeLikelihood(pattern_lh=True)
        part = computed_partials(gt, tree)
        pp, blocks, _ = gt.session.traversal_shape()
        seen.add((pp, blocks))
        if ref is None:
            ref = (lnl, plh, part)
        else:
            assert lnl == ref[0]
            np.testing.assert_array_equal(plh, ref[1])
            if part is not None:
                assert part.keys() == ref[2].keys() and len(part) >= tree.ntaxa - 2
                for key in part:
                    np.testing.assert_array_equal(part[key][0], ref[2][key][0])
                    np.testing.assert_array_equal(part[key][1], ref[2][key][1])
        gt.close()
        gt.session.close()
    # the forced shapes did switch kernels (two kernels may report the same launch shape)
    assert len(seen) >= nshapes - 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_traversal_gets_tuned(gpu, precision):
    tree, model, aln = case(21, 64, 80_000)   # 62 ops x ~80k patterns > 2^22 pattern-updates
    gt = PhyloTree.from_case(tree, model, aln, precision=precision)
    lnl = gt.computeLikelihood()
    pp, blocks, tuned = gt.session.traversal_shape()
    assert tuned and pp >= 1 and blocks >= 1
    ref = PhyloTree.from_case(tree, model, aln, precision=precision)
    ref.session.set_autotune(force_shape=0)
    assert ref.computeLikelihood() == lnl
    for t in (gt, ref):
        t.close()
        t.session.close()
