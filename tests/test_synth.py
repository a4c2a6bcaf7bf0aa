"""The seeded generator: determinism, tree shape, pattern compression."""
import numpy as np

from gems_b200 import synth


def test_tree_shape_and_determinism():
    a = synth.random_tree(30, 0.1, 7)
    b = synth.random_tree(30, 0.1, 7)
    assert a.nedges == 57
    assert np.array_equal(a.eu, b.eu) and np.array_equal(a.length, b.length)
    deg = np.bincount(np.concatenate([a.eu, a.ev]), minlength=a.nnodes)
    assert np.all(deg[:30] == 1) and np.all(deg[30:] == 3)
    assert abs(np.mean(synth.random_tree(400, 0.1, 1).length) - 0.1) < 0.02


def test_compression_round_trip():
    rng = np.random.default_rng(0)
    cols = rng.integers(0, 4, size=(6, 5000)).astype(np.uint8)
    cols[:, 100:200] = cols[:, :100]
    aln = synth.compress(cols, 4)
    assert aln.weights.sum() == 5000
    assert len({aln.patterns[:, i].tobytes() for i in range(aln.npat)}) == aln.npat
    exp = synth.expand_patterns(aln)
    key = lambda m: sorted(m[:, i].tobytes() for i in range(m.shape[1]))
    assert key(exp) == key(cols)


def test_simulation_is_seeded_and_respects_gaps():
    tree, model, aln = synth.config_dna16(seed=3, nsites=4000)
    tree2, model2, aln2 = synth.config_dna16(seed=3, nsites=4000)
    assert np.array_equal(aln.patterns, aln2.patterns)
    rng = np.random.default_rng(1)
    m = synth.dna_gtr(rng)
    t = synth.random_tree(10, 0.1, 2)
    g = synth.simulate(t, m, 20000, 3, gap_frac=0.05)
    cols = synth.expand_patterns(g)
    frac = np.mean(cols == synth.DNA_UNKNOWN)
    assert 0.045 < frac < 0.055
    assert cols.max() <= synth.DNA_UNKNOWN


def test_model_eigensystem():
    rng = np.random.default_rng(2)
    for m in (synth.dna_gtr(rng), synth.protein(rng), synth.codon_gy(rng)):
        q = m.evec @ np.diag(m.eval) @ m.inv_evec
        assert np.allclose(q.sum(1), 0, atol=1e-10)
        assert np.allclose(m.inv_evec @ m.evec, np.eye(m.nstates), atol=1e-9)
    assert len(synth.codon_sense()[0]) == 61
    r = synth.gamma_rates(0.5, 4)
    assert abs(r.mean() - 1) < 1e-12
