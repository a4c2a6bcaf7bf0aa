"""Alignment ingest: the device pattern compression (gems_compress_alignment) against the
reference's pattern building restated in oracle/ingest.py -- same patterns in the same
first-appearance order, weights, site -> pattern map and constant states -- for DNA and protein
characters (ambiguity codes, gaps, lower case) and pre-encoded codon states; and at a larger size
against the host compressor."""
import glob
import os

import numpy as np
import pytest

from gems_b200 import GemsError, compress_alignment, synth
from oracle import ingest

DNA = "ACGTURYWSMKBHDVNXO-?.~acgtn"
PROT = "ARNDCQEGHILKMFPSTWYVBZJX*UO-?arndcq"


def random_chars(rng, ntaxa, nsites, alphabet, common, p_common=0.9):
    """Columns drawn from a small set so that patterns repeat, with random noise."""
    base = rng.choice(list(common), size=(ntaxa, 8))
    cols = base[:, rng.integers(8, size=nsites)]
    noise = rng.random((ntaxa, nsites)) > p_common
    cols[noise] = rng.choice(list(alphabet), size=int(noise.sum()))
    return ["".join(r) for r in cols]


def shuffled_columns(seed, ntaxa, nsites, gap=0.05):
    """Simulated DNA columns in a seeded random site order (so that first appearances are not
    grouped by pattern)."""
    rng = np.random.default_rng(seed)
    tree = synth.random_tree(ntaxa, 0.05, seed + 1)
    aln = synth.simulate(tree, synth.dna_gtr(rng), nsites, seed + 2, gap_frac=gap)
    cols = synth.expand_patterns(aln)
    return np.ascontiguousarray(cols[:, rng.permutation(cols.shape[1])])


def test_restatement_matches_host_compressor():
    """The restatement and the host compressor (synth.c) agree on encoded data."""
    codes = shuffled_columns(1, 12, 3000)
    host = synth.compress(codes, 4)
    pat, w, sp, cc = ingest.build_patterns(codes, 4)
    np.testing.assert_array_equal(host.patterns, pat)
    np.testing.assert_array_equal(host.weights, w)
    np.testing.assert_array_equal(pat[:, sp], codes)


def test_const_char_cases():
    # all unknown; one state with ambiguity around it; DNA ambiguity set; protein B; none
    assert ingest.const_char([18, 18], 4) == 18
    assert ingest.const_char([0, 8, 18], 4) == 0        # A, R = {A, G}, N
    assert ingest.const_char([8, 8], 4) == 8            # R, R -> R
    assert ingest.const_char([20, 23], 20) == 20        # B, X -> B
    assert ingest.const_char([0, 1], 4) == 19
    assert ingest.const_char([60, 61], 61) == 60


@pytest.mark.gpu
@pytest.mark.parametrize("n,alphabet,common", [(4, DNA, "ACGT-RN"), (20, PROT, "ARNDCQ-BX")])
def test_device_ingest_characters(gpu, n, alphabet, common):
    rng = np.random.default_rng(7 + n)
    seqs = random_chars(rng, 17, 5000, alphabet, common)
    raw = np.array([np.frombuffer(s.encode(), np.uint8) for s in seqs])
    pat, w, sp, cc = compress_alignment(raw, n)
    rp, rw, rsp, rcc = ingest.build_patterns(ingest.encode(seqs, n), n)
    np.testing.assert_array_equal(pat, rp)
    np.testing.assert_array_equal(w, rw)
    np.testing.assert_array_equal(sp, rsp)
    np.testing.assert_array_equal(cc, rcc)


@pytest.mark.gpu
def test_device_ingest_codon_states(gpu):
    rng = np.random.default_rng(9)
    codes = rng.integers(0, 62, size=(9, 800)).astype(np.uint8)
    codes[:, 400:] = codes[:, :400]          # every column appears twice
    codes[:, 10] = 61                        # all unknown
    codes[:, 11] = 5                         # constant
    pat, w, sp, cc = compress_alignment(codes, 61, encoded=True)
    rp, rw, rsp, rcc = ingest.build_patterns(codes, 61)
    np.testing.assert_array_equal(pat, rp)
    np.testing.assert_array_equal(w, rw)
    np.testing.assert_array_equal(sp, rsp)
    np.testing.assert_array_equal(cc, rcc)


@pytest.mark.gpu
def test_device_ingest_large_matches_host(gpu):
    """512 taxa x 200,000 sites with 5% gaps: same patterns and weights as the host compressor,
    and the site map reproduces the alignment."""
    codes = shuffled_columns(3, 512, 200_000)
    host = synth.compress(codes, 4)
    pat, w, sp, cc = compress_alignment(codes, 4, encoded=True)
    np.testing.assert_array_equal(pat, host.patterns)
    np.testing.assert_array_equal(w, host.weights)
    np.testing.assert_array_equal(pat[:, sp], codes)


@pytest.mark.gpu
def test_device_ingest_rejects_bad_character(gpu):
    raw = np.frombuffer(b"ACGTACGT" + b"ACGJACGT", np.uint8).reshape(2, 8)
    with pytest.raises(GemsError) as e:
        compress_alignment(raw, 4)
    assert e.value.status == 5


@pytest.mark.gpu
def test_ingest_to_session_lnl_matches_oracle(gpu):
    """Sequences -> device patterns -> session (tips, weights and +I terms loaded on the device):
    the lnL equals the oracle's on the same patterns, constant states and p_invar."""
    from gems_b200 import Ingest, PhyloTree, Session
    from oracle import oracle as orc
    codes = shuffled_columns(21, 20, 6000)
    rng = np.random.default_rng(22)
    amb = rng.random(codes.shape) < 0.02
    codes[amb] = rng.choice([8, 13, 7], size=int(amb.sum()))  # R, Y, M
    rng = np.random.default_rng(23)
    model = synth.dna_gtr(rng, 4, 0.5)
    model.p_invar = 0.2
    tree = synth.random_tree(20, 0.1, 24)
    ing = Ingest(codes, 4, encoded=True)
    pat, w, sp, cc = ing.read()
    s = Session(20, ing.npat, 4, 4, 18)
    ing.to_session(s, model.p_invar, model.freq)
    s.set_model(model.eval, model.evec, model.inv_evec, model.rates, model.props)
    gt = PhyloTree(s, tree.eu, tree.ev, tree.length)
    aln = synth.Alignment(20, 4, int(w.sum()), pat, w)
    ot = orc.OracleTree(tree, model, aln, const_char=cc, p_invar=model.p_invar)
    lo, lg = ot.computeLikelihood(), gt.computeLikelihood()
    assert abs(lg - lo) <= 1e-9 * abs(lo), (lg, lo)
    ing.close()


# ---- pinned to the reference program on the reference's own test alignments ----
INGEST_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ingest",
                                              "*.npz")))
INGEST_IDS = [os.path.basename(p)[:-4] for p in INGEST_GOLDEN]


def _ingest_fixture(path):
    z = np.load(path)
    seqs = [bytes(r).decode() for r in z["chars"]]
    return z, seqs, int(z["nstates"])


@pytest.mark.parametrize("path", INGEST_GOLDEN, ids=INGEST_IDS)
def test_restatement_pattern_statistics_match_program(path):
    """Distinct patterns, constant / invariant / informative site counts and the per-site
    statistic (-alninfo) of the restatement equal the program's on the raw file characters."""
    z, seqs, n = _ingest_fixture(path)
    pat, w, sp, cc = ingest.build_patterns(ingest.encode(seqs, n), n)
    const, invar, inform, distinct = ingest.site_summary(pat, w, n)
    assert distinct == int(z["ref_distinct"])
    assert const == int(z["ref_const"])
    assert invar == int(z["ref_invariant"])
    assert inform == int(z["ref_informative"])
    stat = np.array([ingest.site_stat(pat[:, p], n) for p in range(pat.shape[1])])
    np.testing.assert_array_equal(stat[sp], z["ref_site_stat"])


def _fixture_case(z, pat, w):
    n = int(z["nstates"])
    tree = synth.Tree(int(z["ntaxa"]), z["eu"], z["ev"], z["length"])
    from oracle import oracle as orc
    ev, v, iv = orc.eigensystem(z["exch_upper"], z["freq"])
    model = synth.Model(n, z["exch_upper"], z["freq"], z["rates"], z["props"], ev, v, iv,
                        gamma_shape=float(z["alpha"]))
    aln = synth.Alignment(int(z["ntaxa"]), n, int(w.sum()), pat, w)
    return tree, model, aln


@pytest.mark.parametrize("path", INGEST_GOLDEN, ids=INGEST_IDS)
def test_restatement_site_lnl_matches_program(path):
    """Each site's log-likelihood, read through the restatement's site -> pattern map, equals
    the program's per-site value (printed to 6 significant digits) at a fixed model and tree;
    the total to the program's 12 decimals.  This pins the character encoding (ambiguity codes,
    gaps, case) and the site map together."""
    from oracle import oracle as orc
    z, seqs, n = _ingest_fixture(path)
    pat, w, sp, cc = ingest.build_patterns(ingest.encode(seqs, n), n)
    tree, model, aln = _fixture_case(z, pat, w)
    ot = orc.OracleTree(tree, model, aln, const_char=cc)
    lnl, plh = ot.computeLikelihood(pattern_lh=True)
    ref = float(z["ref_lnl"])
    assert abs(lnl - ref) <= 1e-11 * abs(ref), (lnl, ref)
    site = plh[sp]
    r = z["ref_site_lnl_6sig"]
    assert np.all(np.abs(site - r) <= 1e-5 * np.abs(r) + 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("path", INGEST_GOLDEN, ids=INGEST_IDS)
def test_device_ingest_on_reference_files(gpu, path):
    """The device ingest of the raw file characters gives the restatement's patterns, weights,
    site map and constant states, and a session loaded from it on the device reproduces the
    program's log-likelihood."""
    from gems_b200 import Ingest, PhyloTree, Session
    z, seqs, n = _ingest_fixture(path)
    raw = np.ascontiguousarray(z["chars"], np.uint8)
    ing = Ingest(raw, n)
    pat, w, sp, cc = ing.read()
    rp, rw, rsp, rcc = ingest.build_patterns(ingest.encode(seqs, n), n)
    np.testing.assert_array_equal(pat, rp)
    np.testing.assert_array_equal(w, rw)
    np.testing.assert_array_equal(sp, rsp)
    np.testing.assert_array_equal(cc, rcc)
    tree, model, aln = _fixture_case(z, pat, w)
    s = Session(tree.ntaxa, ing.npat, n, model.ncat, tree.ntaxa - 2)
    ing.to_session(s, 0.0, model.freq)
    s.set_model(model.eval, model.evec, model.inv_evec, model.rates, model.props)
    gt = PhyloTree(s, tree.eu, tree.ev, tree.length)
    lg = gt.computeLikelihood()
    ref = float(z["ref_lnl"])
    assert abs(lg - ref) <= 1e-11 * abs(ref), (lg, ref)
    ing.close()
