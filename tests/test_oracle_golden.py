"""The CPU oracle against outputs of the reference program (golden fixtures made by
tests/golden/make_golden.py from the shipped IQ-TREE 2.4.0 executable and the reference's own
test data)."""
import os

import numpy as np
import pytest

from conftest import golden_files, golden_opt_files, load_golden
from oracle import oracle as orc

CASES = golden_files()


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_lnl_at_fixed_lengths(path):
    tree, model, aln, z = load_golden(path)
    ot = orc.OracleTree(tree, model, aln, safe=bool(z["safe"]), const_char=z["const_char"])
    lnl, plh = ot.computeLikelihood(pattern_lh=True)
    ref = float(z["ref_lnl_fixed"])
    # the program prints 12 decimals; its eigensystem comes from a different solver
    assert abs(lnl - ref) <= 1e-11 * abs(ref)
    if "ref_pattern_lnl_6sig" in z:
        r = z["ref_pattern_lnl_6sig"]
        assert np.all(np.abs(plh - r) <= 1e-5 * np.abs(r) + 1e-5)
    # discrete Gamma category rates (printed to 12 significant digits)
    ncat = int(z["ncat"])
    rr = z["ref_rates"][-ncat:]
    rates = orc.gamma_rates(float(z["alpha"]), ncat)
    if float(z["p_invar"]) > 0:
        rates = rates * (ncat / (1 - float(z["p_invar"]))) / rates.sum()
    assert np.allclose(rates, rr, rtol=1e-10, atol=0)


OPT = golden_opt_files()


@pytest.mark.parametrize("path", OPT, ids=[os.path.basename(p)[:-4] for p in OPT])
def test_branch_optimisation_reaches_reference_optimum(path):
    tree, model, aln, z = load_golden(path)
    ot = orc.OracleTree(tree, model, aln, safe=bool(z["safe"]), const_char=z["const_char"])
    lnl = ot.optimizeAllBranches(100, 0.001, 100)
    ref = float(z["ref_lnl_opt"])
    # both stop at a lnL tolerance of 1e-3 and may visit branches in another order
    assert abs(lnl - ref) < 5e-3
    assert np.max(np.abs(ot.getBranchLengths() - z["ref_len_opt"])) < 5e-3


def test_eigensystem_reconstructs_q():
    from gems_b200 import synth
    rng = np.random.default_rng(7)
    for n, model in ((4, synth.dna_gtr(rng)), (20, synth.protein(rng))):
        ev, v, iv = orc.eigensystem(model.exch_upper, model.freq)
        q = v @ np.diag(ev) @ iv
        assert np.allclose(q.sum(axis=1), 0, atol=1e-12)
        assert np.allclose(iv @ v, np.eye(n), atol=1e-10)
        pi = model.freq / model.freq.sum()
        assert abs(-(pi * np.diag(q)).sum() - 1.0) < 1e-12  # one substitution per unit time
        assert np.allclose(np.sort(ev), np.sort(model.eval), atol=1e-10)
