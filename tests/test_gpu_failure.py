"""Failure handling on the device without a fault: the bounded grid barrier of the Newton loop
is made to wait for a block that never comes; it gives up, reports GEMS_ERR_TIMEOUT, and the
context stays usable -- the likelihood and a Newton branch optimisation afterwards still agree
with the oracle."""
import time

import numpy as np
import pytest

from gems_b200 import PhyloTree, check_barrier_timeout, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_device_stays_usable(gpu):
    t = time.perf_counter()
    assert check_barrier_timeout() == 4  # GEMS_ERR_TIMEOUT
    assert time.perf_counter() - t < 60
    rng = np.random.default_rng(3)
    model = synth.dna_gtr(rng, 4, 0.5)
    tree = synth.random_tree(20, 0.1, 4)
    aln = synth.simulate(tree, model, 2000, 5)
    ot = orc.OracleTree(tree, model, aln)
    gt = PhyloTree.from_case(tree, model, aln)
    lo, lg = ot.computeLikelihood(), gt.computeLikelihood()
    assert abs(lg - lo) <= 1e-9 * abs(lo)
    u, v = int(tree.eu[5]), int(tree.ev[5])
    ot.optimizeOneBranch(u, v)
    gt.optimizeOneBranch(u, v)
    assert abs(gt.getBranchLength(u, v) - ot.getBranchLength(u, v)) <= 1e-9
    gt.close()
    gt.session.close()
