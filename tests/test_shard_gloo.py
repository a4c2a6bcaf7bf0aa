"""Pattern sharding over 2 ranks (gloo, CPU): the per-rank engine is the oracle, the exchange
is the same all-reduce the GPU ranks use.  Sharded lnL, derivatives and lock-step Newton must
equal the unsharded ones."""
import os
import pickle
import socket

import numpy as np
import pytest

from gems_b200 import synth
from gems_b200.shard import ShardedTree, shard_alignment, shard_bounds


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    rng = np.random.default_rng(12)
    model = synth.dna_gtr(rng)
    tree = synth.random_tree(14, 0.1, 5)
    aln = synth.simulate(tree, model, 3000, 6)
    return tree, model, aln


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from oracle import oracle as orc
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    tree, model, aln = _case()
    eng = orc.OracleTree(tree, model, shard_alignment(aln, rank, world))
    st = ShardedTree(eng, dist)
    res = {"lnl": st.computeLikelihood()}
    u, v = int(tree.eu[4]), int(tree.ev[4])
    eng.clearAllPartialLH()
    res["derv"] = st.computeLikelihoodDerv(v, u)
    res["opt"] = st.optimizeOneBranch(u, v)
    eng.clearAllPartialLH()
    res["lnl_after"] = st.computeLikelihood()
    with open(os.path.join(outdir, f"r{rank}.pkl"), "wb") as f:
        pickle.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_bounds_cover_and_align():
    for npat in (1, 63, 64, 1000, 12345):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(npat, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == npat
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and a <= b
            assert all(lo % 64 == 0 for lo, _ in spans if lo < npat)


def test_two_rank_gloo_matches_unsharded(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle as orc
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    res = [pickle.load(open(tmp_path / f"r{r}.pkl", "rb")) for r in range(2)]
    tree, model, aln = _case()
    full = orc.OracleTree(tree, model, aln)
    lnl = full.computeLikelihood()
    u, v = int(tree.eu[4]), int(tree.ev[4])
    full.clearAllPartialLH()
    df, ddf = full.computeLikelihoodDerv(v, u)
    full.optimizeOneBranch(u, v)
    opt = full.getBranchLength(u, v)
    full.clearAllPartialLH()
    lnl_after = full.computeLikelihood()
    for r in res:  # every rank holds the same reduced values
        assert abs(r["lnl"] - lnl) <= 1e-10 * abs(lnl)
        assert abs(r["derv"][0] - df) <= 1e-9 * max(1, abs(df))
        assert abs(r["derv"][1] - ddf) <= 1e-9 * max(1, abs(ddf))
        assert abs(r["opt"] - opt) <= 1e-8
        assert abs(r["lnl_after"] - lnl_after) <= 1e-10 * abs(lnl_after)
    assert res[0] == res[1]


class _FakeEngine:
    """An engine whose -lnL has its minimum at the upper bound and whose lnL at the old
    length is higher than at that minimum: optimizeOneBranch's divergence check must keep
    the old length."""

    def __init__(self):
        self.t = 0.3
        self.lengths = {}

    def getBranchLength(self, u, v):
        return 0.3

    def computeFuncDerv(self, u, v, x, new_branch=False):
        self.t = x
        return -1.0, 1.0  # f < 0 everywhere: Newton walks to the upper bound

    def computeLikelihoodFromBuffer(self):
        return -10.0 if abs(self.t - 0.3) < 1e-12 else -20.0

    def setLength(self, u, v, x):
        self.lengths[(u, v)] = x


class _NoDist:
    @staticmethod
    def all_reduce(buf, group=None):
        return None


def test_divergence_check_keeps_old_length():
    eng = _FakeEngine()
    st = ShardedTree(eng, _NoDist)
    assert st.optimizeOneBranch(0, 1) == 0.3
    assert eng.lengths[(0, 1)] == 0.3
