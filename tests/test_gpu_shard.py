"""Pattern sharding with GPU engines: 2 ranks (gloo for the host-side sum), each holding a
gems_b200.PhyloTree session over its pattern slab on the one available GPU.  The ranks' kernels
never wait on one another (the only exchange is the all-reduce of host scalars between
evaluations).  Sharded lnL, derivatives and lock-step Newton (optimizeOneBranch with its
divergence check) must equal the unsharded oracle at the FP64 bar."""
import os
import pickle
import socket

import numpy as np
import pytest

from gems_b200 import synth
from gems_b200.shard import ShardedTree, shard_alignment

pytestmark = pytest.mark.gpu

BRANCHES = (2, 9, 17)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    rng = np.random.default_rng(31)
    model = synth.dna_gtr(rng)
    tree = synth.random_tree(20, 0.1, 32)
    aln = synth.simulate(tree, model, 8000, 33, gap_frac=0.02)
    return tree, model, aln


def _worker(rank, world, port, outdir, precision):
    import datetime
    import torch.distributed as dist
    from gems_b200 import PhyloTree
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    tree, model, aln = _case()
    eng = PhyloTree.from_case(tree, model, shard_alignment(aln, rank, world),
                              precision=precision, device=0)
    st = ShardedTree(eng, dist)
    res = {"lnl": st.computeLikelihood(), "derv": [], "opt": []}
    for e in BRANCHES:
        u, v = int(tree.eu[e]), int(tree.ev[e])
        eng.clearAllPartialLH()
        res["derv"].append(st.computeLikelihoodDerv(v, u))
    for e in BRANCHES:
        u, v = int(tree.eu[e]), int(tree.ev[e])
        res["opt"].append(st.optimizeOneBranch(u, v))
    eng.clearAllPartialLH()
    res["lnl_after"] = st.computeLikelihood()
    with open(os.path.join(outdir, f"r{rank}.pkl"), "wb") as f:
        pickle.dump(res, f)
    eng.close()
    eng.session.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_rank_gpu_shards_match_unsharded_oracle(gpu, tmp_path, precision):
    import torch.multiprocessing as mp
    from oracle import oracle as orc
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), precision), nprocs=2, join=True)
    res = [pickle.load(open(tmp_path / f"r{r}.pkl", "rb")) for r in range(2)]
    tree, model, aln = _case()
    full = orc.OracleTree(tree, model, aln)
    lnl = full.computeLikelihood()
    derv = []
    for e in BRANCHES:
        u, v = int(tree.eu[e]), int(tree.ev[e])
        full.clearAllPartialLH()
        derv.append(full.computeLikelihoodDerv(v, u))
    opt = []
    for e in BRANCHES:
        u, v = int(tree.eu[e]), int(tree.ev[e])
        full.optimizeOneBranch(u, v)
        opt.append(full.getBranchLength(u, v))
    full.clearAllPartialLH()
    lnl_after = full.computeLikelihood()
    rl, rd, ro = (1e-9, 1e-9, 1e-8) if precision == "fp64" else (1e-6, 1e-5, 1e-5)
    for r in res:
        assert abs(r["lnl"] - lnl) <= rl * abs(lnl)
        for (df, ddf), (gdf, gddf) in zip(derv, r["derv"]):
            assert abs(gdf - df) <= rd * max(abs(df), abs(ddf) * 1e-3, 1.0)
            assert abs(gddf - ddf) <= rd * max(1.0, abs(ddf))
        assert np.allclose(r["opt"], opt, rtol=0, atol=ro)
        assert abs(r["lnl_after"] - lnl_after) <= rl * abs(lnl_after)
    assert res[0] == res[1]  # every rank holds the same reduced values and lengths
