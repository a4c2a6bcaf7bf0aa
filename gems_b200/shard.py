"""Pattern sharding across ranks (one process per GPU).

Every partial, theta entry, scale counter and tip byte at pattern p depends only on pattern p,
so an alignment splits into contiguous pattern slabs, one per rank, with no exchange during a
traversal.  The only collective is a sum over ranks: of the lnL for a likelihood evaluation,
of (df, ddf) for a derivative evaluation.  The Newton iteration then runs in lock-step on every
rank with identical scalars (the same safeguarded update as Optimization::minimizeNewton,
utils/optimization.cpp:422-499).

The per-rank engine is anything with the PhyloTree methods used below (gems_b200.PhyloTree on
a GPU).  Collectives go through torch.distributed (NCCL between GPUs; gloo works too).
"""
from __future__ import annotations

import math

import numpy as np

from .synth import Alignment


def shard_bounds(npat: int, rank: int, world: int, align: int = 64):
    """[lo, hi) pattern range of `rank`: contiguous slabs, boundaries on multiples of `align`."""
    per = -(-npat // world)
    per = -(-per // align) * align
    lo = min(npat, rank * per)
    hi = min(npat, lo + per)
    return lo, hi


def shard_alignment(aln: Alignment, rank: int, world: int) -> Alignment:
    lo, hi = shard_bounds(aln.npat, rank, world)
    pat = np.ascontiguousarray(aln.patterns[:, lo:hi])
    w = np.ascontiguousarray(aln.weights[lo:hi])
    return Alignment(aln.ntaxa, aln.nstates, int(w.sum()), pat, w)


class ShardedTree:
    """The PhyloTree calls of the path over pattern shards, one engine per rank."""

    def __init__(self, engine, dist, group=None, device="cpu"):
        import torch
        self.engine = engine
        self.dist = dist
        self.group = group
        self.buf = torch.zeros(3, dtype=torch.float64, device=device)

    def _sum(self, *vals):
        for i, v in enumerate(vals):
            self.buf[i] = v
        self.dist.all_reduce(self.buf, group=self.group)
        return [float(x) for x in self.buf[: len(vals)].tolist()]

    def computeLikelihood(self):
        return self._sum(self.engine.computeLikelihood())[0]

    def computeLikelihoodBranch(self, node, dad):
        return self._sum(self.engine.computeLikelihoodBranch(node, dad))[0]

    def computeLikelihoodDerv(self, node, dad):
        df, ddf = self.engine.computeLikelihoodDerv(node, dad)
        return tuple(self._sum(df, ddf))

    def optimizeOneBranch(self, node1, node2, min_bl=1e-6, max_bl=10.0, max_nr_step=100):
        """Newton on -lnL(t) of the whole (sharded) alignment; every rank takes the same
        steps, then the reference's divergence check.  Returns the optimal length (also set on
        the engine)."""
        eng = self.engine
        t0 = eng.getBranchLength(node1, node2)
        first = [True]

        def fd(x):
            # computeFuncDerv (phylotree.cpp:2555) on each shard, summed over ranks; theta is
            # rebuilt only for the first evaluation of the branch
            f_loc, df_loc = eng.computeFuncDerv(node1, node2, x, first[0])
            first[0] = False
            return tuple(self._sum(f_loc, df_loc))

        x1, x2, xacc = min_bl, max_bl, min_bl
        rts = min(max(t0, x1), x2)
        f, df = fd(rts)
        res = None
        if not (math.isfinite(f) and math.isfinite(df)):
            res = rts
        elif df >= 0.0 and abs(f) < xacc:
            res = rts
        if res is None:
            if f < 0.0:
                xl, xh = rts, x2
            else:
                xh, xl = rts, x1
            dx = abs(xh - xl)
            for j in range(1, max_nr_step + 1):
                rts_old = rts
                if df <= 0.0 or ((rts - xh) * df - f) * ((rts - xl) * df - f) >= 0.0:
                    dx = 0.5 * (xh - xl)
                    rts = xl + dx
                    if xl == rts:
                        res = rts
                        break
                else:
                    dx = f / df
                    temp = rts
                    rts -= dx
                    if temp == rts:
                        res = rts
                        break
                if abs(dx) < xacc or j == max_nr_step:
                    res = rts_old
                    break
                f, df = fd(rts)
                if not (math.isfinite(f) and math.isfinite(df)):
                    res = rts
                    break
                if df > 0.0 and abs(f) < xacc:
                    res = rts
                    break
                if f < 0.0:
                    xl = rts
                elif f > 0.0:
                    xh = rts
        if res > max_bl * 0.95:
            # Newton diverged towards the upper bound: keep the old length if its lnL is
            # higher (optimizeOneBranch, phylotree.cpp:2640-2650); both lnL values are sums
            # over ranks from the resident theta, and every rank takes the same decision
            eng.computeFuncDerv(node1, node2, res, False)
            opt_lh = self._sum(eng.computeLikelihoodFromBuffer())[0]
            eng.computeFuncDerv(node1, node2, t0, False)
            orig_lh = self._sum(eng.computeLikelihoodFromBuffer())[0]
            if orig_lh > opt_lh:
                res = t0
        eng.setLength(node1, node2, res)  # also invalidates the partials across the branch
        return res
