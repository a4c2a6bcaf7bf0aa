"""ctypes wrapper of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg as the checker.  Never used by the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import byref, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "oracle.c")
        if not os.path.exists(path) or os.path.getmtime(src) > os.path.getmtime(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_tree_new.restype = c_void_p
        for f in ("orc_compute_likelihood", "orc_compute_likelihood_branch",
                  "orc_compute_likelihood_from_buffer", "orc_optimize_all_branches",
                  "orc_get_length"):
            getattr(L, f).restype = c_double
        L.orc_partial_ops.restype = ctypes.c_longlong
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def gamma_rates(alpha, ncat, median=False):
    out = np.zeros(ncat)
    lib().orc_gamma_rates(c_double(alpha), ncat, int(median), _p(out))
    return out


def eigensystem(exch_upper, freq):
    n = len(freq)
    ev, v, iv = np.zeros(n), np.zeros(n * n), np.zeros(n * n)
    rc = lib().orc_eigensystem_sym(n, _p(np.ascontiguousarray(exch_upper, np.float64)),
                                   _p(np.ascontiguousarray(freq, np.float64)), _p(ev), _p(v),
                                   _p(iv))
    assert rc == 0
    return ev, v.reshape(n, n), iv.reshape(n, n)


def set_threads(n):
    lib().orc_set_threads(int(n))


class OracleTree:
    """Same method names as the reference PhyloTree and gems_b200.PhyloTree."""

    def __init__(self, tree, model, aln, safe=False, const_char=None, p_invar=None):
        L = lib()
        self.L = L
        # own copies: doNNI rewrites them in place
        self.eu = np.array(tree.eu, np.int32)
        self.ev = np.array(tree.ev, np.int32)
        ln = np.ascontiguousarray(tree.length, np.float64)
        self.h = c_void_p(L.orc_tree_new(tree.ntaxa, len(self.eu), _p(self.eu), _p(self.ev),
                                         _p(ln), model.nstates, model.ncat, int(safe)))
        assert self.h.value, "oracle: tree must be binary with leaves 0..ntaxa-1"
        pinv = model.p_invar if p_invar is None else p_invar
        arrs = [np.ascontiguousarray(x, np.float64) for x in
                (model.eval, model.evec, model.inv_evec, model.rates, model.props, model.freq)]
        L.orc_set_model(self.h, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), _p(arrs[4]),
                        c_double(pinv), _p(arrs[5]))
        self.pat = np.ascontiguousarray(aln.patterns, np.uint8)
        self.w = np.ascontiguousarray(aln.weights, np.float64)
        cc = None if const_char is None else np.ascontiguousarray(const_char, np.uint8)
        L.orc_set_patterns(self.h, aln.npat, _p(self.pat), _p(self.w), _p(cc))
        self.nptn = aln.npat
        self.nstates, self.ncat = model.nstates, model.ncat
        self.safe = safe

    def __del__(self):
        try:
            if self.h:
                self.L.orc_tree_free(self.h)
        except Exception:
            pass

    def setBranchLimits(self, lo, hi):
        self.L.orc_set_branch_limits(self.h, c_double(lo), c_double(hi))

    def setLength(self, u, v, x):
        assert self.L.orc_set_length(self.h, u, v, c_double(x)) == 0

    def getBranchLengths(self):
        out = np.zeros(len(self.eu))
        self.L.orc_get_lengths(self.h, _p(out))
        return out

    def clearAllPartialLH(self):
        self.L.orc_clear_all_partial_lh(self.h)

    def computeLikelihood(self, pattern_lh=False):
        plh = np.zeros(self.nptn) if pattern_lh else None
        v = self.L.orc_compute_likelihood(self.h, _p(plh))
        return (v, plh) if pattern_lh else v

    def computeLikelihoodBranch(self, node, dad, pattern_lh=False):
        plh = np.zeros(self.nptn) if pattern_lh else None
        v = self.L.orc_compute_likelihood_branch(self.h, node, dad, _p(plh))
        return (v, plh) if pattern_lh else v

    def computeLikelihoodDerv(self, node, dad):
        df, ddf = c_double(), c_double()
        self.L.orc_compute_likelihood_derv(self.h, node, dad, byref(df), byref(ddf))
        return df.value, ddf.value

    def computeLikelihoodFromBuffer(self):
        return self.L.orc_compute_likelihood_from_buffer(self.h)

    def getBranchLength(self, u, v):
        return self.L.orc_get_length(self.h, u, v)

    def doNNI(self, u, v, a, b):
        assert self.L.orc_nni(self.h, u, v, a, b) == 0
        for i in range(len(self.eu)):
            x, y = int(self.eu[i]), int(self.ev[i])
            if {x, y} == {u, a}:
                self.eu[i], self.ev[i] = v, a
            elif {x, y} == {v, b}:
                self.eu[i], self.ev[i] = u, b

    def doSPR(self, node, dad, node2, dad2):
        """Prune the subtree at node from dad and regraft dad into the branch (node2, dad2)."""
        others = sorted(x for x in self.neighbors(dad) if x != node)
        assert len(others) == 2 and node in self.neighbors(dad), "dad must be internal"
        s1, s2 = others
        assert self.L.orc_spr(self.h, node, dad, node2, dad2) == 0
        # edges: (dad, s1) -> (s1, s2), (dad, s2) -> (dad, dad2), (node2, dad2) -> (dad, node2)
        for i in range(len(self.eu)):
            e = {int(self.eu[i]), int(self.ev[i])}
            if e == {dad, s1}:
                self.eu[i], self.ev[i] = s1, s2
            elif e == {dad, s2}:
                self.eu[i], self.ev[i] = dad, dad2
            elif e == {node2, dad2}:
                self.eu[i], self.ev[i] = dad, node2

    def neighbors(self, u):
        return [int(b) if a == u else int(a) for a, b in zip(self.eu, self.ev) if u in (a, b)]

    def computeFuncDerv(self, node1, node2, value, new_branch=False):
        f, df = c_double(), c_double()
        self.L.orc_compute_func_derv(self.h, node1, node2, c_double(value), int(new_branch),
                                     byref(f), byref(df))
        return f.value, df.value

    def optimizeOneBranch(self, n1, n2, clearLH=True, maxNRStep=100):
        self.L.orc_optimize_one_branch(self.h, n1, n2, int(clearLH), maxNRStep)

    def optimizeAllBranches(self, my_iterations=100, tolerance=0.001, maxNRStep=100):
        return self.L.orc_optimize_all_branches(self.h, my_iterations, c_double(tolerance),
                                                maxNRStep)

    def getPartial(self, node, dad):
        P = self.L.orc_nptn_pad(self.h)
        blk = self.nstates * self.ncat
        part = np.zeros(P * blk)
        per = self.ncat if self.safe else 1
        sc = np.zeros(P * per, np.uint16)
        rc = self.L.orc_get_partial(self.h, node, dad, _p(part), _p(sc))
        assert rc == 0, rc
        part = part.reshape(P, self.ncat, self.nstates)[: self.nptn]
        sc = sc.reshape(P, per)[: self.nptn]
        return part, (sc if self.safe else sc[:, 0])

    def getTheta(self):
        P = self.L.orc_nptn_pad(self.h)
        blk = self.nstates * self.ncat
        th, sa = np.zeros(P * blk), np.zeros(P)
        assert self.L.orc_get_theta(self.h, _p(th), _p(sa)) == 0
        return th.reshape(P, blk)[: self.nptn], sa[: self.nptn]

    def dfFrac(self):
        g = np.zeros(self.nptn)
        self.L.orc_get_df_frac(self.h, _p(g))
        return g

    def partialOps(self):
        return self.L.orc_partial_ops(self.h)

    def lastNewtonEvals(self):
        return self.L.orc_last_newton_evals(self.h)
