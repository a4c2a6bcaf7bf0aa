"""Python binding of the C-ABI (ctypes).  Method names of :class:`PhyloTree` follow the
reference's PhyloTree (tree/phylotree.h) so callers and tests read like IQ-TREE code."""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_longlong, c_size_t, c_uint16, c_void_p

import numpy as np

from . import _lib

STATUS = {0: "OK", 1: "OOM", 2: "ADMISSION_REJECTED", 3: "NUMERIC_UNDERFLOW", 4: "TIMEOUT",
          5: "BAD_ARG", 6: "CUDA", 7: "STATE", 8: "NO_DEVICE"}
GEMS_CHILD_TIP = 0
GEMS_CHILD_PARTIAL = 1
PREC = {"fp64": 0, "mixed": 1}
SCALING = {"norm": 0, "safe": 1}


class GemsError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = _lib.gems().gems_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS.get(status, status)} ({msg})")


def _check(st: int, where: str):
    if st != 0:
        raise GemsError(st, where)


class SessionDesc(ctypes.Structure):
    _fields_ = [("ntaxa", c_int), ("nptn", c_int), ("nstates", c_int), ("ncat", c_int),
                ("nslots", c_int), ("precision", c_int), ("scaling", c_int), ("device", c_int)]


class Op(ctypes.Structure):
    _fields_ = [("dst_slot", c_int), ("left_kind", c_int), ("left_id", c_int),
                ("right_kind", c_int), ("right_id", c_int), ("pad_", c_int),
                ("left_len", c_double), ("right_len", c_double)]


class Branch(ctypes.Structure):
    _fields_ = [("dad_slot", c_int), ("node_kind", c_int), ("node_id", c_int), ("pad_", c_int),
                ("length", c_double)]


def op_array(ops):
    """ops: iterable of (dst, lkind, lid, rkind, rid, llen, rlen)."""
    ops = list(ops)
    arr = (Op * max(1, len(ops)))()
    for i, (d, lk, li, rk, ri, ll, rl) in enumerate(ops):
        arr[i] = Op(d, lk, li, rk, ri, 0, ll, rl)
    return arr, len(ops)


def branch_struct(dad_slot, node_kind, node_id, length):
    return Branch(dad_slot, node_kind, node_id, 0, length)


def _dptr(a):
    return a.ctypes.data_as(c_void_p) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def measure_peaks(device=0):
    """Measured FP64 / FP32 FMA and dense TF32 tensor-core peaks of a device (TFLOP/s)."""
    lib = _lib.gems()
    a, b, c = c_double(), c_double(), c_double()
    _check(lib.gems_measure_peaks(device, byref(a), byref(b), byref(c)), "gems_measure_peaks")
    return {"fp64_tflops": a.value, "fp32_tflops": b.value, "tf32_tflops": c.value}


def check_barrier_timeout(device=0):
    """Status the grid barrier reports when a wait cannot complete (GEMS_ERR_TIMEOUT = 4)."""
    st = c_int()
    _check(_lib.gems().gems_check_barrier_timeout(device, byref(st)), "check_barrier_timeout")
    return st.value


def compress_alignment(seqs, nstates, encoded=False, device=0):
    """Encode and compress an alignment on the device (gems_compress_alignment).
    seqs: [ntaxa][nsites] uint8 (characters, or state codes when encoded).  Returns
    (patterns [ntaxa][npat] uint8, weights [npat], site_pattern [nsites], const_char [npat])."""
    a = np.ascontiguousarray(seqs, dtype=np.uint8)
    ntaxa, nsites = a.shape
    pat = np.empty(ntaxa * nsites, np.uint8)
    w = np.empty(nsites, np.float64)
    sp = np.empty(nsites, np.int32)
    cc = np.empty(nsites, np.uint8)
    npat = c_longlong()
    lib = _lib.gems()
    _check(lib.gems_compress_alignment(device, ntaxa, c_longlong(nsites), nstates, _dptr(a),
                                       int(encoded), _dptr(pat), _dptr(w), _dptr(sp), _dptr(cc),
                                       byref(npat)), "gems_compress_alignment")
    k = npat.value
    return (np.ascontiguousarray(pat[: ntaxa * k].reshape(ntaxa, k)), w[:k].copy(), sp,
            cc[:k].copy())


class Ingest:
    """A compressed alignment kept on the device (gems_ingest_*): build it from sequences once,
    read results back or load them straight into a session."""

    def __init__(self, seqs, nstates, encoded=False, device=0):
        a = np.ascontiguousarray(seqs, dtype=np.uint8)
        self.ntaxa, self.nsites = a.shape
        self.nstates = nstates
        self.lib = _lib.gems()
        self.handle = c_void_p()
        npat = c_longlong()
        _check(self.lib.gems_ingest_create(device, self.ntaxa, c_longlong(self.nsites), nstates,
                                           _dptr(a), int(encoded), byref(self.handle),
                                           byref(npat)), "gems_ingest_create")
        self.npat = npat.value

    def read(self):
        """(patterns [ntaxa][npat], weights [npat], site_pattern [nsites], const_char [npat])."""
        pat = np.empty((self.ntaxa, self.npat), np.uint8)
        w = np.empty(self.npat, np.float64)
        sp = np.empty(self.nsites, np.int32)
        cc = np.empty(self.npat, np.uint8)
        _check(self.lib.gems_ingest_read(self.handle, _dptr(pat), _dptr(w), _dptr(sp), _dptr(cc)),
               "gems_ingest_read")
        return pat, w, sp, cc

    def to_session(self, session, p_invar=0.0, state_freq=None):
        f = None if state_freq is None else _f64(state_freq)
        _check(self.lib.gems_ingest_to_session(self.handle, session.handle, c_double(p_invar),
                                               _dptr(f)), "gems_ingest_to_session")

    def close(self):
        if self.handle:
            self.lib.gems_ingest_destroy(self.handle)
            self.handle = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def min_pool_slots(ntaxa):
    """The fewest partial slots a tree may run in (LM_MEM_SAVE: log2(leafNum) + LH_MIN_CONST,
    tree/phylotree.cpp:42,1026-1040)."""
    import math
    return int(math.log2(ntaxa)) + 1


def full_traversal(tree):
    """Ops of a from-scratch traversal with one slot per internal node (slot = node - ntaxa),
    rooted at the branch between leaf 0 and its neighbour, and that branch: (ops, branch)."""
    nt = tree.ntaxa
    adj = {}
    for u, v, ln in zip(tree.eu, tree.ev, tree.length):
        adj.setdefault(int(u), []).append((int(v), float(ln)))
        adj.setdefault(int(v), []).append((int(u), float(ln)))
    root, rlen = adj[0][0]
    ops = []
    stack = [(root, 0, False)]
    while stack:
        x, dad, done = stack.pop()
        kids = [(y, ln) for y, ln in adj[x] if y != dad]
        if not done:
            stack.append((x, dad, True))
            stack.extend((y, x, False) for y, _ in kids if y >= nt)
            continue
        (a, la), (b, lb) = kids
        kind = lambda y: (GEMS_CHILD_TIP, y) if y < nt else (GEMS_CHILD_PARTIAL, y - nt)
        (ka, ia), (kb, ib) = kind(a), kind(b)
        ops.append((x - nt, ka, ia, kb, ib, la, lb))
    return ops, branch_struct(root - nt, GEMS_CHILD_TIP, 0, rlen)


def set_models_from_rates(sessions, exch_upper, freq, rates, props):
    """gems_set_model_from_rates_batch: every session's eigensystem in one launch.  Arguments
    are per-session sequences (stacked row by row)."""
    lib = _lib.gems()
    arr = _session_array(sessions)
    ex = np.ascontiguousarray(np.stack([_f64(x) for x in exch_upper]))
    fr = np.ascontiguousarray(np.stack([_f64(x) for x in freq]))
    rt = np.ascontiguousarray(np.stack([_f64(x) for x in rates]))
    pr = np.ascontiguousarray(np.stack([_f64(x) for x in props]))
    _check(lib.gems_set_model_from_rates_batch(arr, len(sessions), _dptr(ex), _dptr(fr),
                                               _dptr(rt), _dptr(pr)),
           "gems_set_model_from_rates_batch")


def optimize_all_branches_batch(trees, my_iterations=100, tolerance=0.001, maxNRStep=100):
    """gems_tree_optimize_all_branches_batch: optimizeAllBranches on PhyloTrees of one topology
    (one per candidate model), their device work overlapped; returns their lnL."""
    lib = _lib.gems()
    arr = (c_void_p * len(trees))()
    for i, t in enumerate(trees):
        arr[i] = t.handle.value
    out = np.zeros(len(trees))
    _check(lib.gems_tree_optimize_all_branches_batch(arr, len(trees), int(my_iterations),
                                                     c_double(tolerance), int(maxNRStep),
                                                     _dptr(out)),
           "gems_tree_optimize_all_branches_batch")
    return out


def compute_likelihood_batch(trees):
    """gems_tree_compute_likelihood_batch: computeLikelihood of PhyloTrees on sessions that share
    the alignment's shape (one per candidate model), evaluated together; returns their lnL."""
    lib = _lib.gems()
    arr = (c_void_p * len(trees))()
    for i, t in enumerate(trees):
        arr[i] = t.handle.value
    out = np.zeros(len(trees))
    _check(lib.gems_tree_compute_likelihood_batch(arr, len(trees), _dptr(out)),
           "gems_tree_compute_likelihood_batch")
    return out


def evaluate_rates_batch(trees, rates, props=None):
    """Every candidate at new category rates (a new Gamma shape: RateGamma::computeFunction,
    model/rategamma.cpp:178-186, once per candidate): gems_set_rates on each tree's session,
    every partial cleared, then one batched evaluation.  rates[i] (and props[i], default equal
    proportions) are tree i's; returns their lnL."""
    for i, t in enumerate(trees):
        r = _f64(rates[i])
        p = np.full(len(r), 1.0 / len(r)) if props is None else _f64(props[i])
        t.session.set_rates(r, p)
        t.clearAllPartialLH()
    return compute_likelihood_batch(trees)


def _session_array(sessions):
    arr = (c_void_p * len(sessions))()
    for i, s in enumerate(sessions):
        arr[i] = s.handle.value
    return arr


def traverse_batch(sessions, ops):
    """One batched traversal over sessions that share the tree (gems_traverse_batch)."""
    arr, n = op_array(ops)
    lib = sessions[0].lib
    _check(lib.gems_traverse_batch(_session_array(sessions), len(sessions), arr, n),
           "gems_traverse_batch")


def branch_lnl_batch(sessions, ops, br):
    """Batched traversal, then each session's branch lnL (gems_branch_lnl_batch)."""
    arr, n = op_array(ops)
    lib = sessions[0].lib
    out = np.zeros(len(sessions))
    _check(lib.gems_branch_lnl_batch(_session_array(sessions), len(sessions), arr, n, byref(br),
                                     _dptr(out)), "gems_branch_lnl_batch")
    return out


class Session:
    """A device session: tips, pattern weights, model and partial slots resident in HBM."""

    def __init__(self, ntaxa, nptn, nstates, ncat, nslots, precision="fp64", scaling="norm",
                 device=0):
        self.lib = _lib.gems()
        self.desc = SessionDesc(ntaxa, nptn, nstates, ncat, nslots, PREC[precision],
                                SCALING[scaling], device)
        self.handle = c_void_p()
        _check(self.lib.gems_session_create(byref(self.desc), byref(self.handle)),
               "gems_session_create")
        self.ntaxa, self.nptn, self.nstates, self.ncat = ntaxa, nptn, nstates, ncat
        self.block = nstates * ncat
        self.safe = scaling == "safe"

    @staticmethod
    def footprint(ntaxa, nptn, nstates, ncat, nslots, precision="fp64", scaling="norm"):
        d = SessionDesc(ntaxa, nptn, nstates, ncat, nslots, PREC[precision], SCALING[scaling], 0)
        out = c_size_t()
        _check(_lib.gems().gems_session_footprint(byref(d), byref(out)), "footprint")
        return out.value

    def close(self):
        if self.handle:
            self.lib.gems_session_destroy(self.handle)
            self.handle = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_tips(self, states):
        st = np.ascontiguousarray(states, dtype=np.uint8)
        assert st.shape == (self.ntaxa, self.nptn)
        _check(self.lib.gems_upload_tips(self.handle, _dptr(st)), "gems_upload_tips")

    def upload_patterns(self, freq, invar=None):
        f = _f64(freq)
        iv = None if invar is None else _f64(invar)
        _check(self.lib.gems_upload_patterns(self.handle, _dptr(f), _dptr(iv)),
               "gems_upload_patterns")

    def set_model(self, eval_, evec, inv_evec, rates, props):
        arrs = [_f64(x) for x in (eval_, evec, inv_evec, rates, props)]
        _check(self.lib.gems_set_model(self.handle, *[_dptr(a) for a in arrs]), "gems_set_model")

    def set_model_from_rates(self, exch_upper, freq, rates, props):
        arrs = [_f64(x) for x in (exch_upper, freq, rates, props)]
        _check(self.lib.gems_set_model_from_rates(self.handle, *[_dptr(a) for a in arrs]),
               "gems_set_model_from_rates")

    def eigensystem(self):
        n = self.nstates
        ev, v, iv = np.zeros(n), np.zeros((n, n)), np.zeros((n, n))
        _check(self.lib.gems_get_eigensystem(self.handle, _dptr(ev), _dptr(v), _dptr(iv)),
               "gems_get_eigensystem")
        return ev, v, iv

    def traverse(self, ops):
        arr, n = op_array(ops)
        _check(self.lib.gems_traverse(self.handle, arr, n), "gems_traverse")

    def compute_partial(self, op, ptn_lower, ptn_upper):
        """One node update over patterns [ptn_lower, ptn_upper) (computePartialLikelihood of
        one TraversalInfo entry for one packet); op = (dst, lkind, lid, rkind, rid, llen, rlen)."""
        arr, _ = op_array([op])
        _check(self.lib.gems_compute_partial(self.handle, arr, int(ptn_lower), int(ptn_upper)),
               "gems_compute_partial")

    def pattern_granule(self):
        """Alignment that the pattern ranges of compute_partial must respect."""
        g = c_int()
        _check(self.lib.gems_session_pattern_granule(self.handle, byref(g)),
               "gems_session_pattern_granule")
        return g.value

    def branch_lnl(self, ops, br, pattern_lh=False):
        arr, n = op_array(ops)
        out = c_double()
        plh = np.zeros(self.nptn) if pattern_lh else None
        _check(self.lib.gems_branch_lnl(self.handle, arr, n, byref(br), byref(out), _dptr(plh)),
               "gems_branch_lnl")
        return (out.value, plh) if pattern_lh else out.value

    def branch_derv(self, ops, br, compute_theta=True, df_frac=False):
        arr, n = op_array(ops)
        df, ddf = c_double(), c_double()
        g = np.zeros(self.nptn) if df_frac else None
        _check(self.lib.gems_branch_derv(self.handle, arr, n, byref(br), int(compute_theta),
                                         byref(df), byref(ddf), _dptr(g)), "gems_branch_derv")
        return (df.value, ddf.value, g) if df_frac else (df.value, ddf.value)

    def lnl_from_buffer(self, length, pattern_lh=False):
        out = c_double()
        plh = np.zeros(self.nptn) if pattern_lh else None
        _check(self.lib.gems_lnl_from_buffer(self.handle, c_double(length), byref(out),
                                             _dptr(plh)), "gems_lnl_from_buffer")
        return (out.value, plh) if pattern_lh else out.value

    def newton_branch(self, ops, br, compute_theta, min_len, max_len, xacc, max_steps):
        arr, n = op_array(ops)
        opt, nev = c_double(), c_int()
        _check(self.lib.gems_newton_branch(self.handle, arr, n, byref(br), int(compute_theta),
                                           c_double(min_len), c_double(max_len), c_double(xacc),
                                           max_steps, byref(opt), byref(nev)),
               "gems_newton_branch")
        return opt.value, nev.value

    def get_partial(self, slot):
        part = np.zeros((self.nptn, self.ncat, self.nstates))
        per = self.ncat if self.safe else 1
        sc = np.zeros(self.nptn * per, np.uint16)
        _check(self.lib.gems_get_partial(self.handle, slot, _dptr(part), _dptr(sc)),
               "gems_get_partial")
        return part, (sc.reshape(self.nptn, per) if self.safe else sc)

    def get_theta(self):
        th = np.zeros((self.nptn, self.block))
        sa = np.zeros(self.nptn)
        _check(self.lib.gems_get_theta(self.handle, _dptr(th), _dptr(sa)), "gems_get_theta")
        return th, sa

    def launch_count(self):
        n = c_longlong()
        _check(self.lib.gems_launch_count(self.handle, byref(n)), "gems_launch_count")
        return n.value

    def upload_reweightings(self, weights):
        """weights: [R][nptn] pattern counts of R bootstrap replicates (kept in HBM)."""
        w = np.ascontiguousarray(weights, dtype=np.float32)
        assert w.ndim == 2 and w.shape[1] == self.nptn
        _check(self.lib.gems_upload_reweightings(self.handle, _dptr(w), w.shape[0]),
               "gems_upload_reweightings")
        self.rell_R = w.shape[0]

    def reweighted_lnl(self):
        out = np.zeros(self.rell_R)
        _check(self.lib.gems_reweighted_lnl(self.handle, _dptr(out)), "gems_reweighted_lnl")
        return out

    def reweighted_derv(self):
        df, ddf = np.zeros(self.rell_R), np.zeros(self.rell_R)
        _check(self.lib.gems_reweighted_derv(self.handle, _dptr(df), _dptr(ddf)),
               "gems_reweighted_derv")
        return df, ddf

    def set_rates(self, rates, props):
        """New category rates and proportions, eigensystem kept (gems_set_rates); partials
        computed before are stale."""
        r, p = _f64(rates), _f64(props)
        _check(self.lib.gems_set_rates(self.handle, _dptr(r), _dptr(p)), "gems_set_rates")

    def set_tensor_cores(self, on=True):
        """20-state mixed traversal on tcgen05 split-TF32 products (default) or FP32 CUDA
        cores."""
        _check(self.lib.gems_session_set_option(self.handle, 1, int(on)), "set_option")

    def set_tc20_halves(self, on=True):
        """20-state tcgen05 traversal at two CTAs per SM in half-steps (GEMS_OPT_TC20_HALVES);
        same values bit for bit."""
        _check(self.lib.gems_session_set_option(self.handle, 5, int(on)), "set_option")

    def set_tc61_roles(self, on=True):
        """61-state tcgen05 traversal with split / MMA / epilogue warp roles on consecutive steps
        (GEMS_OPT_TC61_ROLES, default) or every warp running the parts in turn; same values bit
        for bit."""
        _check(self.lib.gems_session_set_option(self.handle, 6, int(on)), "set_option")

    def set_newton_share(self, k):
        """The device Newton kernel takes at most 1/k of the GPU (GEMS_OPT_NEWTON_SHARE)."""
        _check(self.lib.gems_session_set_option(self.handle, 4, int(k)), "set_option")

    def set_autotune(self, on=True, force_shape=None):
        """Tune the 4-state traversal's launch shape on its first large traversal (default), or
        force shape k of the kernel's list (comparisons)."""
        v = 2 + int(force_shape) if force_shape is not None else int(on)
        _check(self.lib.gems_session_set_option(self.handle, 3, v), "set_option")

    def traversal_shape(self):
        """(patterns per lane group, blocks per SM, tuned) of the 4-state traversal in use."""
        a, b, t = c_int(), c_int(), c_int()
        _check(self.lib.gems_session_traversal_shape(self.handle, byref(a), byref(b), byref(t)),
               "traversal_shape")
        return a.value, b.value, bool(t.value)

    def set_tiled_fp64(self, on=True):
        """61-state FP64 traversal as register-tiled GEMMs (default) or the per-row kernel."""
        _check(self.lib.gems_session_set_option(self.handle, 2, int(on)), "set_option")

    def stream_handle(self):
        p = c_void_p()
        _check(self.lib.gems_session_stream(self.handle, byref(p)), "gems_session_stream")
        return p.value or 0

    def profile(self, on=True):
        _check(self.lib.gems_profile_enable(self.handle, int(on)), "gems_profile_enable")

    def profile_read(self, kernel_id):
        """(total_ms, launches) of kernel_id (0 traverse, 1 branch, 2 theta, 3 derv,
        4 from-buffer, 5 newton) since the last read."""
        ms, n = c_double(), c_longlong()
        _check(self.lib.gems_profile_read(self.handle, kernel_id, byref(ms), byref(n)),
               "gems_profile_read")
        return ms.value, n.value

    def sync(self):
        _check(self.lib.gems_session_sync(self.handle), "gems_session_sync")


class PhyloTree:
    """PhyloTree calls of the likelihood path on a device session (C++ mirror in
    csrc/phylotree.cpp)."""

    def __init__(self, session: Session, eu, ev, lengths):
        self.session = session
        self.lib = session.lib
        # own copies: doNNI rewrites them in place
        self.eu = np.array(eu, np.int32)
        self.ev = np.array(ev, np.int32)
        ln = _f64(lengths)
        self.handle = c_void_p()
        _check(self.lib.gems_tree_create(session.handle, len(self.eu), _dptr(self.eu),
                                         _dptr(self.ev), _dptr(ln), byref(self.handle)),
               "gems_tree_create")

    @classmethod
    def from_case(cls, tree, model, aln, precision="fp64", scaling="norm", device=0,
                  slots="node", invar=None):
        """Session + tree for a synthetic case (synth.Tree, synth.Model, synth.Alignment).
        slots: "node" (one partial per internal node, LM_PER_NODE), "node+spare" (the same
        with two spare slots for evaluateNNI, the reference's nni_partial_lh), "branch" (one
        per directed branch), "pool" (LM_MEM_SAVE at its floor, log2(ntaxa) + 1 slots) or a
        slot count."""
        nint = tree.ntaxa - 2
        if isinstance(slots, int):
            nslots = slots
        else:
            nslots = {"node": nint, "node+spare": nint + 2, "branch": 3 * nint,
                      "pool": min_pool_slots(tree.ntaxa)}[slots]
        s = Session(tree.ntaxa, aln.npat, model.nstates, model.ncat, nslots, precision,
                    scaling, device)
        s.upload_tips(aln.patterns)
        s.upload_patterns(aln.weights, invar)
        s.set_model(model.eval, model.evec, model.inv_evec, model.rates, model.props)
        return cls(s, tree.eu, tree.ev, tree.length)

    def close(self):
        if self.handle:
            self.lib.gems_tree_destroy(self.handle)
            self.handle = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference API names --
    def setBranchLimits(self, min_len, max_len):
        _check(self.lib.gems_tree_set_branch_limits(self.handle, c_double(min_len),
                                                    c_double(max_len)), "set_branch_limits")

    def setLength(self, u, v, x):
        _check(self.lib.gems_tree_set_length(self.handle, u, v, c_double(x)), "set_length")

    def getBranchLengths(self):
        out = np.zeros(len(self.eu))
        _check(self.lib.gems_tree_get_lengths(self.handle, _dptr(out)), "get_lengths")
        return out

    def clearAllPartialLH(self):
        _check(self.lib.gems_tree_clear_all_partial_lh(self.handle), "clearAllPartialLH")

    def computeLikelihood(self, pattern_lh=False):
        out = c_double()
        plh = np.zeros(self.session.nptn) if pattern_lh else None
        _check(self.lib.gems_tree_compute_likelihood(self.handle, byref(out), _dptr(plh)),
               "computeLikelihood")
        return (out.value, plh) if pattern_lh else out.value

    def computeLikelihoodFromHost(self, states, ptn_freq, ptn_invar=None, chunks=16,
                                  pattern_lh=False):
        """computeLikelihood on new tip states [ntaxa][nptn], pattern weights and +I terms:
        the tip upload overlaps the traversal in up to `chunks` pattern chunks (pinned host
        arrays needed for the overlap).  pattern_lh: False, True, or a float64 array [nptn]
        to fill (pinned for the fastest copy)."""
        st = np.ascontiguousarray(states, dtype=np.uint8)
        assert st.shape == (self.session.ntaxa, self.session.nptn)
        f = _f64(ptn_freq)
        iv = None if ptn_invar is None else _f64(ptn_invar)
        out = c_double()
        if isinstance(pattern_lh, np.ndarray):
            assert pattern_lh.dtype == np.float64 and pattern_lh.shape == (self.session.nptn,)
            assert pattern_lh.flags.c_contiguous
            plh = pattern_lh
        else:
            plh = np.zeros(self.session.nptn) if pattern_lh else None
        _check(self.lib.gems_tree_compute_likelihood_from_host(
            self.handle, _dptr(st), _dptr(f), _dptr(iv), int(chunks), byref(out), _dptr(plh)),
            "computeLikelihoodFromHost")
        return (out.value, plh) if plh is not None else out.value

    def computeLikelihoodBranch(self, node, dad, pattern_lh=False):
        out = c_double()
        plh = np.zeros(self.session.nptn) if pattern_lh else None
        _check(self.lib.gems_tree_compute_likelihood_branch(self.handle, node, dad, byref(out),
                                                            _dptr(plh)),
               "computeLikelihoodBranch")
        return (out.value, plh) if pattern_lh else out.value

    def computeLikelihoodDerv(self, node, dad):
        df, ddf = c_double(), c_double()
        _check(self.lib.gems_tree_compute_likelihood_derv(self.handle, node, dad, byref(df),
                                                          byref(ddf)), "computeLikelihoodDerv")
        return df.value, ddf.value

    def computeLikelihoodFromBuffer(self):
        out = c_double()
        _check(self.lib.gems_tree_compute_likelihood_from_buffer(self.handle, byref(out)),
               "computeLikelihoodFromBuffer")
        return out.value

    def optimizeOneBranch(self, node1, node2, clearLH=True, maxNRStep=100):
        _check(self.lib.gems_tree_optimize_one_branch(self.handle, node1, node2, int(clearLH),
                                                      maxNRStep), "optimizeOneBranch")

    def optimizeAllBranches(self, my_iterations=100, tolerance=0.001, maxNRStep=100):
        out = c_double()
        _check(self.lib.gems_tree_optimize_all_branches(self.handle, my_iterations,
                                                        c_double(tolerance), maxNRStep,
                                                        byref(out)), "optimizeAllBranches")
        return out.value

    def getBranchLength(self, u, v):
        i = np.nonzero(((self.eu == u) & (self.ev == v)) | ((self.eu == v) & (self.ev == u)))[0]
        if len(i) == 0:
            raise KeyError((u, v))
        return float(self.getBranchLengths()[i[0]])

    def evaluateNNI(self, u, v, maxNRStep=10):
        """getBestNNIForBran's evaluation of the internal branch (u, v), the tree unchanged
        (gems_tree_nni_evaluate): [(a, b, lnl, lengths[5])] for the two NNIs, lengths =
        central, u's outer two, v's outer two."""
        moves = np.zeros(4, np.int32)
        lnl = np.zeros(2)
        lens = np.zeros(10)
        _check(self.lib.gems_tree_nni_evaluate(self.handle, u, v, int(maxNRStep), _dptr(moves),
                                               _dptr(lnl), _dptr(lens)), "evaluateNNI")
        return [(int(moves[2 * c]), int(moves[2 * c + 1]), float(lnl[c]), lens[5 * c:5 * c + 5])
                for c in range(2)]

    def doNNI(self, u, v, a, b):
        """Swap subtree a (at u) with subtree b (at v) across the internal branch (u, v)."""
        _check(self.lib.gems_tree_nni(self.handle, u, v, a, b), "doNNI")
        _check(self.lib.gems_tree_get_edges(self.handle, _dptr(self.eu), _dptr(self.ev)),
               "get_edges")

    def doSPR(self, node, dad, node2, dad2):
        """Prune the subtree at node from the internal node dad and regraft dad into the branch
        (node2, dad2) (gems_tree_spr: assessSPRMove's move, tree/phylotree.cpp:4822)."""
        _check(self.lib.gems_tree_spr(self.handle, node, dad, node2, dad2), "doSPR")
        _check(self.lib.gems_tree_get_edges(self.handle, _dptr(self.eu), _dptr(self.ev)),
               "get_edges")

    def neighbors(self, u):
        """Nodes adjacent to u, in edge order."""
        i = np.nonzero((self.eu == u) | (self.ev == u))[0]
        return np.where(self.eu[i] == u, self.ev[i], self.eu[i]).tolist()

    def computeFuncDerv(self, node1, node2, value, new_branch=False):
        f, df = c_double(), c_double()
        _check(self.lib.gems_tree_compute_func_derv(self.handle, node1, node2, c_double(value),
                                                    int(new_branch), byref(f), byref(df)),
               "computeFuncDerv")
        return f.value, df.value

    def getPartial(self, node, dad):
        s = self.session
        part = np.zeros((s.nptn, s.ncat, s.nstates))
        per = s.ncat if s.safe else 1
        sc = np.zeros(s.nptn * per, np.uint16)
        _check(self.lib.gems_tree_get_partial(self.handle, node, dad, _dptr(part), _dptr(sc)),
               "getPartial")
        return part, (sc.reshape(s.nptn, per) if s.safe else sc)

    def stats(self):
        ops, nev = c_longlong(), c_int()
        _check(self.lib.gems_tree_stats(self.handle, byref(ops), byref(nev)), "stats")
        return ops.value, nev.value
