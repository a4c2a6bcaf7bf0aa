"""Serving loop: many tree-search sessions resident in HBM, requests batched continuously.

A session is one alignment + model + tree kept on the GPU (its partials, scale counters,
theta and tip bytes).  A request is a local tree move as tree search issues them, then the
tree log-likelihood:
  * an NNI on an internal branch (tree/phylotree.cpp:4059 doNNI), then Newton optimisation of
    the five branches around it (the central one and its four neighbours, as the NNI-5
    evaluation of getBestNNIForBran does, tree/phylotree.cpp:4176);
  * or an SPR: a subtree pruned and regrafted within a radius (tree/phylotree.cpp:4822
    assessSPRMove's move), then Newton on the four branches swapSPR optimises
    (tree/phylotree.cpp:4764-4768).
Only the partials on the affected paths are recomputed.

Scheduling:
  * admission by HBM footprint: a session is created on the GPU when its footprint
    (gems_session_footprint) fits the remaining budget.  A session whose last request has
    finished stays resident until admission needs its memory or the stream ends: freeing
    device memory synchronises the whole GPU, so closing it at once stalls every other
    session's requests.  Admission plans with that memory as free and releases finished
    sessions first.  When the session at the head of the admission queue still does not fit,
    idle sessions (no request running or queued) are evicted,
    least recently used first: the evolved tree (topology and branch lengths) is kept on the
    host and the session is rebuilt from it at its next request -- partials are a function of
    the tree, so its results are the same as if it had stayed;
  * continuous batching: requests arrive over time (Poisson); a pool of worker threads takes
    the oldest runnable request of any admitted session whose previous request has finished.
    Each session has its own CUDA stream and the C-ABI calls release the GIL, so the work of
    different sessions overlaps on the device;
  * per-session order is the arrival order, so a session's results do not depend on what else
    runs (tests/test_gpu_serve.py checks this against each session run alone).

    python -m gems_b200.serve --sessions 48 --requests 1000 --rate 300
"""
from __future__ import annotations

import argparse
import collections
import dataclasses
import json
import threading
import time
import types

import numpy as np

from . import synth
from .api import GemsError, PhyloTree, Session, min_pool_slots


@dataclasses.dataclass
class SessionSpec:
    sid: int
    ntaxa: int
    nsites: int
    nstates: int
    ncat: int
    precision: str
    seed: int

    def footprint(self, npat, nslots=None):
        """Device bytes of the session with `nslots` partial slots (default: one per internal
        node, LM_PER_NODE)."""
        nslots = self.ntaxa - 2 if nslots is None else nslots
        scaling = "safe" if self.nstates == 61 else "norm"
        return Session.footprint(self.ntaxa, npat, self.nstates, self.ncat, nslots,
                                 self.precision, scaling)

    def slot_plan(self, npat, avail, memsave=True):
        """(nslots, bytes) of the largest session that fits `avail` bytes: one slot per internal
        node when it fits, else (memsave) the most slots of the LM_MEM_SAVE pool that fit, down
        to its floor; None when nothing fits."""
        full = self.footprint(npat)
        if full <= avail:
            return None, full
        if not memsave:
            return None
        lo = min_pool_slots(self.ntaxa)
        base = self.footprint(npat, lo)
        per = self.footprint(npat, lo + 1) - base
        if base > avail:
            return None
        n = min(self.ntaxa - 3, lo + (avail - base) // max(per, 1))
        return int(n), base + (int(n) - lo) * per


def build_case(spec: SessionSpec):
    rng = np.random.default_rng(spec.seed)
    if spec.nstates == 4:
        model = synth.dna_gtr(rng, spec.ncat, 0.5)
    elif spec.nstates == 20:
        model = synth.protein(rng, spec.ncat, 0.8)
    else:
        model = synth.codon_gy(rng, spec.ncat, 0.5, freerate=spec.ncat == 8)
    tree = synth.random_tree(spec.ntaxa, 0.1, spec.seed + 1)
    aln = synth.simulate(tree, model, spec.nsites, spec.seed + 2)
    return tree, model, aln


def open_session(spec, case, device=0, tree=None, nslots=None):
    """The session of a case, on the case's tree or on `tree` (an evicted session's), with one
    partial slot per internal node or `nslots` (an LM_MEM_SAVE pool)."""
    t0, model, aln = case
    gt = PhyloTree.from_case(tree if tree is not None else t0, model, aln,
                             precision=spec.precision,
                             scaling="safe" if spec.nstates == 61 else "norm", device=device,
                             slots="node" if nslots is None else int(nslots))
    # many sessions share the GPU: a Newton loop takes at most a quarter of it, so that it runs
    # beside the others' work instead of waiting for the whole device
    gt.session.set_newton_share(4)
    return gt


def saved_tree(gt: PhyloTree, ntaxa: int):
    """Topology and branch lengths of a session's tree, to rebuild it after an eviction."""
    return types.SimpleNamespace(ntaxa=ntaxa, eu=gt.eu.copy(), ev=gt.ev.copy(),
                                 length=gt.getBranchLengths())


def nni5(gt: PhyloTree, ntaxa: int, rng: np.random.Generator):
    """One request: a random NNI on an internal branch, Newton on the 5 branches around it,
    then lnL.  Returns (lnL, branches optimised)."""
    mask = (gt.eu >= ntaxa) & (gt.ev >= ntaxa)
    internal = list(zip(gt.eu[mask].tolist(), gt.ev[mask].tolist()))
    u, v = internal[int(rng.integers(len(internal)))]
    nu = [x for x in gt.neighbors(u) if x != v]
    nv = [x for x in gt.neighbors(v) if x != u]
    a, b = nu[int(rng.integers(2))], nv[int(rng.integers(2))]
    gt.doNNI(u, v, a, b)
    branches = [(u, v)] + [(u, x) for x in gt.neighbors(u) if x != v] + \
               [(v, y) for y in gt.neighbors(v) if y != u]
    for p, q in branches:
        gt.optimizeOneBranch(p, q)
    return gt.computeLikelihoodFromBuffer(), len(branches)


SPR_RADIUS = 3      # regraft branches at most this many branches from the pruned joint
SPR_SHARE = 0.3     # share of requests that are SPR moves (the rest are NNI)


def _adjacency(gt):
    """Every node's neighbours in edge order (the order gt.neighbors returns them in), built in
    one pass over the edge list."""
    adj = collections.defaultdict(list)
    for a, b in zip(gt.eu.tolist(), gt.ev.tolist()):
        adj[a].append(b)
        adj[b].append(a)
    return adj


def spr_regraft_branches(gt, node, dad, radius=SPR_RADIUS, adj=None):
    """Branches (x, y) the subtree at node (pruned from dad) can be regrafted into: those of the
    remaining tree within `radius` branches of the joint that pruning leaves (dad's two other
    neighbours s1, s2, joined), the joint itself excluded (regrafting there is no move).  The
    search walks outwards from s1 and s2, as swapSPR does up to its radius
    (tree/phylotree.cpp:4694-4820)."""
    adj = _adjacency(gt) if adj is None else adj
    s1, s2 = sorted(x for x in adj[dad] if x != node)
    out, frontier = [], [(s1, dad), (s2, dad)]
    for _ in range(radius):
        nxt = []
        for x, back in frontier:
            for y in adj[x]:
                if y == back or y == dad:
                    continue
                out.append((y, x))
                nxt.append((y, x))
        frontier = nxt
    return s1, s2, out


def spr4(gt, ntaxa: int, rng: np.random.Generator, radius=SPR_RADIUS):
    """One SPR request: the subtree at a random neighbour of a random internal node pruned and
    regrafted into a branch within `radius` (assessSPRMove's move,
    tree/phylotree.cpp:4822-4880), Newton on the four branches swapSPR optimises after a move
    (the pruned subtree's branch, the two halves of the regraft branch and the joined branch,
    tree/phylotree.cpp:4764-4768), then the lnL from the buffers.  Returns (lnL, branches
    optimised)."""
    adj = _adjacency(gt)
    internal = sorted(u for u, nb in adj.items() if len(nb) == 3)
    for _ in range(16):
        dad = internal[int(rng.integers(len(internal)))]
        node = adj[dad][int(rng.integers(3))]
        s1, s2, cand = spr_regraft_branches(gt, node, dad, radius, adj)
        if cand:
            break
    else:
        return nni5(gt, ntaxa, rng)
    node2, dad2 = cand[int(rng.integers(len(cand)))]
    gt.doSPR(node, dad, node2, dad2)
    branches = [(node, dad), (dad2, dad), (node2, dad), (s1, s2)]
    for p, q in branches:
        gt.optimizeOneBranch(p, q)
    return gt.computeLikelihoodFromBuffer(), len(branches)


def tree_move(gt, ntaxa: int, rng: np.random.Generator):
    """One serving request: an SPR (share SPR_SHARE) or an NNI, drawn from the request's own
    seeded generator, so a session's results do not depend on scheduling."""
    if rng.random() < SPR_SHARE:
        return spr4(gt, ntaxa, rng)
    return nni5(gt, ntaxa, rng)


def run_alone(spec, case, nreq, device=0, opener=open_session):
    """The session's requests in order, nothing else on the GPU."""
    gt = opener(spec, case, device)
    gt.computeLikelihood()
    out = []
    for k in range(nreq):
        out.append(tree_move(gt, spec.ntaxa, np.random.default_rng((spec.seed, k)))[0])
    gt.close()
    gt.session.close()
    return out


class Server:
    def __init__(self, device=0, budget_bytes=None, workers=8, evict=True, opener=open_session,
                 memsave=True):
        """opener(spec, case, device, tree[, nslots]) builds a session's tree object
        (open_session: a PhyloTree on the GPU); budget_bytes defaults to 85% of the device's
        free memory.  With memsave, a session that does not fit with one partial slot per
        internal node is admitted with the largest LM_MEM_SAVE pool that fits the free budget
        (its evicted partials are recomputed when needed) before any idle session is evicted;
        only a session whose smallest pool cannot fit waits for evictions."""
        if budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            budget_bytes = int(0.85 * free)
        self.device = device
        self.budget = int(budget_bytes)
        self.workers = workers
        self.evict = evict
        self.opener = opener
        self.memsave = memsave

    def run(self, specs, cases, requests, preopen=False):
        """requests: list of (arrival_s, sid) in arrival order, arrival times counted from the
        start of the request stream.  A session opens when its first request arrives; with
        `preopen`, the sessions that fit the budget are opened (in first-arrival order) before
        the stream starts, as a server does with the datasets it holds.  Session open times are
        kept in self.open_ms.  Returns the per-request records and the stream's wall time."""
        lock = threading.Condition()
        npat = {s.sid: cases[s.sid][2].npat for s in specs}
        spec_of = {s.sid: s for s in specs}
        # bytes a session holds once admitted (its plan), and the least it can be admitted with
        fp = {s.sid: s.footprint(npat[s.sid]) for s in specs}
        fp_min = {s.sid: (s.slot_plan(npat[s.sid], 1 << 62, False)[1] if not self.memsave else
                          s.footprint(npat[s.sid], min_pool_slots(s.ntaxa)))
                  for s in specs}
        nslots_of = {}   # sid -> slots of an admitted pool session (absent: one per node)
        self.pool_admissions = 0
        remaining = collections.Counter(sid for _, sid in requests)
        pending = collections.defaultdict(collections.deque)  # sid -> deque of (arr, idx, seq)
        seq_of = collections.Counter()
        state = {"used": 0, "next": 0, "done": 0, "rejected": set()}
        open_sess = {}   # sid -> PhyloTree
        busy = set()
        waiting_admit = collections.deque()
        records = [None] * len(requests)
        self.open_ms = []
        self.evictions = 0
        saved = {}       # sid -> tree of an evicted session
        # sessions whose last request has finished: they stay resident until admission needs
        # their memory or the stream ends -- freeing device memory synchronises the whole GPU,
        # so closing them while other sessions' requests run would stall those requests
        finished = set()
        open_fail = collections.Counter()
        last_used = {}   # sid -> end of its last request
        for sid in fp:
            if fp_min[sid] > self.budget:
                state["rejected"].add(sid)

        def plan_locked(sid, extra=0):
            """Admission plan of sid in the free budget (plus `extra` bytes about to be released):
            sets fp[sid] (and its slots)."""
            plan = spec_of[sid].slot_plan(npat[sid], self.budget - state["used"] + extra,
                                          self.memsave)
            if plan is None:
                return False
            n, b = plan
            fp[sid] = b
            if n is None:
                nslots_of.pop(sid, None)
            else:
                nslots_of[sid] = n
                self.pool_admissions += 1
            return True

        def open_one(sid):
            t = time.perf_counter()
            try:
                if sid in nslots_of:
                    gt = self.opener(spec_of[sid], cases[sid], self.device, saved.get(sid),
                                     nslots=nslots_of[sid])
                else:
                    gt = self.opener(spec_of[sid], cases[sid], self.device, saved.get(sid))
                gt.computeLikelihood()
            except GemsError:
                return None
            with lock:
                self.open_ms.append(1e3 * (time.perf_counter() - t))
            return gt

        if preopen:
            queue = collections.deque()
            for sid in dict.fromkeys(sid for _, sid in requests):
                if sid in state["rejected"]:
                    continue
                if not plan_locked(sid):
                    break
                state["used"] += fp[sid]
                queue.append(sid)

            def opener():
                while True:
                    with lock:
                        if not queue:
                            return
                        sid = queue.popleft()
                    gt = open_one(sid)
                    with lock:
                        if gt is None:
                            state["rejected"].add(sid)
                            state["used"] -= fp[sid]
                        else:
                            open_sess[sid] = gt

            openers = [threading.Thread(target=opener) for _ in range(self.workers)]
            for th in openers:
                th.start()
            for th in openers:
                th.join()
        t0 = time.perf_counter()

        def admit_locked():
            """The next waiting session to open (arrival order) and the idle sessions to evict
            first to make room for it, or (None, [])."""
            if not waiting_admit:
                return None, []
            sid = waiting_admit[0]
            victims = []
            # finished sessions hold memory nobody needs: plan as if it were free
            releasable = sum(fp[s] for s, g in open_sess.items()
                             if s in finished and not isinstance(g, str))
            if plan_locked(sid, releasable):  # fits, at full size or as a pool
                need = state["used"] + fp[sid] - self.budget
            else:  # room for its smallest admissible form, from idle sessions
                fp[sid] = fp_min[sid]
                if self.memsave:
                    nslots_of[sid] = min_pool_slots(spec_of[sid].ntaxa)
                need = state["used"] + fp[sid] - self.budget
            if need > 0:
                # finished sessions first, then (with eviction) idle ones least recently used
                # first
                idle = sorted((s not in finished, last_used.get(s, 0.0), s)
                              for s, g in open_sess.items()
                              if not isinstance(g, str) and s not in busy and not pending[s]
                              and (self.evict or s in finished))
                freed = 0
                for _, _, s in idle:
                    if freed >= need:
                        break
                    victims.append((s, open_sess.pop(s)))
                    freed += fp[s]
                if freed < need:  # not enough idle memory: put them back and wait
                    for s, g in victims:
                        open_sess[s] = g
                    return None, []
                for s, g in victims:  # their memory counts as used until they are closed
                    if s in finished:
                        continue
                    saved[s] = saved_tree(g, spec_of[s].ntaxa)  # before any reopen can read it
                    self.evictions += 1
            waiting_admit.popleft()
            state["used"] += fp[sid]
            open_sess[sid] = "opening"
            return sid, victims

        def dispatcher():
            for i, (arr, sid) in enumerate(requests):
                delay = arr - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                with lock:
                    if sid in state["rejected"]:
                        records[i] = {"sid": sid, "rejected": True}
                        state["done"] += 1
                    else:
                        pending[sid].append((arr, i, seq_of[sid]))
                        seq_of[sid] += 1
                        if sid not in open_sess and sid not in waiting_admit:
                            waiting_admit.append(sid)
                    lock.notify_all()

        def worker():
            while True:
                job = None
                to_open = None
                victims = []
                with lock:
                    while True:
                        if state["done"] >= len(requests):
                            return
                        to_open, victims = admit_locked()
                        if to_open is not None:
                            break
                        best = None
                        for sid, dq in pending.items():
                            if dq and sid not in busy and sid in open_sess and \
                                    not isinstance(open_sess[sid], str):
                                if best is None or dq[0][0] < pending[best][0][0]:
                                    best = sid
                        if best is not None:
                            job = (best, pending[best].popleft())
                            busy.add(best)
                            break
                        lock.wait(0.05)
                if to_open is not None:
                    for s, g in victims:  # evicted (tree saved): free the device memory
                        g.close()
                        g.session.close()
                        with lock:
                            state["used"] -= fp[s]
                            lock.notify_all()
                    gt = open_one(to_open)
                    with lock:
                        if gt is None and open_fail[to_open] < 3:
                            # out of memory while the budget said it fits: try again later
                            open_fail[to_open] += 1
                            state["used"] -= fp[to_open]
                            del open_sess[to_open]
                            waiting_admit.append(to_open)
                            lock.notify_all()
                            continue
                        if gt is None:
                            state["rejected"].add(to_open)
                            state["used"] -= fp[to_open]
                            del open_sess[to_open]
                            for arr, i, _ in pending.pop(to_open, []):
                                records[i] = {"sid": to_open, "rejected": True}
                                state["done"] += 1
                        else:
                            open_sess[to_open] = gt
                        lock.notify_all()
                    continue
                sid, (arr, i, seq) = job
                gt = open_sess[sid]
                ts = time.perf_counter() - t0
                try:
                    lnl, nbr = tree_move(gt, spec_of[sid].ntaxa,
                                         np.random.default_rng((spec_of[sid].seed, seq)))
                    err = None
                except GemsError as e:  # the request fails; the server carries on
                    lnl, nbr, err = None, 0, str(e)
                te = time.perf_counter() - t0
                with lock:
                    records[i] = {"sid": sid, "seq": seq, "arrival": arr, "start": ts, "end": te,
                                  "latency_ms": 1e3 * (te - arr), "lnl": lnl, "branches": nbr}
                    if err is not None:
                        records[i]["error"] = err
                        records[i]["spec"] = dataclasses.asdict(spec_of[sid])
                    busy.discard(sid)
                    last_used[sid] = te
                    state["done"] += 1
                    remaining[sid] -= 1
                    if remaining[sid] == 0:
                        finished.add(sid)
                    lock.notify_all()

        threads = [threading.Thread(target=worker) for _ in range(self.workers)]
        disp = threading.Thread(target=dispatcher)
        disp.start()
        for th in threads:
            th.start()
        disp.join()
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        for s, g in open_sess.items():  # the stream is over: release every session
            if not isinstance(g, str):
                g.close()
                g.session.close()
        return records, wall


def make_stream(nsessions, nrequests, rate, seed, taxa=(8, 1024), sites=(500, 500_000),
                states=(4, 20, 61), cats=(1, 4, 8), precisions=("fp64", "mixed")):
    """Session specs (log-uniform taxa and sites) and Poisson arrivals at `rate` requests/s
    spread uniformly over the sessions."""
    rng = np.random.default_rng(seed)
    specs = []
    for sid in range(nsessions):
        nt = int(round(np.exp(rng.uniform(np.log(taxa[0]), np.log(taxa[1])))))
        ns = int(round(np.exp(rng.uniform(np.log(sites[0]), np.log(sites[1])))))
        specs.append(SessionSpec(sid, max(nt, 8), ns, int(rng.choice(states)),
                                 int(rng.choice(cats)), str(rng.choice(precisions)),
                                 int(seed * 1000 + sid)))
    gaps = rng.exponential(1.0 / rate, nrequests)
    arr = np.cumsum(gaps)
    sids = rng.integers(nsessions, size=nrequests)
    return specs, list(zip(arr.tolist(), sids.tolist()))


def summarize(records, wall, specs, cases):
    failed = [r for r in records if r and r.get("error")]
    done = [r for r in records if r and not r.get("rejected") and not r.get("error")]
    lat = np.array([r["latency_ms"] for r in done]) if done else np.zeros(1)
    upd = 0
    for r in done:
        spec = specs[r["sid"]]
        npat = cases[r["sid"]][2].npat
        upd += npat  # at least one partial per touched branch; reported as patterns served
    return {"requests": len(records), "served": len(done), "failed": len(failed),
            "errors": sorted({f"{r['error']} {r['spec']}" for r in failed})[:5],
            "rejected": sum(1 for r in records if r and r.get("rejected")),
            "wall_s": wall, "throughput_req_s": len(done) / wall,
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p90": float(np.percentile(lat, 90)),
                           "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "patterns_served_per_s": upd / wall}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sessions", type=int, default=48)
    ap.add_argument("--requests", type=int, default=1000)
    ap.add_argument("--rate", type=float, default=300.0)
    ap.add_argument("--workers", type=int, default=16)
    ap.add_argument("--max-taxa", type=int, default=256)
    ap.add_argument("--max-sites", type=int, default=50_000)
    ap.add_argument("--seed", type=int, default=5)
    args = ap.parse_args()
    specs, reqs = make_stream(args.sessions, args.requests, args.rate, args.seed,
                              taxa=(8, args.max_taxa), sites=(500, args.max_sites))
    cases = {s.sid: build_case(s) for s in specs}
    srv = Server(workers=args.workers)
    records, wall = srv.run(specs, cases, reqs)
    out = summarize(records, wall, specs, cases)
    out.update({"sessions": args.sessions, "offered_rate_req_s": args.rate,
                "workers": args.workers, "taxa": [8, args.max_taxa],
                "sites": [500, args.max_sites], "states": [4, 20, 61], "categories": [1, 4, 8],
                "precisions": ["fp64", "mixed"]})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
