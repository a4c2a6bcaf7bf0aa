"""The serving loop's scheduler on the CPU: sessions are oracle trees in the place of device
sessions, so admission by footprint, continuous batching over worker threads, eviction of idle
sessions and their rebuild from saved trees run without a GPU.  Every session's results must be
the same as running it alone, and a session that can never fit must have its requests
rejected."""
import types

import numpy as np

from gems_b200 import serve
from oracle import oracle as orc


class OracleSession:
    """An oracle tree in the role of a session's tree object (same method names)."""

    def __init__(self, spec, case, device=0, tree=None, nslots=None):
        t0, model, aln = case
        self.t = orc.OracleTree(tree if tree is not None else t0, model, aln,
                                safe=spec.nstates == 61)
        self.session = types.SimpleNamespace(close=lambda: None)

    def __getattr__(self, name):
        return getattr(self.t, name)

    def close(self):
        pass


def stream(nsess, nreq, seed, rate=5000.0):
    specs, reqs = serve.make_stream(nsess, nreq, rate=rate, seed=seed, taxa=(6, 14),
                                    sites=(60, 300), states=(4, 20), cats=(1, 4))
    cases = {s.sid: serve.build_case(s) for s in specs}
    return specs, reqs, cases


def same_as_alone(specs, cases, records):
    by_sid = {}
    for r in records:
        by_sid.setdefault(r["sid"], []).append(r)
    for sid, rs in by_sid.items():
        rs.sort(key=lambda r: r["seq"])
        alone = serve.run_alone(specs[sid], cases[sid], len(rs), opener=OracleSession)
        assert [r["lnl"] for r in rs] == alone, sid


def test_admission_batching_and_eviction_keep_results():
    # arrivals spread out, so that sessions sit idle with requests still to come
    specs, reqs, cases = stream(5, 40, seed=8, rate=300.0)
    fps = sorted(s.footprint(cases[s.sid][2].npat) for s in specs)
    srv = serve.Server(budget_bytes=fps[-1] + fps[0], workers=3, opener=OracleSession,
                       memsave=False)
    records, _ = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") and not r.get("error") for r in records)
    assert srv.evictions > 0
    same_as_alone(specs, cases, records)


def test_memsave_admits_pools_before_evicting():
    """With LM_MEM_SAVE pools, sessions that do not fit at full size are admitted with fewer
    slots instead of waiting for evictions; results are unchanged."""
    specs, reqs, cases = stream(5, 40, seed=8, rate=300.0)
    fps = sorted(s.footprint(cases[s.sid][2].npat) for s in specs)
    srv = serve.Server(budget_bytes=fps[-1] + fps[0], workers=3, opener=OracleSession)
    records, _ = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") and not r.get("error") for r in records)
    assert srv.pool_admissions > 0
    same_as_alone(specs, cases, records)


def test_memsave_admits_a_session_only_its_pool_fits():
    """A budget below a session's full footprint but above its smallest pool: admitted as a
    pool (no rejection), results unchanged; below the pool: rejected."""
    specs, reqs, cases = stream(4, 24, seed=9)
    fps = {s.sid: s.footprint(cases[s.sid][2].npat) for s in specs}
    big = max(fps, key=fps.get)
    sp = specs[big]
    floor = sp.footprint(cases[big][2].npat, serve.min_pool_slots(sp.ntaxa))
    assert floor < fps[big]
    srv = serve.Server(budget_bytes=fps[big] - 1, workers=2, opener=OracleSession)
    records, _ = srv.run(specs, cases, reqs)
    assert not any(r.get("rejected") for r in records)
    assert srv.pool_admissions > 0
    same_as_alone(specs, cases, records)
    srv = serve.Server(budget_bytes=floor - 1, workers=2, opener=OracleSession)
    records, _ = srv.run(specs, cases, reqs)
    assert all(r.get("rejected") for r, (_, sid) in zip(records, reqs) if sid == big)


def test_session_that_cannot_fit_is_rejected():
    specs, reqs, cases = stream(4, 24, seed=9)
    fps = {s.sid: s.footprint(cases[s.sid][2].npat) for s in specs}
    budget = sorted(fps.values())[-1] - 1
    srv = serve.Server(budget_bytes=budget, workers=2, opener=OracleSession, memsave=False)
    records, _ = srv.run(specs, cases, reqs)
    for r, (_, sid) in zip(records, reqs):
        assert bool(r.get("rejected")) == (fps[sid] > budget)
    same_as_alone(specs, cases, [r for r in records if not r.get("rejected")])


class CountingSession(OracleSession):
    """OracleSession that records when it was closed and whether requests were still running."""
    log = []

    def __init__(self, spec, case, device=0, tree=None, nslots=None):
        super().__init__(spec, case, device, tree, nslots)
        self.sid = spec.sid
        self.session = types.SimpleNamespace(close=lambda: None)

    def close(self):
        CountingSession.log.append(self.sid)


def test_finished_sessions_stay_resident_until_the_stream_ends():
    """With room for every session, none is closed while the stream runs (closing frees device
    memory, which synchronises the GPU): every close comes after the last request."""
    specs, reqs, cases = stream(5, 30, seed=12, rate=2000.0)
    CountingSession.log = []
    srv = serve.Server(budget_bytes=1 << 60, workers=3, opener=CountingSession)
    done_before = []
    orig = serve.tree_move

    def move(gt, ntaxa, rng):
        done_before.append(len(CountingSession.log))
        return orig(gt, ntaxa, rng)

    serve.tree_move = move
    try:
        records, _ = srv.run(specs, cases, reqs)
    finally:
        serve.tree_move = orig
    assert all(r is not None and not r.get("error") for r in records)
    assert max(done_before) == 0            # nothing was closed while requests ran
    assert sorted(CountingSession.log) == sorted({sid for _, sid in reqs})
    assert srv.evictions == 0
    same_as_alone(specs, cases, records)


def test_finished_sessions_released_before_idle_ones_are_evicted():
    """A budget for about two sessions: finished sessions make room first, so fewer idle
    sessions (with requests still to come) are evicted than sessions are admitted late; results
    are unchanged."""
    specs, reqs, cases = stream(6, 36, seed=13, rate=400.0)
    fps = sorted(s.footprint(cases[s.sid][2].npat) for s in specs)
    CountingSession.log = []
    srv = serve.Server(budget_bytes=fps[-1] + fps[-2], workers=2, opener=CountingSession,
                       memsave=False)
    records, _ = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") and not r.get("error") for r in records)
    same_as_alone(specs, cases, records)
    # every close of a session with requests still to come is an eviction; the others were
    # finished sessions released for room or at the end
    assert len(CountingSession.log) >= len({sid for _, sid in reqs})
    assert srv.evictions == len(CountingSession.log) - len({sid for _, sid in reqs})
