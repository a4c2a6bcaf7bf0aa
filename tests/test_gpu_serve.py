"""Serving loop: results of each session's requests are the same alone and in the mix, every
request is served, and admission by HBM footprint holds sessions back without losing
requests."""
import numpy as np
import pytest

from gems_b200 import serve

pytestmark = pytest.mark.gpu


def workload(nsess=6, nreq=30, seed=3):
    specs, reqs = serve.make_stream(nsess, nreq, rate=2000.0, seed=seed, taxa=(8, 40),
                                    sites=(500, 4000), states=(4, 20, 61), cats=(1, 4))
    cases = {s.sid: serve.build_case(s) for s in specs}
    return specs, reqs, cases


def check_same_as_alone(specs, cases, records):
    by_sid = {}
    for r in records:
        by_sid.setdefault(r["sid"], []).append(r)
    for sid, rs in by_sid.items():
        rs.sort(key=lambda r: r["seq"])
        alone = serve.run_alone(specs[sid], cases[sid], len(rs))
        mixed = [r["lnl"] for r in rs]
        # same operations in the same order on the same buffers: bit-identical
        assert mixed == alone, (sid, mixed, alone)


def test_same_alone_and_in_mix(gpu):
    specs, reqs, cases = workload()
    srv = serve.Server(workers=4)
    records, wall = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") and not r.get("error") for r in records)
    check_same_as_alone(specs, cases, records)
    s = serve.summarize(records, wall, specs, cases)
    assert s["served"] == len(reqs) and s["latency_ms"]["p99"] >= s["latency_ms"]["p50"] > 0


def test_admission_by_footprint(gpu):
    specs, reqs, cases = workload(nsess=5, nreq=25, seed=4)
    fps = sorted(s.footprint(cases[s.sid][2].npat) for s in specs)
    # room for the two largest sessions at once: the others wait for a release
    srv = serve.Server(workers=4, budget_bytes=fps[-1] + fps[-2])
    records, _ = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") for r in records)
    check_same_as_alone(specs, cases, records)
    # a budget below the largest footprint rejects exactly the sessions that cannot fit at one
    # slot per internal node (pools off) ...
    budget = fps[-1] - 1
    srv = serve.Server(workers=2, budget_bytes=budget, memsave=False)
    records, _ = srv.run(specs, cases, reqs)
    for r, (_, sid) in zip(records, reqs):
        assert r is not None
        assert bool(r.get("rejected")) == (specs[sid].footprint(cases[sid][2].npat) > budget)
    assert any(r.get("rejected") for r in records)
    # ... and with LM_MEM_SAVE pools that session is served from a pool, with the same results
    srv = serve.Server(workers=2, budget_bytes=budget)
    records, _ = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") and not r.get("error") for r in records)
    assert srv.pool_admissions > 0
    check_same_as_alone(specs, cases, records)


def test_eviction_keeps_results(gpu):
    """A budget that holds the largest session and little more: idle sessions are evicted while
    they still have requests to come, rebuilt from their saved trees, and every session's
    results stay bit-identical to running it alone.  The requests come round-robin over the
    sessions, 50 ms apart (longer than a request takes), so a session is idle between its
    requests while another one waits for room: eviction is needed whatever the sessions' speed."""
    specs, _, cases = workload(nsess=6, nreq=40, seed=6)
    sids = [s.sid for s in specs]
    reqs = [((r * len(sids) + i) * 0.05, sid) for r in range(3) for i, sid in enumerate(sids)]
    fps = sorted(s.footprint(cases[s.sid][2].npat) for s in specs)
    srv = serve.Server(workers=3, budget_bytes=fps[-1] + fps[0], memsave=False)
    records, _ = srv.run(specs, cases, reqs)
    assert all(r is not None and not r.get("rejected") and not r.get("error") for r in records)
    assert srv.evictions > 0
    check_same_as_alone(specs, cases, records)


def test_concurrent_sessions_of_different_shapes(gpu):
    """Host threads driving tensor-core sessions of different category counts at the same time
    (what the serving loop does): no launch may fail because another thread's session set up
    the same kernel for a different shape."""
    import threading
    from gems_b200 import PhyloTree, synth
    trees = []
    for ncat, seed in ((1, 5), (4, 6), (2, 7), (4, 8)):
        rng = np.random.default_rng(seed)
        model = synth.protein(rng, ncat, 0.8)
        tree = synth.random_tree(24, 0.1, seed)
        aln = synth.simulate(tree, model, 3000, seed + 1)
        trees.append(PhyloTree.from_case(tree, model, aln, precision="mixed"))
    ref = [gt.computeLikelihood() for gt in trees]
    errors = []

    def run(gt, expect):
        try:
            for _ in range(40):
                gt.clearAllPartialLH()
                assert gt.computeLikelihood() == expect
        except Exception as e:  # collected and reported by the main thread
            errors.append(repr(e))

    th = [threading.Thread(target=run, args=(gt, r)) for gt, r in zip(trees, ref)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert not errors, errors
