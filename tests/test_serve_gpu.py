"""Serving with continuous batching (gw_serve_*).

Each result must be the same alone and in a mix (bit-exact: a query's draws
depend only on its source, budget and stream), equal to the batch API for
stream 0, and equal between the batched and the plain per-query servers.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# every wait is bounded: a scheduler thread that died fails the test with
# GW_E_TIMEOUT instead of hanging it
WAIT_MS = 60_000


@pytest.fixture(scope="module")
def graph(cuda_device):
    import graphwalker_b200 as gw
    G = gw.Graph.rmat(16, 16, seed=8, blocksize_kb=256)
    yield G
    G.close()


def _queries(G, n, seed, max_budget=5000):
    rp, _ = G.export_csr()
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(seed)
    src = rng.choice(np.nonzero(deg)[0], n).astype(np.uint32)
    bud = rng.integers(1, max_budget, n).astype(np.uint32)
    return src, bud


def test_result_is_the_same_alone_and_in_a_mix(graph):
    import graphwalker_b200 as gw
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=3)
    src, bud = _queries(graph, 200, 1)
    x_src, x_bud, x_stream = int(src[0]), 20000, 777
    with graph.serve(p, quantum=4096) as S:
        alone = S.wait(S.submit(x_src, x_bud, x_stream), WAIT_MS)
    with graph.serve(p, quantum=4096) as S:
        tickets = [S.submit(int(s), int(b), i) for i, (s, b) in enumerate(zip(src[:100], bud[:100]))]
        tx = S.submit(x_src, x_bud, x_stream)
        tickets += [S.submit(int(s), int(b), 1000 + i) for i, (s, b) in enumerate(zip(src[100:], bud[100:]))]
        mixed = S.wait(tx, WAIT_MS)
        for t in tickets:
            S.wait(t, WAIT_MS)
        st = S.stats()
    assert np.array_equal(alone[0], mixed[0]) and np.array_equal(alone[1], mixed[1])
    assert st.completed == 201 and st.supersteps < 201  # queries shared supersteps
    assert mixed[2].done_ns >= mixed[2].admit_ns >= mixed[2].arrival_ns


def test_served_stream_zero_equals_batch_api_and_plain_server(graph):
    import graphwalker_b200 as gw
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=11)
    src, bud = _queries(graph, 30, 2)
    res = {}
    for mode in (gw._lib.SERVE_BATCHED, gw._lib.SERVE_PLAIN):
        with graph.serve(p, mode=mode) as S:
            tickets = [S.submit(int(s), int(b), 0) for s, b in zip(src, bud)]
            res[mode] = [S.wait(t, WAIT_MS)[:2] for t in tickets]
    for q in range(30):
        ids, cnt, _ = graph.ppr(p, src[q:q + 1], bud[q:q + 1], k=100)
        for mode in res:
            assert np.array_equal(res[mode][q][0], ids[0]) and np.array_equal(res[mode][q][1], cnt[0])


def test_table_restarts_and_arena_admission(graph):
    import graphwalker_b200 as gw
    from graphwalker_b200._lib import GW_E_NOMEM, GwError
    p = gw.params(gw.RULE_JUMP, gw.SINK_NONE, 20, seed=5)
    src, bud = _queries(graph, 40, 3, max_budget=3000)
    with graph.serve(p) as S:
        ref = [S.wait(S.submit(int(s), int(b), 9), WAIT_MS)[:2] for s, b in zip(src, bud)]
    p.table_factor = 1  # tables fill up: restarts with larger tables
    with graph.serve(p, table_slots=1 << 18) as S:  # a small arena: queries queue for space
        tickets = [S.submit(int(s), int(b), 9) for s, b in zip(src, bud)]
        got = [S.wait(t, WAIT_MS) for t in tickets]
        assert S.stats().restarts > 0
        with pytest.raises(GwError) as e:
            S.submit(int(src[0]), 1 << 20, 1)  # needs more slots than the arena has
        assert e.value.code == GW_E_NOMEM
    for (ri, rc), (gi, gc, _) in zip(ref, got):
        assert np.array_equal(ri, gi) and np.array_equal(rc, gc)


def test_scheduled_arrivals_and_latency_accounting(graph):
    import graphwalker_b200 as gw
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=1)
    src, bud = _queries(graph, 300, 4, max_budget=500)
    with graph.serve(p) as S:
        t0 = S.clock_ns() + 2_000_000
        arrivals = t0 + np.cumsum(np.random.default_rng(0).exponential(1e9 / 20000, 300)).astype(np.int64)
        tickets = [S.submit(int(s), int(b), i, int(a)) for i, (s, b, a) in enumerate(zip(src, bud, arrivals))]
        timings = [S.wait(t, WAIT_MS)[2] for t in tickets]
    for a, tm in zip(arrivals, timings):
        assert tm.arrival_ns == a and tm.admit_ns >= a and tm.done_ns > tm.admit_ns
