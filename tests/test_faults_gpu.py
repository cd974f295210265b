"""Failure detection without a GPU fault: host-side injected failures
(gw_inject_fault) of device allocations, pinned allocations and graph-file
reads.  Each must surface as a status code from the call that met it, and
leave the process and its contexts usable: the next call gives the oracle's
results.  Nothing here faults, traps or hangs the GPU."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def disarm():
    import graphwalker_b200 as gw
    yield
    gw.inject_fault(gw.FAULT_NONE)


def _counts(G, g, oracle):
    import graphwalker_b200 as gw
    cur = np.arange(G.nv, dtype=np.uint32)
    G.walks_clear()
    G.add_walks_at(cur)
    G.run(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, 10, seed=5))
    ref = oracle.run_walks(g["rowptr"], g["colidx"], cur, rule=0, L=10, seed=5)
    return np.array_equal(G.read_counts(), ref["counts"])


def test_every_device_allocation_of_open_and_run_can_fail(cuda_device, oracle):
    """The k-th device allocation of open + run fails, for every k until the
    whole sequence succeeds; each failure is a status code, and a fresh
    context afterwards gives the oracle's counts."""
    import graphwalker_b200 as gw
    g = load_golden("rmat10")
    failures = 0
    for k in range(64):
        gw.inject_fault(gw.FAULT_DEVICE_ALLOC, k)
        try:
            with gw.Graph.from_csr(g["rowptr"], g["colidx"], g["blocks"]) as G:
                ok = _counts(G, g, oracle)
        except gw.GwError as e:
            assert e.code in (gw._lib.GW_E_CUDA, gw._lib.GW_E_NOMEM), e
            failures += 1
            gw.inject_fault(gw.FAULT_NONE)
            with gw.Graph.from_csr(g["rowptr"], g["colidx"], g["blocks"]) as G:
                assert _counts(G, g, oracle)
            continue
        assert ok
        break  # the fault point lay beyond the last allocation: all of them were covered
    else:
        pytest.fail("open + run made more than 64 device allocations")
    assert failures >= 5


def test_failed_query_batch_leaves_the_context_usable(cuda_device, oracle):
    import graphwalker_b200 as gw
    g = load_golden("rmat13")
    rng = np.random.default_rng(2)
    deg = np.diff(g["rowptr"].astype(np.int64))
    src = rng.choice(np.nonzero(deg)[0], 30).astype(np.uint32)
    bud = rng.integers(10, 800, 30).astype(np.uint32)
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=4)
    with gw.Graph.from_csr(g["rowptr"], g["colidx"], g["blocks"]) as G:
        ref_ids, ref_cnt, _ = G.ppr(p, src, 2 * bud)  # twice the budgets: the next batch needs larger buffers
        gw.inject_fault(gw.FAULT_DEVICE_ALLOC, 0)
        with pytest.raises(gw.GwError):
            G.ppr(p, src, 4 * bud)
        gw.inject_fault(gw.FAULT_NONE)
        ids, cnt, _ = G.ppr(p, src, 2 * bud)
        assert np.array_equal(ids, ref_ids) and np.array_equal(cnt, ref_cnt)
        assert _counts(G, g, oracle)


@pytest.mark.parametrize("kind,code", [("FAULT_FILE_READ", 4), ("FAULT_PINNED_ALLOC", 3)])
def test_graph_file_faults(cuda_device, oracle, tmp_path, kind, code):
    """A short read of the preprocessed files, or a failed pinned buffer,
    fails gw_open with GW_E_IO / GW_E_NOMEM; the next open works."""
    import graphwalker_b200 as gw
    from graphwalker_b200 import formats
    g = load_golden("rmat10")
    base = str(tmp_path / "g")
    formats.write_graph(base, g["rowptr"], g["colidx"], int(g["blocksize_kb"]))
    gw.inject_fault(getattr(gw, kind), 0)
    with pytest.raises(gw.GwError) as ei:
        gw.Graph.open(base, int(g["blocksize_kb"]))
    assert ei.value.code == code
    with gw.Graph.open(base, int(g["blocksize_kb"])) as G:
        assert _counts(G, g, oracle)


def test_server_open_fails_cleanly_without_memory(cuda_device):
    import graphwalker_b200 as gw
    g = load_golden("rmat10")
    p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=1)
    with gw.Graph.from_csr(g["rowptr"], g["colidx"], g["blocks"]) as G:
        gw.inject_fault(gw.FAULT_DEVICE_ALLOC, 0)
        with pytest.raises(gw.GwError):
            G.serve(p, table_slots=1 << 16)
        gw.inject_fault(gw.FAULT_NONE)
        with G.serve(p, table_slots=1 << 16) as S:
            t = S.submit(5, 200)
            ids, counts, _ = S.wait(t, 60_000)
            assert counts[0] >= 200  # the source is visited by every walk
