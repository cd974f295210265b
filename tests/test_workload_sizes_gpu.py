"""Parity at the benchmark workloads' own sizes.

The headline workload exactly as bench.py runs it (R-MAT scale 24, edge
factor 16, 33 blocks, one walk per vertex, L = 10, the jump rule, Philox
seed 42, edge-record layout, autotuned launch shape), the single-source PPR
workload (scale 20, 100,000 walks from the top vertex, L <= 20), a 64-query
subset of the scale-26 msppr batch, and a mega-hub graph whose hub has more
out-edges than the packed vertex record's 24-bit degree field holds.

Integer results, so every comparison is bit for bit: the device R-MAT graph
equals the C generator's, visit counts equal the oracle's (and, at scale 24,
the reference engine's own with its rand_r routed to Philox), and top-100
lists equal the oracle's.  The accuracy test judges the PPR estimate against
the FP64 power series within three standard deviations of the Poisson noise
model (graphwalker_b200/accuracy.py).
"""
import struct
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCALE1, EF, NBLOCKS, L1, SEED = 24, 16, 32, 10, 42


def _blocksize_kb(scale, ef, nblocks):
    return -(-ef * (1 << scale) * 4 // nblocks // 1024)


@pytest.fixture(scope="module")
def rawwalks24(cuda_device, oracle):
    """The scale-24 graph on the device and, from the C generator, on the host."""
    import graphwalker_b200 as gw
    G = gw.Graph.rmat(SCALE1, EF, seed=1, blocksize_kb=_blocksize_kb(SCALE1, EF, NBLOCKS))
    rp, ci = oracle.rmat_csr(SCALE1, EF, seed=1)
    yield G, rp, ci
    G.close()


def test_rawwalks24_device_graph_equals_c_generator(rawwalks24, oracle):
    G, rp, ci = rawwalks24
    drp, dci = G.export_csr()
    assert np.array_equal(drp, rp) and np.array_equal(dci, ci)
    assert G.nblocks == 33
    assert np.array_equal(G.blocks, oracle.compute_blocks(rp, _blocksize_kb(SCALE1, EF, NBLOCKS)))


@pytest.fixture(scope="module")
def rawwalks24_oracle_counts(rawwalks24, oracle):
    _, rp, ci = rawwalks24
    cur = np.arange(len(rp) - 1, dtype=np.uint32)
    r = oracle.run_walks(rp, ci, cur, rule=oracle.RULE_JUMP, L=L1, seed=SEED)
    assert r["status"] == 0
    return r["counts"]


@pytest.mark.parametrize("layout", [1, 0], ids=["edge_records", "csr"])
def test_rawwalks24_counts_equal_oracle_as_benched(rawwalks24, rawwalks24_oracle_counts, layout):
    """bench.py's timed step: gw_walk_autotune, then gw_walk_device over all
    16,777,216 resident walk records into u32 counters."""
    import torch

    import graphwalker_b200 as gw
    G, _, _ = rawwalks24
    assert G.set_edge_records(layout) == bool(layout)
    nv = G.nv
    v = torch.arange(nv, dtype=torch.int64, device="cuda")
    walks = torch.stack([v, v, v, torch.zeros_like(v)], dim=1).to(torch.int32).contiguous()
    del v
    counts = torch.zeros(nv, dtype=torch.int32, device="cuda")
    p = gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, L1, seed=SEED)
    G.walk_autotune(p, walks, nv)
    for _ in range(2):  # a repeated step gives the same counts
        counts.zero_()
        G.walk_device(p, walks, nv, counts=counts)
        G.sync()
        got = counts.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, rawwalks24_oracle_counts)


def test_rawwalks24_counts_equal_oracle_through_host_api(rawwalks24, rawwalks24_oracle_counts):
    """bench.py's e2e call: gw_run_pools with the reference's 64-bit walk
    words in pinned host memory, per-block pools, counts copied back."""
    import torch

    import graphwalker_b200 as gw
    G, _, _ = rawwalks24
    nv = G.nv
    vv = np.arange(nv, dtype=np.uint64)
    blocks = G.blocks.astype(np.int64)
    blk = np.searchsorted(blocks[1:], np.arange(nv), side="right")
    words = torch.from_numpy(gw.encode(vv, vv - blocks[blk].astype(np.uint64), 0).view(np.int64)).pin_memory()
    offs = torch.from_numpy(np.r_[0, np.cumsum(np.bincount(blk, minlength=G.nblocks))].astype(np.int64)).pin_memory()
    out = torch.zeros(nv, dtype=torch.int32).pin_memory()
    G.run_pools(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, L1, seed=SEED), words.data_ptr(), offs.data_ptr(),
                out.data_ptr())
    assert np.array_equal(out.numpy().view(np.uint32), rawwalks24_oracle_counts)


def test_rawwalks24_counts_equal_reference_engine(rawwalks24, rawwalks24_oracle_counts, oracle, tmp_path):
    """The reference's own engine (graphwalker.hpp), walk manager and
    RandomWalkwithJump, compiled from its sources with rand_r routed to the
    Philox stream, on the scale-24 graph files: the oracle's counts, hence
    the device's."""
    exe = oracle.REF_DIR / "gw_ref_shim_0"
    if not exe.exists():
        pytest.skip("the shimmed reference engine is built where the reference tree exists")
    from graphwalker_b200 import formats
    _, rp, ci = rawwalks24
    nv = len(rp) - 1
    kb = _blocksize_kb(SCALE1, EF, NBLOCKS)
    base = str(tmp_path / "rmat24")
    blocks = formats.write_graph(base, rp, ci, kb).astype(np.int64)
    (tmp_path / "conf").mkdir()
    (tmp_path / "conf" / "graphwalker.cnf").write_text("\n")
    v = np.arange(nv, dtype=np.uint64)
    blk = np.searchsorted(blocks[1:], np.arange(nv), side="right")
    rec = np.zeros(nv, dtype=[("b", "<u4"), ("pad", "<u4"), ("w", "<u8")])
    rec["b"] = blk
    rec["w"] = (v << np.uint64(40)) | ((v - blocks[blk].astype(np.uint64)) << np.uint64(14))
    wf, of = tmp_path / "walks.bin", tmp_path / "out.bin"
    with open(wf, "wb") as f:
        f.write(struct.pack("<Q", nv))
        f.write(rec.tobytes())
    subprocess.run([str(exe), base, str(kb), str(wf), str(of), str(L1), f"{SEED:x}", str(nv), "0", "0.2", "0", "0"],
                   cwd=tmp_path, check=True, capture_output=True, timeout=1200)
    raw = of.read_bytes()
    status, nv_ref = struct.unpack_from("<II", raw, 0)
    assert status == 0 and nv_ref == nv
    assert np.array_equal(np.frombuffer(raw, np.uint32, nv, 8), rawwalks24_oracle_counts)


def test_rawwalks24_streamed_blocks_equal_oracle(rawwalks24, rawwalks24_oracle_counts):
    """The out-of-core path at the scale-24 raw-walk size: the CSR held in pinned host memory,
    8 device block slots for 33 blocks, the blocked engine (state-aware block
    choice, block copies on a side stream, eviction of the block with the
    fewest walks).  Counts equal the oracle's."""
    import graphwalker_b200 as gw
    G, _, _ = rawwalks24
    try:
        G.walks_clear()
        G.add_walks_at(np.arange(G.nv, dtype=np.uint32))
        G.set_residency(gw.STREAM_PINNED, nmblocks=8)
        steps = None
        # every chosen block copied into a slot (findSubGraph); blocks with at
        # most 64 k pending walks read in place; the default per-block rule
        for limit in (0, 1 << 16, gw.MAPPED_AUTO):
            G.set_mapped_block_walks(limit)
            st = G.run(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, L1, seed=SEED, mode=gw.MODE_BLOCKED,
                                 prob=0.2))
            assert np.array_equal(G.read_counts(), rawwalks24_oracle_counts), limit
            steps = steps or st.supersteps
            assert st.supersteps == steps  # the same block order
            if limit == 0:
                assert st.block_loads > 33 and st.mapped_supersteps == 0  # blocks evicted and loaded again
            else:
                assert 0 < st.mapped_supersteps < st.supersteps
    finally:
        G.set_mapped_block_walks(gw.MAPPED_AUTO)
        G.set_residency(gw.RESIDENT_HBM)


# ---------------------------------------------------------------- single-source PPR, scale 20
@pytest.fixture(scope="module")
def ppr20(cuda_device, oracle):
    import graphwalker_b200 as gw
    G = gw.Graph.rmat(20, EF, seed=1, blocksize_kb=_blocksize_kb(20, EF, 16))
    rp, ci = G.export_csr()
    src = int(np.argmax(np.diff(rp.astype(np.int64))))
    yield G, rp, ci, src
    G.close()


def _source_walks(src, B, first_id=0):
    import torch
    j = torch.arange(first_id, first_id + B, dtype=torch.int64, device="cuda")
    w = torch.stack([torch.full_like(j, src), j, torch.full_like(j, src), torch.zeros_like(j)], 1)
    return w.to(torch.int32).contiguous()


def test_ppr20_counts_and_top100_equal_oracle(ppr20, oracle):
    """100,000 walks from the top vertex under the PPR rule (stop w.p. 0.15,
    a dangling vertex returns the walk to its source, at most 20 hops): the
    counts of the device walk launch and the top-100 of gw_ppr_run equal the
    oracle's."""
    import torch

    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    G, rp, ci, src = ppr20
    B, L = 100_000, 20
    ref = oracle.run_walks(rp, ci, np.full(B, src, np.uint32), ids=np.arange(B, dtype=np.uint32),
                           src=np.full(B, src, np.uint32), rule=oracle.RULE_PPR, L=L, seed=SEED)
    assert ref["status"] == 0
    for aggregate in (True, False):
        counts = torch.zeros(G.nv, dtype=torch.int32, device="cuda")
        G.walk_device(gw.params(gw.RULE_PPR, gw.SINK_VERTEX_COUNT, L, seed=SEED, aggregate=aggregate),
                      _source_walks(src, B), B, counts=counts)
        G.sync()
        assert np.array_equal(counts.cpu().numpy().view(np.uint32), ref["counts"])
    nz = np.flatnonzero(ref["counts"])
    want = accuracy.count_topk(nz, ref["counts"][nz], 100)
    for batched in (True, False):
        ids, cnt, _ = G.ppr(gw.params(gw.RULE_PPR, gw.SINK_NONE, L, seed=SEED), np.array([src], np.uint32),
                            np.array([B], np.uint32), k=100, batched=batched)
        assert np.array_equal(ids[0], want)
        assert np.array_equal(cnt[0], ref["counts"][want])


@pytest.mark.parametrize("rule", [4, 1], ids=["ppr", "stop"])
def test_ppr20_accuracy_within_monte_carlo_noise(ppr20, rule):
    """The estimate's L1 error and top-100 overlap against the FP64 power
    series lie within three standard deviations of what Poisson noise at
    this budget predicts, over several seeds."""
    import torch

    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    G, _, _, src = ppr20
    B, L = 100_000, 20
    mu = G.expected_visits(gw.params(rule, gw.SINK_NONE, L), src)
    assert mu[src] >= 1.0
    exp = accuracy.expected_accuracy(mu, B, L, k=100)
    overlaps, l1s = [], []
    for seed in range(5):
        counts = torch.zeros(G.nv, dtype=torch.int32, device="cuda")
        G.walk_device(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=1000 + seed), _source_walks(src, B), B,
                      counts=counts)
        G.sync()
        c = counts.cpu().numpy().view(np.uint32)
        m = accuracy.measured_accuracy(mu, B, L, accuracy.count_topk(np.arange(G.nv), c, 100), counts=c, k=100)
        assert m["within_3_sigma"], m
        overlaps.append(m["top_overlap"])
        l1s.append(m["l1_error"])
    # the mean of five draws is tighter still
    assert np.mean(overlaps) >= exp["expected_overlap"] - 3 * exp["overlap_sigma"] / np.sqrt(5)
    assert np.mean(l1s) <= exp["expected_l1"] + 3 * exp["l1_sigma"] / np.sqrt(5)
    assert exp["expected_l1"] <= exp["l1_bound"]


# ---------------------------------------------------------------- multi-source PPR, scale 26
def test_msppr26_subset_top100_equals_oracle(cuda_device, oracle):
    """The scale-26 msppr batch as benched (4,096 queries, sources uniform
    over out-degree >= 1, budgets round(10^U(2,5)), stop rule, L <= 20,
    top-100), batched in one launch; 64 of its queries (every 64th, with
    their batch positions as walk ids) equal the oracle's top-100 lists."""
    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    scale, nq, k, L = 26, 4096, 100, 20
    with gw.Graph.rmat(scale, EF, seed=1, blocksize_kb=_blocksize_kb(scale, EF, NBLOCKS)) as G:
        G.set_edge_records(2)
        rp, ci = G.export_csr()
        rng = np.random.default_rng(7)  # bench.py msppr_queries
        sources = rng.choice(np.nonzero(np.diff(rp.astype(np.int64)) > 0)[0], nq).astype(np.uint32)
        budgets = np.round(10 ** rng.uniform(2, 5, nq)).astype(np.uint32)
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, L, seed=SEED)
        G.ppr_autotune(p, sources[:256], budgets[:256])
        ids, cnt, st = G.ppr(p, sources, budgets, k=k, batched=True)
        assert st.walks == int(budgets.astype(np.int64).sum())
        prefix = np.r_[0, np.cumsum(budgets.astype(np.int64))]
        # the two largest queries' lists, judged against the FP64 series
        # within the Monte Carlo noise of their budgets
        for q in np.argsort(-budgets.astype(np.int64), kind="stable")[:2]:
            mu = G.expected_visits(p, int(sources[q]))
            m = accuracy.measured_accuracy(mu, int(budgets[q]), L, ids[q], k=k)
            assert m["within_3_sigma"], m
    for q in range(0, nq, 64):
        B = int(budgets[q])
        cur = np.full(B, sources[q], np.uint32)
        r = oracle.run_walks(rp, ci, cur, ids=np.arange(prefix[q], prefix[q + 1], dtype=np.uint32), src=cur,
                             rule=oracle.RULE_STOP, L=L, seed=SEED)
        assert r["status"] == 0
        nz = np.flatnonzero(r["counts"])
        want = accuracy.count_topk(nz, r["counts"][nz], k)
        got = ids[q][ids[q] != 0xFFFFFFFF]
        assert np.array_equal(got, want), f"query {q}"
        assert np.array_equal(cnt[q][: len(want)], r["counts"][want]), f"query {q}"


# ---------------------------------------------------------------- mega-hub
def _star_graph(nv=1 << 16, hub_deg=(1 << 24) + 1):
    """Vertex 0 has hub_deg out-edges (more than the packed record's 24-bit
    degree field holds: its record escapes to the row pointer).  Vertex
    v >= 1 points back to the hub and to v + 1, except every 7th vertex,
    which is dangling."""
    deg = np.full(nv, 2, np.int64)
    deg[0] = hub_deg
    deg[np.arange(nv) % 7 == 3] = 0
    rowptr = np.r_[0, np.cumsum(deg)].astype(np.uint64)
    colidx = np.empty(int(rowptr[-1]), np.uint32)
    colidx[:hub_deg] = (np.arange(hub_deg, dtype=np.int64) % (nv - 1) + 1).astype(np.uint32)
    rest = np.flatnonzero(deg[1:] == 2) + 1
    starts = rowptr[rest].astype(np.int64)
    colidx[starts] = 0
    colidx[starts + 1] = ((rest + 1) % nv).astype(np.uint32)
    return rowptr, colidx


@pytest.fixture(scope="module")
def star(cuda_device, oracle):
    rp, ci = _star_graph()
    return rp, ci, oracle.compute_blocks(rp, 64)


@pytest.mark.parametrize("layout", [0, 1], ids=["csr", "edge_records"])
@pytest.mark.parametrize("rule", [0, 1, 3], ids=["jump", "stop", "restart"])
def test_mega_hub_walks_equal_oracle(star, oracle, layout, rule):
    """Walks through a vertex of out-degree 2^24 + 1, resident and blocked."""
    import graphwalker_b200 as gw
    rp, ci, blocks = star
    nv = len(rp) - 1
    assert np.diff(rp.astype(np.int64))[0] >= 0xFFFFFF
    L = 12
    cur = np.r_[np.arange(nv), np.zeros(8192, np.int64)].astype(np.uint32)  # and 8192 walks at the hub
    ids = np.arange(len(cur), dtype=np.uint32)
    ref = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, rule=rule, L=L, seed=SEED)
    assert ref["status"] == 0
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        assert G.set_edge_records(layout) == bool(layout)
        for mode in (gw.MODE_RESIDENT, gw.MODE_BLOCKED):
            G.walks_clear()
            G.add_walks_at(cur, ids=ids)
            G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=SEED, mode=mode))
            assert np.array_equal(G.read_counts(), ref["counts"]), f"mode {mode}"


@pytest.mark.parametrize("layout", [0, 1], ids=["csr", "edge_records"])
def test_mega_hub_queries_equal_oracle(star, oracle, layout):
    """msppr queries from the hub and from vertices next to it: top-100
    lists batched and plain equal the oracle's."""
    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    rp, ci, blocks = star
    sources = np.array([0, 1, 2, 0, 5], np.uint32)
    budgets = np.array([30000, 500, 700, 1, 9000], np.uint32)
    prefix = np.r_[0, np.cumsum(budgets.astype(np.int64))]
    L, k = 20, 100
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        assert G.set_edge_records(layout) == bool(layout)
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, L, seed=SEED)
        for batched in (True, False):
            ids, cnt, _ = G.ppr(p, sources, budgets, k=k, batched=batched)
            for q in range(len(sources)):
                cur = np.full(int(budgets[q]), sources[q], np.uint32)
                r = oracle.run_walks(rp, ci, cur, ids=np.arange(prefix[q], prefix[q + 1], dtype=np.uint32),
                                     src=cur, rule=oracle.RULE_STOP, L=L, seed=SEED)
                nz = np.flatnonzero(r["counts"])
                want = accuracy.count_topk(nz, r["counts"][nz], k)
                assert np.array_equal(ids[q][ids[q] != 0xFFFFFFFF], want), (batched, q)
                assert np.array_equal(cnt[q][: len(want)], r["counts"][want]), (batched, q)
