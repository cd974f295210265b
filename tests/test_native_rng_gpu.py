"""Native-RNG mode (GW_RNG_NATIVE): one Philox block serves two hops.

Its draws are a pure function of (seed, walk id, hop, stream), so it is
checked two ways: bit for bit against the oracle's restatement of the same
draw layout (every kernel and layout that walks), and statistically against
the FP64 power series at the single-source PPR workload's size -- the L1
error and top-100 overlap within three standard deviations of the Poisson
noise model (graphwalker_b200/accuracy.py).  The reference's own stream
(rand_r seeded with the clock) cannot be reproduced, so only the statistics
connect this mode to it.
"""
import struct
import subprocess

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

NATIVE = 1


@pytest.fixture(scope="module")
def small(cuda_device, oracle):
    rp, ci = oracle.rmat_csr(12, 8, seed=3)
    return rp, ci, oracle.compute_blocks(rp, 16)


@pytest.mark.parametrize("rule", [0, 1, 2, 3, 4], ids=["jump", "stop", "prob", "restart", "ppr"])
@pytest.mark.parametrize("layout", [0, 1], ids=["csr", "edge_records"])
def test_native_walks_equal_oracle(small, oracle, rule, layout):
    """Resident and blocked engines, walks starting at odd and even hops."""
    import graphwalker_b200 as gw
    rp, ci, blocks = small
    nv = len(rp) - 1
    L = 9
    cur = np.arange(nv, dtype=np.uint32)
    hop0 = (np.arange(nv) % 3 if rule != 3 else np.zeros(nv)).astype(np.uint32)  # odd and even starting hops
    ref = oracle.run_walks(rp, ci, cur, rule=rule, L=L, seed=17, hop0=hop0, rng=NATIVE)
    assert ref["status"] == 0
    philox = oracle.run_walks(rp, ci, cur, rule=rule, L=L, seed=17, hop0=hop0)
    assert not np.array_equal(ref["counts"], philox["counts"])  # a different stream
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        assert G.set_edge_records(layout) == bool(layout)
        for mode in (gw.MODE_RESIDENT, gw.MODE_BLOCKED):
            G.walks_clear()
            G.add_walks_at(cur, hop=hop0)
            G.run(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=17, mode=mode, rng=gw.RNG_NATIVE))
            assert np.array_equal(G.read_counts(), ref["counts"]), f"mode {mode}"


@pytest.mark.parametrize("layout", [0, 1], ids=["csr", "edge_records"])
def test_native_queries_equal_oracle(small, oracle, layout):
    """msppr queries, batched and plain: each top-k list equals the oracle's."""
    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    rp, ci, blocks = small
    deg = np.diff(rp.astype(np.int64))
    rng = np.random.default_rng(4)
    sources = rng.choice(np.nonzero(deg)[0], 24).astype(np.uint32)
    budgets = rng.integers(1, 3000, 24).astype(np.uint32)
    prefix = np.r_[0, np.cumsum(budgets.astype(np.int64))]
    k = 40
    with gw.Graph.from_csr(rp, ci, blocks) as G:
        assert G.set_edge_records(layout) == bool(layout)
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=23, rng=gw.RNG_NATIVE)
        for batched in (True, False):
            ids, cnt, _ = G.ppr(p, sources, budgets, k=k, batched=batched)
            for q in range(len(sources)):
                cur = np.full(int(budgets[q]), sources[q], np.uint32)
                r = oracle.run_walks(rp, ci, cur, ids=np.arange(prefix[q], prefix[q + 1], dtype=np.uint32), src=cur,
                                     rule=1, L=20, seed=23, rng=NATIVE)
                nz = np.flatnonzero(r["counts"])
                want = accuracy.count_topk(nz, r["counts"][nz], k)
                assert np.array_equal(ids[q][ids[q] != 0xFFFFFFFF], want), (batched, q)
                assert np.array_equal(cnt[q][: len(want)], r["counts"][want]), (batched, q)


@pytest.mark.parametrize("rule", [4, 1], ids=["ppr", "stop"])
def test_native_accuracy_within_monte_carlo_noise(cuda_device, rule):
    """R-MAT scale 20, 100,000 walks from the top vertex, L <= 20: the
    native-mode estimate's L1 error and top-100 overlap against the FP64 power
    series lie within three standard deviations of the Poisson model, for each
    of five seeds."""
    import torch

    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    B, L = 100_000, 20
    with gw.Graph.rmat(20, 16, seed=1, blocksize_kb=-(-16 * (1 << 20) * 4 // 16 // 1024)) as G:
        rp, _ = G.export_csr()
        src = int(np.argmax(np.diff(rp.astype(np.int64))))
        mu = G.expected_visits(gw.params(rule, gw.SINK_NONE, L), src)
        j = torch.arange(B, dtype=torch.int64, device="cuda")
        walks = torch.stack([torch.full_like(j, src), j, torch.full_like(j, src), torch.zeros_like(j)], 1)
        walks = walks.to(torch.int32).contiguous()
        for seed in range(5):
            counts = torch.zeros(G.nv, dtype=torch.int32, device="cuda")
            G.walk_device(gw.params(rule, gw.SINK_VERTEX_COUNT, L, seed=2000 + seed, rng=gw.RNG_NATIVE), walks, B,
                          counts=counts)
            G.sync()
            c = counts.cpu().numpy().view(np.uint32)
            m = accuracy.measured_accuracy(mu, B, L, accuracy.count_topk(np.arange(G.nv), c, 100), counts=c)
            assert m["within_3_sigma"], m


def test_native_mode_through_the_drop_in_knob(cuda_device, oracle, tmp_path):
    """A program written against GraphWalker's API selects the native stream
    with the gw_rng knob and receives the oracle's native-mode visits."""
    from test_compat import _prepare, _walks_file, build_compat_app
    g = load_golden("rmat10")
    base = _prepare(tmp_path, g, "rmat10")
    nv = len(g["rowptr"]) - 1
    tag = "jump"
    rule, L = int(g[f"{tag}_rule"]), int(g[f"{tag}_L"])
    app = build_compat_app(rule, tmp_path / "app")
    _walks_file(tmp_path / "walks.bin", g, tag)
    out = tmp_path / "out.bin"
    subprocess.run([str(app), base, str(int(g["blocksize_kb"])), str(tmp_path / "walks.bin"), str(out), str(L),
                    str(int(g["seed"])), str(nv), "0", "0", "gw_walk_id", "source", "seed", str(int(g["seed"])),
                    "gw_rng", "native"], cwd=tmp_path, check=True, capture_output=True)
    counts = np.frombuffer(out.read_bytes(), np.uint32, nv, 8)
    cur, src, hop = g[f"{tag}_cur"], g[f"{tag}_src"], g[f"{tag}_hop"]
    ref = oracle.run_walks(g["rowptr"], g["colidx"], cur, ids=src, src=src, hop0=hop, rule=rule, L=L,
                           seed=int(g["seed"]), rng=NATIVE)
    assert np.array_equal(counts, ref["counts"])
    assert not np.array_equal(counts, g[f"{tag}_counts"])  # the deterministic mode's goldens differ
