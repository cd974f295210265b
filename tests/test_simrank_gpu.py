"""SimRank's meeting reduction on the device (gw_simrank_meet) against the
oracle's restatement of SimRank::computeResult (apps/simrank.cpp:71-84).

Meeting counts are integers and must match exactly; the estimate built from
them is compared with the app's float sum at rel 1e-5 (the app accumulates
in float, the estimate in double)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.uint32).view(np.int32)).cuda()


def _graph(g):
    import graphwalker_b200 as gw
    return gw.Graph.from_csr(g["rowptr"], g["colidx"], g["blocks"])


def test_meet_counts_on_reference_paths(cuda_device, oracle):
    """The reference engine's SimRank paths (golden): counts and estimate."""
    import graphwalker_b200 as gw
    g = load_golden("rmat10")
    R, L = 20, 11
    gp = g["simrank_paths"]
    for a, b in [(7, 9), (7, 7), (9, 7)]:
        pa, pb = gp[a][: R * L].reshape(R, L), gp[b][: R * L].reshape(R, L)
        ref_est, ref_meet = oracle.simrank(pa, pb, R, L)
        with _graph(g) as G:
            meet = G.simrank_meet(_dev(pa), _dev(pb), R, L)
        assert np.array_equal(meet, ref_meet), (a, b)
        assert gw.simrank_estimate(meet, R) == pytest.approx(ref_est, rel=1e-5, abs=1e-7)


@pytest.mark.parametrize("R,L", [(1, 1), (64, 32), (300, 13), (257, 70)])
def test_meet_counts_random_paths(cuda_device, oracle, R, L):
    """Partial tiles, positions across the 32-position staging chunks, empty
    visits (0xFFFFFFFF, never a meeting) and dense collisions."""
    g = load_golden("hand")
    rng = np.random.default_rng(R * 1000 + L)
    pa = rng.integers(0, 12, (R, L)).astype(np.uint32)
    pb = rng.integers(0, 12, (R, L)).astype(np.uint32)
    pa[rng.random((R, L)) < 0.2] = 0xFFFFFFFF
    pb[rng.random((R, L)) < 0.2] = 0xFFFFFFFF
    _, ref_meet = oracle.simrank(pa, pb, R, L)
    with _graph(g) as G:
        meet = G.simrank_meet(_dev(pa), _dev(pb), R, L)
    assert np.array_equal(meet, ref_meet)
    assert int(meet.sum()) <= R * R


def test_simrank_end_to_end_on_device(cuda_device, oracle):
    """SimRank placement (apps/simrank.cpp:30-57: replica i of a and of b
    starts at hop i*L, walk key = the source) walked on the device with the
    path sink, then reduced on the device: equals the app's value computed
    from the reference engine's own paths."""
    import graphwalker_b200 as gw
    g = load_golden("rmat10")
    R, L, a, b = 20, 11, 7, 9
    cur = np.r_[np.full(R, a), np.full(R, b)].astype(np.uint32)
    hop = np.r_[np.arange(R) * L, np.arange(R) * L].astype(np.uint32)
    gp = g["simrank_paths"]
    ref_est, ref_meet = oracle.simrank(gp[a][: R * L].reshape(R, L), gp[b][: R * L].reshape(R, L), R, L)
    with _graph(g) as G:
        G.walks_clear()
        G.add_walks_at(cur, source=cur, hop=hop, ids=cur)
        G.run(gw.params(gw.RULE_RESTART, gw.SINK_PATH_RECORD, L, seed=int(g["seed"]), path_stride=L))
        paths, lens = G.read_paths(2 * R, L)
        # both sources lie in one block, so the pool keeps insertion order
        assert np.all(np.searchsorted(G.blocks[1:], cur, side="right") == np.searchsorted(G.blocks[1:], a, side="right"))
        meet = G.simrank_meet(_dev(paths[:R]), _dev(paths[R:]), R, L)
    assert np.array_equal(meet, ref_meet)
    assert gw.simrank_estimate(meet, R) == pytest.approx(ref_est, rel=1e-5, abs=1e-7)


def test_simrank_batch_matches_oracle(cuda_device, oracle):
    """A batch of SimRank queries in one walk launch and one reduction: each
    query's meeting counts equal the oracle's SimRank on the oracle's walks
    (replica i of vertex v starts at hop i*L, keyed on v)."""
    import graphwalker_b200 as gw
    rp, ci = oracle.rmat_csr(12, 8, seed=4)
    blocks = oracle.compute_blocks(rp, 64)
    rng = np.random.default_rng(5)
    nq, R, L = 40, 96, 7
    a = rng.integers(0, len(rp) - 1, nq).astype(np.uint32)
    b = rng.integers(0, len(rp) - 1, nq).astype(np.uint32)
    b[:5] = a[:5]          # a vertex with itself: both sides are the same walks
    a[10:14] = a[9]        # queries sharing a vertex share its walks
    seed = 21

    def walks_of(v):
        cur = np.full(R, v, np.uint32)
        r = oracle.run_walks(rp, ci, cur, ids=cur, src=cur, hop0=(np.arange(R) * L).astype(np.uint32),
                             rule=3, L=L, seed=seed, stride=L, counts=False)
        return r["paths"]

    with gw.Graph.from_csr(rp, ci, blocks) as G:
        scores, meet = G.simrank_batch(a, b, R, L, seed=seed)
    cache = {}
    for q in range(nq):
        pa = cache.setdefault(int(a[q]), walks_of(int(a[q])))
        pb = cache.setdefault(int(b[q]), walks_of(int(b[q])))
        _, ref_meet = oracle.simrank(pa, pb, R, L)
        assert np.array_equal(meet[q], ref_meet), q
        assert scores[q] == pytest.approx(gw.simrank_estimate(ref_meet, R), rel=1e-12)
    assert np.all(meet[:5, 0] >= R)  # every walk meets itself at its source
