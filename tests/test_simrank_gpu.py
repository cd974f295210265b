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
