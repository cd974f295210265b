"""Pins the C oracle to the reference: golden vectors made by GraphWalker's
own engine and walk classes (tests/golden/make_golden.py), the published
Philox4x32-10 known-answer vectors, and the float continuation test."""
from pathlib import Path

import numpy as np
import pytest

from conftest import golden_runs, load_golden

CASES = ["hand", "rmat10", "rmat13"]


def test_philox_known_answers(oracle):
    # Random123 kat_vectors for philox4x32_10 (Salmon et al., SC'11)
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_continue_threshold_matches_float_test(oracle):
    # (float)r/RAND_MAX > 0.15 (randomwalkwithjump.hpp:45) <=> r >= 322122544
    thr = oracle.continue_threshold(0.15)
    assert thr == 322122544
    lib = oracle.lib()
    for r in list(range(thr - 70, thr + 70)) + [0, 1, 2**31 - 1, 2**30, 2**29 + 17]:
        assert bool(lib.gwo_continue_test(r, 0.15)) == (r >= thr), r
    # other probabilities stay monotone and exact around the threshold
    for p in (0.0, 0.05, 0.5, 0.85, 0.999):
        t = oracle.continue_threshold(p)
        for r in range(max(0, t - 40), min(2**31, t + 40)):
            assert bool(lib.gwo_continue_test(r, p)) == (r >= t)
    assert oracle.continue_threshold(1.0) == 2**31


def test_continue_threshold_exhaustive(oracle):
    # every 31-bit draw: the integer comparison the kernels make equals the
    # reference's float expression for the reference's 0.15
    assert oracle.lib().gwo_threshold_mismatches(0.15) == 0


def test_codec_matches_walk_hpp(oracle):
    lib = oracle.lib()
    rng = np.random.default_rng(5)
    for _ in range(200):
        s, c, h = int(rng.integers(0, 2**24)), int(rng.integers(0, 2**26)), int(rng.integers(0, 2**14))
        w = lib.gwo_encode(s, c, h)
        assert (lib.gwo_get_source(w), lib.gwo_get_current(w), lib.gwo_get_hop(w)) == (s, c, h)
    # fields are masked exactly as WalkManager::encode does
    w = lib.gwo_encode(0x1FFFFFF, 0x7FFFFFF, 0x7FFF)
    assert (lib.gwo_get_source(w), lib.gwo_get_current(w), lib.gwo_get_hop(w)) == (0xFFFFFF, 0x3FFFFFF, 0x3FFF)


@pytest.mark.parametrize("case", CASES)
def test_compute_blocks_matches_reference(oracle, case):
    g = load_golden(case)
    assert np.array_equal(oracle.compute_blocks(g["rowptr"], int(g["blocksize_kb"])), g["blocks"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_walks_match_reference_engine(oracle, case):
    g = load_golden(case)
    for tag in golden_runs(g):
        rule, L = int(g[f"{tag}_rule"]), int(g[f"{tag}_L"])
        cur, src, hop = g[f"{tag}_cur"], g[f"{tag}_src"], g[f"{tag}_hop"]
        gp = g[f"{tag}_paths"]
        stride = gp.shape[1]
        per_walk = stride if tag != "simrank" else L
        r = oracle.run_walks(g["rowptr"], g["colidx"], cur, src=src, ids=src, hop0=hop, rule=rule, L=L,
                             seed=int(g["seed"]), stride=per_walk, closure=True)
        assert r["status"] == 0
        assert np.array_equal(r["counts"], g[f"{tag}_counts"]), f"{case}/{tag} counts"
        assert r["closure"] == int(g[f"{tag}_closure"]), f"{case}/{tag} closure"
        if tag == "simrank":
            # shim records paths[source][hop]; replica i of a source starts at hop i*L
            nrep = len(cur) // 2
            for j, s in enumerate(cur):
                i = j % nrep
                seg = gp[s][i * L: i * L + L]
                k = int(r["plen"][j])
                assert np.array_equal(r["paths"][j][:k], seg[:k])
                assert np.all(seg[k:] == 0xFFFFFFFF)
        else:
            for j, s in enumerate(src):
                k = min(int(r["plen"][j]), stride)
                assert np.array_equal(r["paths"][j][:k], gp[s][:k]), f"{case}/{tag} walk {j}"
                assert np.all(gp[s][k:] == 0xFFFFFFFF)


def test_oracle_block_engine_equals_whole_graph_run(oracle):
    g = load_golden("rmat10")
    for rule, L in [(0, 10), (1, 10), (3, 6)]:
        cur = np.arange(len(g["rowptr"]) - 1, dtype=np.uint32)
        whole = oracle.run_walks(g["rowptr"], g["colidx"], cur, rule=rule, L=L, seed=7)
        for prob in (0.0, 0.2, 1.0):
            be = oracle.block_engine(g["rowptr"], g["colidx"], g["blocks"], cur, rule=rule, L=L, seed=7, prob=prob)
            assert np.array_equal(be["counts"], whole["counts"])


def test_rmat_generator_properties(oracle):
    rp, ci = oracle.rmat_csr(12, 16, seed=11)
    nv = 1 << 12
    assert rp[0] == 0 and rp[-1] == len(ci) and np.all(np.diff(rp.astype(np.int64)) >= 0)
    src = np.repeat(np.arange(nv), np.diff(rp.astype(np.int64)))
    assert not np.any(src == ci), "self-loops must be removed"
    key = src.astype(np.uint64) << np.uint64(32) | ci.astype(np.uint64)
    assert np.all(np.diff(key.astype(np.float64)) >= 0), "rows sorted by (src, dst)"
    assert len(ci) > 0.9 * 16 * nv  # few self-loops
    # the permutation is a bijection
    lib = oracle.lib()
    perm = np.array([lib.gwo_rmat_permute(v, 12, 11) for v in range(nv)])
    assert len(np.unique(perm)) == nv
    # skew: R-MAT(0.57, 0.19, 0.19) concentrates out-degree
    deg = np.diff(rp.astype(np.int64))
    assert deg.max() > 20 * deg.mean()


def test_oracle_simrank_is_the_apps_float_loop(oracle):
    """gwo_simrank restates SimRank::computeResult (apps/simrank.cpp:71-84):
    its float estimate equals the app's loop run on the reference engine's
    golden paths, bit for bit, and its meeting counts rebuild that estimate."""
    g = load_golden("rmat10")
    R, L = 20, 11
    gp = g["simrank_paths"]
    for a, b in [(7, 9), (9, 7), (7, 7)]:
        fa, fb = gp[a], gp[b]
        sim = np.float32(0.0)
        meet = np.zeros(L, np.uint64)
        for i in range(R):
            for j in range(R):
                for l in range(L):
                    if fa[i * L + l] == fb[j * L + l] and fa[i * L + l] != 0xFFFFFFFF:
                        sim = np.float32(float(sim) + (1.0 / (R * R)) * 0.8 ** l)
                        meet[l] += 1
                        break
        est, m = oracle.simrank(fa.reshape(R, L), fb.reshape(R, L), R, L)
        assert np.float32(est) == sim, (a, b)
        assert np.array_equal(m, meet)


def test_oracle_converter_is_the_references(oracle):
    """gwo_convert_text restates convert_to_csr (conversions.hpp:181-291): on
    every golden edge list it builds the row pointer and column array the
    reference's own preprocessor wrote, and compute_blocks gives its block
    range (compute_block, conversions.hpp:293-359)."""
    g = np.load(Path(__file__).parent / "golden" / "convert.npz")
    kb = int(g["blocksize_kb"])
    for case in g["cases"]:
        rp, ci = oracle.convert_text(g[f"{case}_text"].tobytes())
        assert np.array_equal(rp, g[f"{case}_beg_pos"]), case
        assert np.array_equal(ci, g[f"{case}_csr"]), case
        assert g[f"{case}_nvertices"].tobytes() == f"{len(rp) - 1}\n".encode()
        assert np.array_equal(oracle.compute_blocks(rp, kb), g[f"{case}_blockrange"]), case


@pytest.mark.parametrize("text,line", [(b"0 1\n\n1 2\n", 2), (b"0 1\n7\n", 2), (b"0 1\r\n\r\n", 2),
                                       (b"# x\n" + b"1 " * 600 + b"\n", 2)])
def test_oracle_converter_rejects_what_the_reference_rejects(oracle, text, line):
    """An empty line or a one-token line has no second token (the reference
    asserts, conversions.hpp:226-233); an over-long line would be split by fgets."""
    with pytest.raises(ValueError, match=f"line {line} "):
        oracle.convert_text(text)


def _restart_walk_literal(oracle, rp, ci, src, walk_id, nsteps, seed):
    """RandomWalkwithRestart::updateByWalk (randomwalkwithrestart.hpp:40-51),
    restated hop by hop in Python: updateInfo, then the test draw (only when
    the vertex has out-edges), then the neighbour draw; on failure or at a
    dangling vertex back to the source; nsteps visits."""
    thr = oracle.continue_threshold(0.15)
    key = [seed & 0xFFFFFFFF, seed >> 32]
    v, visits = src, []
    for hop in range(nsteps):
        visits.append(v)
        d = [w >> 1 for w in oracle.philox([walk_id, hop, 0, 0], key)]
        deg = int(rp[v + 1] - rp[v])
        if deg > 0 and d[0] >= thr:
            v = int(ci[int(rp[v]) + d[1] % deg])
        else:
            v = src
    return visits


def test_restart_class_is_the_restart_rule_one_segment_longer(oracle):
    """The revived apps' walk class (RandomWalkwithRestart, nsteps visits from
    hop 0) runs on the engine as the restart rule with segment length
    nsteps + 1: per-walk visits equal the literal hop loop's."""
    g = load_golden("hand")
    rp, ci = g["rowptr"], g["colidx"]
    nv = len(rp) - 1
    seed, nsteps = 0x5EED, 7
    for src in range(nv):
        ids = np.arange(40, dtype=np.uint32) + 1000 * src
        cur = np.full(len(ids), src, np.uint32)
        r = oracle.run_walks(rp, ci, cur, ids=ids, src=cur, rule=oracle.RULE_RESTART, L=nsteps + 1, seed=seed,
                             stride=nsteps + 1)
        assert r["status"] == 0
        for w, wid in enumerate(ids):
            want = _restart_walk_literal(oracle, rp, ci, src, int(wid), nsteps, seed)
            assert int(r["plen"][w]) == nsteps
            assert r["paths"][w][:nsteps].tolist() == want
