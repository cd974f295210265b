"""The drop-in C++ API (graphwalker_b200/compat): GraphWalker programs compile
unchanged against it, and a program written against GraphWalker's API,
running on the B200 engine, receives in its updateInfo exactly the visits
the reference engine delivers (golden vectors, Philox-keyed draws)."""
import os
import re
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, golden_runs, load_golden
from oracle.refpath import REFERENCE

COMPAT = ROOT / "graphwalker_b200" / "compat"
APPS_DIR = COMPAT / "_apps"
REFERENCE_APPS = REFERENCE / "apps"
LIVE_APPS = ["rwdomination", "rawrandomwalks", "msppr", "kk_ppr", "graphlet", "simrank"]


def build_compat_app(rule: int, out: Path) -> Path:
    subprocess.run(["make", "-s", "-C", str(COMPAT), "app", f"SRC={ROOT / 'tests' / 'compat' / 'gw_compat_app.cpp'}",
                    f"OUT={out}", f"DEFS=-DGW_APP_RULE={rule}"], check=True)
    return out


@pytest.mark.skipif(not REFERENCE_APPS.is_dir(), reason="needs the reference's apps/ sources")
def test_reference_apps_compile_unchanged():
    subprocess.run(["make", "-s", "-C", str(COMPAT), "apps", f"REF={REFERENCE_APPS.parent}"], check=True)
    for app in LIVE_APPS:
        assert (APPS_DIR / app).exists(), app


def test_compat_program_compiles(tmp_path):
    for rule in range(4):
        assert build_compat_app(rule, tmp_path / f"app{rule}").exists()


def _prepare(tmp: Path, g: dict, name: str) -> str:
    from graphwalker_b200 import formats
    (tmp / "conf").mkdir(exist_ok=True)
    (tmp / "conf" / "graphwalker.cnf").write_text("# empty\n")
    base = str(tmp / name)
    formats.write_graph(base, g["rowptr"], g["colidx"], int(g["blocksize_kb"]))
    return base


def _walks_file(path: Path, g: dict, tag: str):
    import graphwalker_b200 as gw
    cur, src, hop = g[f"{tag}_cur"], g[f"{tag}_src"], g[f"{tag}_hop"]
    blocks = g["blocks"]
    blk = np.searchsorted(blocks[1:], cur, side="right").astype(np.uint32)
    rec = np.zeros(len(cur), dtype=[("b", "<u4"), ("pad", "<u4"), ("w", "<u8")])
    rec["b"] = blk
    rec["w"] = gw.encode(src, cur - blocks[blk], hop)
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", len(cur)))
        f.write(rec.tobytes())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["hand", "rmat10", "rmat13"])
def test_compat_program_matches_reference_goldens(cuda_device, case, tmp_path):
    g = load_golden(case)
    base = _prepare(tmp_path, g, case)
    nv = len(g["rowptr"]) - 1
    bins = {}
    for tag in golden_runs(g):
        rule, L = int(g[f"{tag}_rule"]), int(g[f"{tag}_L"])
        if rule not in bins:
            bins[rule] = build_compat_app(rule, tmp_path / f"app{rule}")
        gp = g[f"{tag}_paths"]
        nkeys, stride = gp.shape
        _walks_file(tmp_path / "walks.bin", g, tag)
        out = tmp_path / "out.bin"
        subprocess.run([str(bins[rule]), base, str(int(g["blocksize_kb"])), str(tmp_path / "walks.bin"), str(out),
                        str(L), str(int(g["seed"])), str(nv), str(nkeys), str(stride),
                        "gw_walk_id", "source", "seed", str(int(g["seed"]))],
                       cwd=tmp_path, check=True, capture_output=True)
        raw = out.read_bytes()
        counts = np.frombuffer(raw, np.uint32, nv, 8)
        paths = np.frombuffer(raw, np.uint32, nkeys * stride, 8 + 4 * nv).reshape(nkeys, stride)
        closure = struct.unpack_from("<Q", raw, 8 + 4 * nv + 4 * nkeys * stride)[0]
        assert np.array_equal(counts, g[f"{tag}_counts"]), f"{case}/{tag}"
        assert np.array_equal(paths, gp), f"{case}/{tag} paths"
        assert closure == int(g[f"{tag}_closure"])


@pytest.mark.gpu
@pytest.mark.parametrize("mapped", ["0", "auto", "1000000"])
def test_compat_streamed_block_loop_counts(cuda_device, mapped, tmp_path):
    """The knobs of the streamed block loop through the drop-in engine
    (gw_mode blocked, gw_residency stream, gw_mapped_walks, gw_sink count):
    the program's counts equal the reference engine's goldens whether blocks
    are copied into slots or read in place."""
    g = load_golden("rmat13")
    base = _prepare(tmp_path, g, "rmat13")
    nv = len(g["rowptr"]) - 1
    app = build_compat_app(0, tmp_path / "app0")
    for tag in golden_runs(g):
        if int(g[f"{tag}_rule"]) != 0:
            continue
        _walks_file(tmp_path / "walks.bin", g, tag)
        out = tmp_path / "out.bin"
        r = subprocess.run([str(app), base, str(int(g["blocksize_kb"])), str(tmp_path / "walks.bin"), str(out),
                            str(int(g[f"{tag}_L"])), str(int(g["seed"])), str(nv), "1", "1",
                            "gw_walk_id", "source", "seed", str(int(g["seed"])), "gw_mode", "blocked",
                            "gw_residency", "stream", "gw_mapped_walks", mapped, "gw_sink", "count",
                            "gw_pool_budget_mb", "1"],
                           cwd=tmp_path, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
        counts = np.frombuffer(out.read_bytes(), np.uint32, nv, 8)
        assert np.array_equal(counts, g[f"{tag}_counts"]), f"{tag}/{mapped}"
        metrics = "".join(p.read_text() for p in tmp_path.glob("*metrics.txt"))
        in_place = int(float(re.search(r"gpu_blocks_read_in_place\D*?([\d.]+)", metrics).group(1)))
        if mapped == "0":
            assert in_place == 0, metrics[-500:]
        elif mapped == "1000000":  # every block in place: none is ever copied
            assert in_place > 0, metrics[-500:]


def _run_app(app: str, args: list[str], cwd: Path) -> subprocess.CompletedProcess:
    exe = APPS_DIR / app
    if not exe.exists():
        pytest.skip(f"{exe} not built (make -C graphwalker_b200/compat apps)")
    return subprocess.run([str(exe), *args], cwd=cwd, capture_output=True, text=True, timeout=300)


@pytest.mark.gpu
def test_unchanged_simrank_app(cuda_device, tmp_path):
    """apps/simrank.cpp, unchanged, on the B200 engine: its SimRank equals the
    value computed from the reference engine's golden walk paths."""
    g = load_golden("rmat10")
    base = _prepare(tmp_path, g, "rmat10")
    a, b, R, L = 7, 9, 20, 11
    r = _run_app("simrank", ["file", base, "a", str(a), "b", str(b), "R", str(R), "L", str(L),
                             "blocksize_kb", str(int(g["blocksize_kb"])), "gw_walk_id", "source",
                             "seed", str(int(g["seed"]))], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    got = float(re.search(r"SimRank for \d+ and \d+ = (\S+)", r.stdout).group(1))
    gp = g["simrank_paths"]
    fa, fb = gp[a], gp[b]
    sim = np.float32(0.0)
    for i in range(R):
        for j in range(R):
            for l in range(L):
                if fa[i * L + l] == fb[j * L + l] and fa[i * L + l] != 0xFFFFFFFF:
                    sim = np.float32(float(sim) + (1.0 / (R * R)) * 0.8 ** l)
                    break
    assert got == pytest.approx(float(sim), rel=1e-5, abs=1e-7)


@pytest.mark.gpu
def test_unchanged_rwdomination_graphlet_kkppr_apps(cuda_device, tmp_path):
    g = load_golden("rmat10")
    base = _prepare(tmp_path, g, "rmat10")
    kb = str(int(g["blocksize_kb"]))
    r = _run_app("rwdomination", ["file", base, "N", "1024", "R", "2", "L", "10", "blocksize_kb", kb], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    metrics = (tmp_path / "graphwalker_metrics.txt").read_text()
    assert "00_runtime=" in metrics and "5_exec_updates=" in metrics
    assert "gpu_walks" in metrics and "gpu_ms_walk" in metrics  # the device's counters beside the reference's timers
    assert (tmp_path / "graphwalker_metrics.txt.statistics").read_text().strip()
    r = _run_app("graphlet", ["file", base, "N", "1024", "R", "5000", "L", "4", "blocksize_kb", kb], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "cnt_all:\t5000" in r.stdout
    ok = int(re.search(r"cnt_ok:\t(\d+)", r.stdout).group(1))
    assert 0 <= ok <= 5000
    r = _run_app("kk_ppr", ["file", base, "firstsource", "3", "numsources", "4", "walkspersource", "500",
                            "blocksize_kb", kb], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    r = _run_app("rawrandomwalks", ["file", base, "N", "1024", "R", "3000", "L", "6", "blocksize_kb", kb], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.gpu
def test_unchanged_app_preprocesses_a_text_edge_list(cuda_device, tmp_path):
    """apps/rwdomination.cpp, unchanged, given a text edge list with no
    preprocessed files: its convert_if_notexists call runs the GPU converter,
    which writes exactly the files the reference's preprocessor writes."""
    gold = np.load(ROOT / "tests" / "golden" / "convert.npz")
    (tmp_path / "conf").mkdir()
    (tmp_path / "conf" / "graphwalker.cnf").write_text("# empty\n")
    text = tmp_path / "g.txt"
    text.write_bytes(gold["rmat10_text"].tobytes())
    kb = int(gold["blocksize_kb"])
    r = _run_app("rwdomination", ["file", str(text), "N", "1024", "R", "1", "L", "5", "blocksize_kb", str(kb)],
                 tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    d = Path(str(text) + "_GraphWalker")
    assert np.array_equal(np.fromfile(d / "graphinfo" / "file_0.beg_pos", np.uint64), gold["rmat10_beg_pos"])
    assert np.array_equal(np.fromfile(d / "graphinfo" / "file_0.csr", np.uint32), gold["rmat10_csr"])
    br = np.array((d / f"blocksize_{kb}KB.blockrange").read_text().split(), np.uint32)
    assert np.array_equal(br, gold["rmat10_blockrange"])


def _run_revived(app: str, args: list[str], cwd: Path) -> subprocess.CompletedProcess:
    exe = APPS_DIR / app
    if not exe.exists():
        subprocess.run(["make", "-s", "-C", str(COMPAT), "revived"], check=True)
    return subprocess.run([str(exe), *args], cwd=cwd, capture_output=True, text=True, timeout=300)


@pytest.mark.gpu
def test_revived_personalizedpagerank_equals_oracle(cuda_device, oracle, tmp_path):
    """apps/personalizedpagerank.cpp's computation on the live API: R walks
    from `source` (restart at the source on the 0.15 branch and at dangling
    vertices, L visits each), counted per vertex.  The 4B.vvalue file it
    writes equals the oracle's counts for the same walks (walk ids = pool
    positions, Philox seed 42)."""
    g = load_golden("rmat13")
    base = _prepare(tmp_path, g, "rmat13")
    rp, ci = g["rowptr"], g["colidx"]
    nv = len(rp) - 1
    source = int(np.argmax(np.diff(rp.astype(np.int64))))
    R, L = 3000, 10
    r = _run_revived("personalizedpagerank", ["file", base, "nvertices", str(nv), "source", str(source), "R", str(R),
                                              "L", str(L), "shardsize", str(int(g["blocksize_kb"]))], tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    got = np.fromfile(base + "_GraphWalker/4B.vvalue", np.uint32)
    cur = np.full(R, source, np.uint32)
    ref = oracle.run_walks(rp, ci, cur, ids=np.arange(R, dtype=np.uint32), src=cur, rule=oracle.RULE_RESTART,
                           L=L + 1, seed=42)
    assert np.array_equal(got, ref["counts"])
    assert int(got.sum()) == R * L
    # the class accepts only tail = 0, the app's default
    r = _run_revived("personalizedpagerank", ["file", base, "nvertices", str(nv), "source", str(source), "R", "10",
                                              "tail", "0.5", "shardsize", str(int(g["blocksize_kb"]))], tmp_path)
    assert r.returncode != 0


@pytest.mark.gpu
def test_revived_reachability_answers_like_the_oracle(cuda_device, oracle, tmp_path):
    """apps/reachability.cpp's computation on the live API: whether any of R
    walks of L visits from a reaches b, for a b the walks reach and a b they
    do not."""
    g = load_golden("rmat13")
    base = _prepare(tmp_path, g, "rmat13")
    rp, ci = g["rowptr"], g["colidx"]
    a = int(np.argmax(np.diff(rp.astype(np.int64))))
    R, L = 200, 12
    cur = np.full(R, a, np.uint32)
    ref = oracle.run_walks(rp, ci, cur, ids=np.arange(R, dtype=np.uint32), src=cur, rule=oracle.RULE_RESTART,
                           L=L + 1, seed=42)["counts"]
    seen = np.flatnonzero(ref)
    unseen = np.flatnonzero(ref == 0)
    cases = {int(seen[np.argmin(ref[seen])]): 1, int(unseen[0]): 0}
    for b, want in cases.items():
        r = _run_revived("reachability", ["file", base, "a", str(a), "b", str(b), "R", str(R), "L", str(L),
                                          "shardsize", str(int(g["blocksize_kb"]))], tmp_path)
        assert r.returncode == 0, r.stderr[-2000:]
        assert f"Reachability from {a} to {b} = {want}" in r.stdout
