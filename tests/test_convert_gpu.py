"""The device graph preprocessor (gw_convert_edgelist) against the reference's
own preprocessor (golden files from tests/golden/make_convert_golden.py) and
against the oracle's restatement of convert_to_csr.

The files are integers and bytes: they must match exactly."""
import os
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = np.load(Path(__file__).parent / "golden" / "convert.npz")
KB = int(GOLD["blocksize_kb"])


def _convert(tmp_path, text: bytes, kb=KB, name="g.txt"):
    import graphwalker_b200 as gw
    f = tmp_path / name
    f.write_bytes(text)
    st = gw.convert_edgelist(str(f), kb)
    d = Path(str(f) + "_GraphWalker")
    out = {
        "beg_pos": np.fromfile(d / "graphinfo" / "file_0.beg_pos", np.uint64),
        "csr": np.fromfile(d / "graphinfo" / "file_0.csr", np.uint32),
        "filerange": (d / "filesize_1024GB.filerange").read_bytes(),
        "nvertices": (d / "N.nvertices").read_bytes(),
    }
    if kb:
        out["blockrange"] = np.array((d / f"blocksize_{kb}KB.blockrange").read_text().split(), np.uint32)
    return out, st


@pytest.fixture(params=[None, "4096"], ids=["one_chunk", "4k_chunks"])
def chunking(request, monkeypatch):
    """The whole file in one device round, or 4 KiB rounds (lines cross
    chunk boundaries and are carried over)."""
    if request.param:
        monkeypatch.setenv("GW_CONVERT_CHUNK_BYTES", request.param)
    else:
        monkeypatch.delenv("GW_CONVERT_CHUNK_BYTES", raising=False)
    return request.param


@pytest.mark.parametrize("case", [str(c) for c in GOLD["cases"]])
def test_files_equal_the_reference_preprocessor(cuda_device, tmp_path, chunking, case):
    out, st = _convert(tmp_path, GOLD[f"{case}_text"].tobytes())
    assert np.array_equal(out["beg_pos"], GOLD[f"{case}_beg_pos"])
    assert np.array_equal(out["csr"], GOLD[f"{case}_csr"])
    assert out["filerange"] == GOLD[f"{case}_filerange"].tobytes()
    assert out["nvertices"] == GOLD[f"{case}_nvertices"].tobytes()
    assert np.array_equal(out["blockrange"], GOLD[f"{case}_blockrange"])
    assert st.edges == len(GOLD[f"{case}_csr"]) and st.nvertices == len(GOLD[f"{case}_beg_pos"]) - 1
    assert st.sorted == 1


def test_unsorted_lists_are_grouped_stably(cuda_device, oracle, tmp_path, chunking):
    """Lines not grouped by source (the reference needs them grouped): each
    source keeps its edges in file order, as the oracle's stable sort does."""
    rng = np.random.default_rng(11)
    n = 20000
    src = rng.integers(0, 3000, n)
    dst = rng.integers(0, 5000, n)
    seps = np.array([" ", "\t", ",", " , "])[rng.integers(0, 4, n)]
    text = "".join(f"{a}{s}{b}\n" for a, s, b in zip(src, seps, dst)).encode()
    ref_rp, ref_ci = oracle.convert_text(text)
    out, st = _convert(tmp_path, text, kb=4)
    assert st.sorted == 0
    assert np.array_equal(out["beg_pos"], ref_rp)
    assert np.array_equal(out["csr"], ref_ci)
    assert np.array_equal(out["blockrange"], oracle.compute_blocks(ref_rp, 4))


def test_large_rmat_list_matches_oracle(cuda_device, oracle, tmp_path):
    """A scale-16 R-MAT edge list (1 M lines) in 64 KiB rounds."""
    rp, ci = oracle.rmat_csr(16, 16, seed=9)
    src = np.repeat(np.arange(len(rp) - 1), np.diff(rp.astype(np.int64)))
    text = "\n".join(f"{a} {b}" for a, b in zip(src.tolist(), ci.tolist())).encode() + b"\n"
    os.environ["GW_CONVERT_CHUNK_BYTES"] = str(64 << 10)
    try:
        out, st = _convert(tmp_path, text, kb=256)
    finally:
        del os.environ["GW_CONVERT_CHUNK_BYTES"]
    # a text list knows vertices up to the largest id it names, as the reference does
    ref_rp, ref_ci = oracle.convert_text(text)
    assert np.array_equal(out["beg_pos"], ref_rp) and np.array_equal(out["csr"], ref_ci)
    assert np.array_equal(ref_rp, rp[: len(ref_rp)]) and np.array_equal(ref_ci, ci)
    assert np.array_equal(out["blockrange"], oracle.compute_blocks(ref_rp, 256))
    assert st.lines == len(ci) and st.bytes == len(text)


@pytest.mark.parametrize("text,line", [(b"0 1\n\n1 2\n", 2), (b"0 1\n7\n", 2), (b"0 1\r\n\r\n", 2),
                                       (b"# x\n" + b"1 " * 600 + b"\n", 2)])
def test_rejected_lines_are_named(cuda_device, tmp_path, text, line):
    import graphwalker_b200 as gw
    with pytest.raises(gw.GwError, match=f"line {line} "):
        _convert(tmp_path, text)


def test_converted_graph_opens_and_walks(cuda_device, oracle, tmp_path):
    """The converted files are the engine's graph input: gw_open on them
    gives the oracle's walks."""
    import graphwalker_b200 as gw
    text = GOLD["rmat10_text"].tobytes()
    _convert(tmp_path, text, kb=KB)
    rp, ci = oracle.convert_text(text)
    with gw.Graph.open(str(tmp_path / "g.txt"), KB) as G:
        nv = G.nv
        cur = np.arange(nv, dtype=np.uint32)
        ref = oracle.run_walks(rp, ci, cur, ids=cur, src=cur, rule=0, L=10, seed=3)
        G.add_walks_at(cur)
        G.run(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, 10, seed=3))
        assert np.array_equal(G.read_counts(), ref["counts"])
