"""The C-ABI library without a GPU: it loads, exports every entry point that
include/graphwalker_b200.h declares, and its host-only functions (codec,
continuation threshold, compute_block, getblock, block sizing) agree with the
oracle and the reference's golden block ranges."""
import ctypes
import re
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_golden


def header_functions(path: Path) -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", path.read_text(), flags=re.S)
    return re.findall(r"^[a-z_][\w \*]*?\b(gw_\w+)\s*\(", text, flags=re.M)


def test_library_exports_every_declared_symbol():
    import graphwalker_b200._lib as L
    lib = L.load()
    declared = header_functions(ROOT / "include" / "graphwalker_b200.h")
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), f"{name} declared but not exported"
        assert name in L.exported_symbols(), f"{name} has no ctypes signature"


def test_product_does_not_reference_the_oracle():
    for f in (ROOT / "graphwalker_b200").rglob("*"):
        if f.suffix in {".py", ".cu", ".cuh", ".h", ".cpp", ".hpp"}:
            txt = f.read_text()
            assert "py_oracle" not in txt and "gw_oracle" not in txt and "gwo_" not in txt, f


def test_codec_and_threshold_match_oracle(oracle):
    import graphwalker_b200 as gw
    lib = gw.load()
    olib = oracle.lib()
    rng = np.random.default_rng(1)
    for _ in range(300):
        s, c, h = (int(x) for x in (rng.integers(0, 2**26), rng.integers(0, 2**27), rng.integers(0, 2**15)))
        assert lib.gw_encode(s, c, h) == olib.gwo_encode(s, c, h)
        w = lib.gw_encode(s, c, h)
        assert lib.gw_get_source(w) == olib.gwo_get_source(w)
        assert lib.gw_get_current(w) == olib.gwo_get_current(w)
        assert lib.gw_get_hop(w) == olib.gwo_get_hop(w)
    words = gw.encode([1, 2**24 - 1], [5, 2**26 - 1], [0, 2**14 - 1])
    assert list(gw.get_source(words)) == [1, 2**24 - 1]
    assert list(gw.get_current(words)) == [5, 2**26 - 1]
    assert list(gw.get_hop(words)) == [0, 2**14 - 1]
    for p in (0.0, 0.15, 0.3, 0.5, 0.85, 1.0):
        assert lib.gw_continue_threshold(p) == oracle.continue_threshold(p)


@pytest.mark.parametrize("case", ["hand", "rmat10", "rmat13"])
def test_compute_blocks_matches_reference(case):
    import graphwalker_b200 as gw
    g = load_golden(case)
    assert np.array_equal(gw.compute_blocks(g["rowptr"], int(g["blocksize_kb"])), g["blocks"])


def test_compute_blocks_edge_cases(oracle):
    import graphwalker_b200 as gw
    # two consecutive vertices whose degrees each exceed the budget (256 edges)
    deg = np.array([3, 300, 400, 1, 0, 2, 700, 0], np.uint64)
    rowptr = np.r_[0, np.cumsum(deg)].astype(np.uint64)
    assert np.array_equal(gw.compute_blocks(rowptr, 1), oracle.compute_blocks(rowptr, 1))
    # no edges at all
    rowptr = np.zeros(6, np.uint64)
    assert list(gw.compute_blocks(rowptr, 4)) == [0, 5]


def test_getblock_and_block_sizing(oracle):
    import graphwalker_b200 as gw
    lib = gw.load()
    blocks = np.array([0, 3, 3, 10, 17], np.uint32)  # includes an empty block
    for v in range(20):
        ref = oracle.lib().gwo_getblock(blocks.ctypes.data, 4, v)
        assert lib.gw_getblock(blocks.ctypes.data, 4, v) == ref
    # RandomWalk::compBlockSize / compNmblocks (randomwalk.hpp:96-114)
    assert lib.gw_comp_block_size(0) == 2048
    assert lib.gw_comp_block_size(9) == 4096
    assert lib.gw_comp_block_size(16777216) == 2**19
    assert lib.gw_comp_nmblocks(2**19, 0) == 44 * 1024 * 1024 // 2**19


def test_reference_format_roundtrip():
    from graphwalker_b200 import formats
    g = load_golden("rmat10")
    with tempfile.TemporaryDirectory() as td:
        base = str(Path(td) / "g")
        blocks = formats.write_graph(base, g["rowptr"], g["colidx"], int(g["blocksize_kb"]))
        assert np.array_equal(blocks, g["blocks"])
        rp, ci = formats.read_graph(base)
        assert np.array_equal(rp, g["rowptr"]) and np.array_equal(ci, g["colidx"])
        assert np.array_equal(formats.read_blocks(base, int(g["blocksize_kb"])), g["blocks"])
        d = Path(base + "_GraphWalker")
        assert (d / "filesize_1024GB.filerange").read_text() == "0\n1024\n"


def test_invalid_arguments_fail_cleanly():
    import graphwalker_b200 as gw
    from graphwalker_b200._lib import GwError
    with pytest.raises(GwError):
        gw.Graph.open("/nonexistent/graph", 1024)


def test_struct_layouts_match_the_header(tmp_path):
    """Every struct of include/graphwalker_b200.h has the same size and field
    offsets in the Python binding (ctypes) as a C compiler gives it."""
    import ctypes
    import subprocess

    from graphwalker_b200 import _lib
    pairs = {"gw_walk_rec": _lib.WalkRec, "gw_walk_params": _lib.WalkParams, "gw_run_stats": _lib.RunStats,
             "gw_graph_desc": _lib.GraphDesc, "gw_ppr_stats": _lib.PprStats, "gw_serve_config": _lib.ServeConfig,
             "gw_serve_timing": _lib.ServeTiming, "gw_serve_stats": _lib.ServeStats,
             "gw_convert_stats": _lib.ConvertStats}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "graphwalker_b200.h"', "int main(void) {"]
    for c, py in pairs.items():
        lines.append(f'  printf("{c} size %zu\\n", sizeof({c}));')
        for name, _ in py._fields_:
            lines.append(f'  printf("{c} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        c, field, v = line.split()
        got[(c, field)] = int(v)
    for c, py in pairs.items():
        assert got[(c, "size")] == ctypes.sizeof(py), c
        for name, _ in py._fields_:
            assert got[(c, name)] == getattr(py, name).offset, (c, name)


def test_close_releases_every_context_buffer():
    """gw_close frees every device and pinned buffer the context struct holds:
    each gw_devbuf / gw_hostbuf member of gw_ctx is named in gw_close."""
    ctx_h = (ROOT / "graphwalker_b200" / "csrc" / "gw_ctx.h").read_text()
    body = re.search(r"struct gw_ctx \{(.*?)\n\};", ctx_h, re.S).group(1)
    code = "\n".join(line.split("//")[0] for line in body.splitlines())
    # the submit/wait pipeline's buffers live in a nested struct, freed by
    # gw::pipe_release, which gw_close calls
    pipe = re.search(r"struct PoolsPipe \{(.*?)\} pipe;", code, re.S)
    code = code.replace(pipe.group(0), "")

    def buffers(text):
        held = set()
        for decl in re.findall(r"\bgw_(?:dev|host)buf\s+([^;(){}]*);", text):
            held |= {name.split("[")[0].strip() for name in decl.split(",")}
        return held

    held = buffers(code)
    capi = (ROOT / "graphwalker_b200" / "csrc" / "gw_capi.cu").read_text()
    start = capi.index("gw_status gw_close(gw_ctx* ctx)")
    close = capi[start:capi.index("\n}\n", start)]
    named = set(re.findall(r"ctx->(\w+)", close))
    assert held and held <= named, sorted(held - named)
    assert "gw::pipe_release(ctx)" in close
    src = (ROOT / "graphwalker_b200" / "csrc" / "gw_pools_async.cu").read_text()
    start = src.index("void pipe_release(gw_ctx* ctx)")
    release = src[start:src.index("\n}\n", start)]
    held_pipe = buffers(pipe.group(1))
    named_pipe = set(re.findall(r"P\.(\w+)", release))
    assert held_pipe and held_pipe <= named_pipe, sorted(held_pipe - named_pipe)
