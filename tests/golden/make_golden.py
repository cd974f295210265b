"""Generates the golden fixtures in tests/golden/*.npz from the reference.

Runs GraphWalker's own engine and walk classes -- compiled from the reference
sources by oracle/Makefile (`make -C oracle ref`) with the Philox rand_r shim
of oracle/ref_shim/gw_ref_shim.cpp -- on small graphs written in the
reference's preprocessed on-disk format, and stores graph, block range (as
the reference's compute_block wrote it), start walks and results.

The graphs: a hand-made 12-vertex graph (a dangling vertex, a vertex whose
out-degree alone exceeds the block budget, an isolated last vertex) and
seeded R-MAT graphs at scales 10 and 13 (the scale-13 pools exceed the
reference's 4096-walk buffers, so its spill-to-disk path runs).

    python tests/golden/make_golden.py          (needs the reference tree)
"""
from __future__ import annotations

import os
import struct
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import py_oracle  # noqa: E402

OUT = Path(__file__).resolve().parent
SHIM = {0: "gw_ref_shim_0", 1: "gw_ref_shim_1", 2: "gw_ref_shim_2", 3: "gw_ref_shim_3"}
SEED = 0x5EED0000000042


def encode(s, c, h):
    s = np.asarray(s, np.uint64) & np.uint64(0xFFFFFF)
    c = np.asarray(c, np.uint64) & np.uint64(0x3FFFFFF)
    h = np.asarray(h, np.uint64) & np.uint64(0x3FFF)
    return (s << np.uint64(40)) | (c << np.uint64(14)) | h


def write_ref_graph(base: Path, rowptr, colidx):
    """The reference's preprocessed layout, without a block range: the
    reference computes and writes that itself (convert_if_notexists)."""
    d = Path(str(base) + "_GraphWalker")
    (d / "graphinfo").mkdir(parents=True, exist_ok=True)
    np.asarray(rowptr, np.uint64).tofile(d / "graphinfo" / "file_0.beg_pos")
    np.asarray(colidx, np.uint32).tofile(d / "graphinfo" / "file_0.csr")
    nv = len(rowptr) - 1
    (d / "filesize_1024GB.filerange").write_text(f"0\n{nv}\n")
    (d / "N.nvertices").write_text(f"{nv}\n")


def run_shim(rule, base: Path, blocksize_kb, walks_blocks, walks_words, L, njump, nmblocks, prob,
             nkeys, stride, threads, cwd: Path):
    wf = cwd / "walks.bin"
    with open(wf, "wb") as f:
        f.write(struct.pack("<Q", len(walks_words)))
        rec = np.zeros(len(walks_words), dtype=[("b", "<u4"), ("pad", "<u4"), ("w", "<u8")])
        rec["b"] = walks_blocks
        rec["w"] = walks_words
        f.write(rec.tobytes())
    of = cwd / "out.bin"
    cmd = [str(py_oracle.REF_DIR / SHIM[rule]), str(base), str(blocksize_kb), str(wf), str(of), str(L),
           f"{SEED:x}", str(njump), str(nmblocks), str(prob), str(nkeys), str(stride),
           "execthreads", str(threads)]
    subprocess.run(cmd, cwd=cwd, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    raw = of.read_bytes()
    st, nv = struct.unpack_from("<II", raw, 0)
    counts = np.frombuffer(raw, np.uint32, nv, 8).copy()
    paths = np.frombuffer(raw, np.uint32, nkeys * stride, 8 + 4 * nv).copy().reshape(nkeys, stride)
    closure = struct.unpack_from("<Q", raw, 8 + 4 * nv + 4 * nkeys * stride)[0]
    return st, counts, paths, closure


def hand_graph():
    adj = {0: [1, 2, 5], 1: [2, 5], 2: [0, 3, 5], 3: [], 4: [5, 0],
           5: [[0, 1, 2, 4, 6, 7, 8, 9, 10][i % 9] for i in range(300)],
           6: [7], 7: [8, 5], 8: [9, 6], 9: [10, 5], 10: [5, 0], 11: []}
    rowptr = np.zeros(13, np.uint64)
    cols = []
    for v in range(12):
        cols += adj[v]
        rowptr[v + 1] = len(cols)
    return rowptr, np.array(cols, np.uint32)


def reference_blocks(tmp: Path, base: Path, blocksize_kb: int) -> np.ndarray:
    # an empty walk set: the reference computes the block range and exits
    run_shim(1, base, blocksize_kb, np.zeros(0, np.uint32), np.zeros(0, np.uint64), 1, 1, 0, 0.2, 1, 1, 1, tmp)
    txt = (Path(str(base) + "_GraphWalker") / f"blocksize_{blocksize_kb}KB.blockrange").read_text()
    return np.array([int(x) for x in txt.split()], np.uint32)


def make_case(name, rowptr, colidx, blocksize_kb, runs):
    with tempfile.TemporaryDirectory() as td:
        tmp = Path(td)
        (tmp / "conf").mkdir()
        (tmp / "conf" / "graphwalker.cnf").write_text("# empty\n")
        base = tmp / name
        write_ref_graph(base, rowptr, colidx)
        blocks = reference_blocks(tmp, base, blocksize_kb)
        nv = len(rowptr) - 1
        out = {"rowptr": rowptr, "colidx": colidx, "blocks": blocks, "blocksize_kb": blocksize_kb,
               "seed": SEED}
        for r in runs:
            tag = r["tag"]
            cur = np.asarray(r["cur"], np.uint32)
            src = np.asarray(r.get("src", cur), np.uint32)
            hop = np.asarray(r.get("hop", np.zeros(len(cur), np.uint32)), np.uint32)
            blk = np.searchsorted(blocks[1:], cur, side="right").astype(np.uint32)
            words = encode(src, cur - blocks[blk], hop)
            results = []
            for nmb, prob, thr in r.get("schedules", [(0, 0.2, 4)]):
                results.append(run_shim(r["rule"], base, blocksize_kb, blk, words, r["L"], nv, nmb, prob,
                                        r["nkeys"], r["stride"], thr, tmp))
            st, counts, paths, closure = results[0]
            for other in results[1:]:  # the shimmed reference is schedule-invariant
                assert other[0] == st and np.array_equal(other[1], counts)
                assert np.array_equal(other[2], paths) and other[3] == closure
            assert st == 0, f"{name}/{tag}: shim status {st}"
            out.update({f"{tag}_rule": r["rule"], f"{tag}_L": r["L"], f"{tag}_cur": cur,
                        f"{tag}_src": src, f"{tag}_hop": hop, f"{tag}_counts": counts,
                        f"{tag}_paths": paths, f"{tag}_closure": closure})
        np.savez_compressed(OUT / f"{name}.npz", **out)
        print(f"{name}: nv={nv} ne={len(colidx)} blocks={len(blocks) - 1} runs={[r['tag'] for r in runs]}")


def main():
    if not (py_oracle.REF_DIR / SHIM[0]).exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref"], check=True)
    py_oracle.build()

    rp, ci = hand_graph()
    allv = np.arange(12, dtype=np.uint32)
    make_case("hand", rp, ci, 1, [
        dict(tag="jump", rule=0, L=10, cur=allv, nkeys=12, stride=10,
             schedules=[(0, 0.2, 4), (2, 1.0, 1), (1, 0.0, 3)]),
        dict(tag="stop", rule=1, L=10, cur=allv, nkeys=12, stride=10),
        dict(tag="prob", rule=2, L=10, cur=allv, nkeys=12, stride=64),
        dict(tag="restart", rule=3, L=5, cur=allv, nkeys=12, stride=5),
    ])

    rp, ci = py_oracle.rmat_csr(10, 16, seed=1)
    v = np.arange(1 << 10, dtype=np.uint32)
    a, b = 7, 9
    R, Ls = 20, 11
    make_case("rmat10", rp, ci, 8, [
        dict(tag="jump", rule=0, L=10, cur=v, nkeys=1 << 10, stride=10,
             schedules=[(0, 0.2, 4), (3, 0.5, 2)]),
        dict(tag="stop", rule=1, L=10, cur=v, nkeys=1 << 10, stride=10),
        dict(tag="prob", rule=2, L=10, cur=v, nkeys=1 << 10, stride=64),
        dict(tag="restart", rule=3, L=6, cur=v, nkeys=1 << 10, stride=6),
        # simrank placement (apps/simrank.cpp:30-57): replica i starts at hop i*L
        dict(tag="simrank", rule=3, L=Ls, cur=np.r_[np.full(R, a), np.full(R, b)].astype(np.uint32),
             hop=np.r_[np.arange(R) * Ls, np.arange(R) * Ls].astype(np.uint32), nkeys=b + 1, stride=R * Ls),
    ])

    rp, ci = py_oracle.rmat_csr(13, 8, seed=3)
    v = np.arange(1 << 13, dtype=np.uint32)
    make_case("rmat13", rp, ci, 128, [
        dict(tag="jump", rule=0, L=10, cur=v, nkeys=1 << 13, stride=10,
             schedules=[(1, 0.2, 4), (0, 0.0, 8)]),
        dict(tag="stop", rule=1, L=10, cur=v, nkeys=1 << 13, stride=10),
    ])


if __name__ == "__main__":
    main()
