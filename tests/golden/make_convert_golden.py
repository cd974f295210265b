"""Generates tests/golden/convert.npz: text edge lists and the files the
reference's own preprocessor writes for them.

The preprocessor is convert_if_notexists (convert_to_csr + compute_block,
src/preprocess/conversions.hpp:181-404), compiled unmodified from the
reference tree by oracle/Makefile (`make -C oracle ref` -> oracle/_ref/gw_ref_convert).
The reference reads lines with fgets, splits them with strtok on tab, comma
and space, converts with atoi, skips '#'/'%' comment lines and self-loops,
keeps duplicate edges, and expects the lines grouped by ascending source, so
every case here is source-ordered.

    python tests/golden/make_convert_golden.py          (needs the reference tree)
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import py_oracle  # noqa: E402

OUT = Path(__file__).resolve().parent
BLOCKSIZE_KB = 1  # 256 edges per block, so the small cases have several blocks


def edge_cases() -> bytes:
    lines = [
        "# a comment line",
        "% another comment",
        "0 1", "0\t2", "0,3", "0 , 4", "  0 5", ",\t0\t6", "0 1",       # separators, a duplicate
        " # 0",                   # not a comment (the '#' is not first): atoi("#") = atoi("0") = 0, a self-loop
        "0 0",                    # self-loop
        "1 9",                    # vertices 2..3 get no out-edges
        "4 007", "4 +8", "4 12abc", "\v4 \f10",   # leading zeros, '+', trailing garbage, other whitespace
        "4 4294967297",           # atoi keeps the low 32 bits of strtol: 1
        "4 5 6 7",                # tokens after the second are ignored
        "9 2\r",                  # CRLF line ending
        "11 0",
        "11 30",                  # the last vertex only appears as a target
    ]
    return ("\n".join(lines) + "\n").encode()


def gaps_case() -> bytes:
    return b"5 6\n5 7\n100 3\n100 101\n250 0\n"


def comments_only() -> bytes:
    return b"# nothing here\n% still nothing\n"


def no_final_newline() -> bytes:
    return b"0 1\n1 2\n2 0"


def rmat_case(scale: int, ef: int, seed: int) -> bytes:
    rp, ci = py_oracle.rmat_csr(scale, ef, seed=seed)
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(len(rp) - 1), np.diff(rp.astype(np.int64)))
    # put back some self-loops (the reference drops them) and mix separators
    extra = rng.choice(len(src), len(src) // 50, replace=False)
    seps = np.array([" ", "\t", ",", " , "])
    out = []
    j = 0
    loops = set(extra.tolist())
    for i, (s, d) in enumerate(zip(src.tolist(), ci.tolist())):
        out.append(f"{s}{seps[i % 4]}{d}\n")
        if i in loops:
            out.append(f"{s} {s}\n")
        j += 1
    return ("# rmat\n" + "".join(out)).encode()


CASES = {
    "edge_cases": edge_cases,
    "gaps": gaps_case,
    "comments_only": comments_only,
    "no_final_newline": no_final_newline,
    "rmat10": lambda: rmat_case(10, 8, 3),
    "rmat13": lambda: rmat_case(13, 8, 5),
}


def run_reference(text: bytes, tmp: Path) -> dict:
    exe = ROOT / "oracle" / "_ref" / "gw_ref_convert"
    if not exe.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "_ref/gw_ref_convert"], check=True)
    f = tmp / "g.txt"
    f.write_bytes(text)
    subprocess.run([str(exe), str(f), str(BLOCKSIZE_KB)], check=True, capture_output=True)
    d = Path(str(f) + "_GraphWalker")
    return {
        "beg_pos": np.fromfile(d / "graphinfo" / "file_0.beg_pos", np.uint64),
        "csr": np.fromfile(d / "graphinfo" / "file_0.csr", np.uint32),
        "blockrange": np.array((d / f"blocksize_{BLOCKSIZE_KB}KB.blockrange").read_text().split(), np.uint32),
        "filerange": np.frombuffer((d / "filesize_1024GB.filerange").read_bytes(), np.uint8),
        "nvertices": np.frombuffer((d / "N.nvertices").read_bytes(), np.uint8),
    }


def main() -> None:
    out = {"blocksize_kb": np.array(BLOCKSIZE_KB)}
    for name, make in CASES.items():
        text = make()
        with tempfile.TemporaryDirectory() as td:
            r = run_reference(text, Path(td))
        out[f"{name}_text"] = np.frombuffer(text, np.uint8)
        for k, v in r.items():
            out[f"{name}_{k}"] = v
        print(f"{name}: {len(text)} bytes, nv={len(r['beg_pos']) - 1}, ne={len(r['csr'])}, "
              f"blocks={len(r['blockrange']) - 1}")
    np.savez_compressed(OUT / "convert.npz", cases=np.array(list(CASES)), **out)


if __name__ == "__main__":
    main()
