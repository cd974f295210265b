"""GraphWalker's preprocessed on-disk graph format (reader and writer).

Files under `<base>_GraphWalker/` (src/api/filename.hpp:16-51):
  graphinfo/file_0.beg_pos          uint64 row pointer, nvertices + 1 entries
  graphinfo/file_0.csr              uint32 column ids
  filesize_1024GB.filerange         "0\\n<nvertices>\\n" (one CSR file)
  N.nvertices                       "<nvertices>\\n"
  blocksize_<KB>KB.blockrange       block boundaries, one per line
This is what convert_to_csr / compute_block write (conversions.hpp:127-141,
181-364); a directory written here is taken as already preprocessed by the
reference's convert_if_notexists (conversions.hpp:371-404).
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

from .engine import compute_blocks

FILE_SIZE_GB = 1024  # FILE_SIZE, src/api/datatype.hpp:9


def graph_dir(base: str) -> Path:
    return Path(base + "_GraphWalker")


def blockrange_path(base: str, blocksize_kb: int) -> Path:
    return graph_dir(base) / f"blocksize_{blocksize_kb}KB.blockrange"


def write_graph(base: str, rowptr: np.ndarray, colidx: np.ndarray,
                blocksize_kb: int | None = None, write_blockrange: bool = True) -> np.ndarray | None:
    """Writes the CSR in the reference's preprocessed layout; returns the blocks."""
    d = graph_dir(base)
    (d / "graphinfo").mkdir(parents=True, exist_ok=True)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    colidx = np.ascontiguousarray(colidx, dtype=np.uint32)
    nv = len(rowptr) - 1
    rowptr.tofile(d / "graphinfo" / "file_0.beg_pos")
    colidx.tofile(d / "graphinfo" / "file_0.csr")
    (d / f"filesize_{FILE_SIZE_GB}GB.filerange").write_text(f"0\n{nv}\n")
    (d / "N.nvertices").write_text(f"{nv}\n")
    os.makedirs(d / "walks", exist_ok=True)
    if blocksize_kb is None or not write_blockrange:
        return None
    blocks = compute_blocks(rowptr, blocksize_kb)
    blockrange_path(base, blocksize_kb).write_text("".join(f"{int(b)}\n" for b in blocks))
    return blocks


def read_graph(base: str) -> tuple[np.ndarray, np.ndarray]:
    d = graph_dir(base) / "graphinfo"
    return (np.fromfile(d / "file_0.beg_pos", dtype=np.uint64),
            np.fromfile(d / "file_0.csr", dtype=np.uint32))


def read_blocks(base: str, blocksize_kb: int) -> np.ndarray:
    txt = blockrange_path(base, blocksize_kb).read_text().split()
    return np.array([int(x) for x in txt], dtype=np.uint32)


def blocksize_for(nedges: int, nblocks: int) -> int:
    """A blocksize_kb whose compute_block budget yields about `nblocks` blocks."""
    per_block_edges = -(-nedges // nblocks)
    return max(1, -(-per_block_edges * 4 // 1024))
