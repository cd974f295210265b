"""TEST INFRASTRUCTURE ONLY -- Python handle of the C oracle (oracle/gw_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, as the checker.  The product (graphwalker_b200/) never does.

It also restates, in numpy, the reference engine's block loop
(src/engine/graphwalker.hpp:272-311) with the scheduler of
src/walks/walk.hpp:204-252 and a stable (input-ordered) walk pool, for the
parity tests of the device's blocked mode.
"""
from __future__ import annotations

import ctypes
import subprocess
from ctypes import POINTER, Structure, c_double, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "_build" / "libgw_oracle.so"
REF_DIR = ORACLE_DIR / "_ref"

RULE_JUMP, RULE_STOP, RULE_PROB, RULE_RESTART, RULE_PPR = 0, 1, 2, 3, 4
ST_BOUNDS, ST_PATH_OVF, ST_HOP_OVF = 1, 2, 4


class Params(Structure):
    _fields_ = [("rule", c_uint32), ("L", c_uint32), ("jump_prob", c_double), ("njump", c_uint32),
                ("seed", c_uint64), ("max_hops", c_uint32), ("rng", c_uint32)]


def build() -> Path:
    """Compiles the C restatement with gcc (seconds) when it is not built yet."""
    src = ORACLE_DIR / "gw_oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "all"], check=True)
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = c_void_p
        sig = {
            "gwo_philox4x32_10": (None, [P, P, P]),
            "gwo_continue_threshold": (c_uint32, [c_double]),
            "gwo_continue_test": (ctypes.c_int, [c_uint32, c_double]),
            "gwo_threshold_mismatches": (c_uint64, [c_double]),
            "gwo_encode": (c_uint64, [c_uint32, c_uint32, c_uint32]),
            "gwo_get_source": (c_uint32, [c_uint64]),
            "gwo_get_current": (c_uint32, [c_uint64]),
            "gwo_get_hop": (c_uint32, [c_uint64]),
            "gwo_run_walks": (c_uint32, [P, P, c_uint32, P, P, P, P, c_uint64, POINTER(Params), P, P,
                                         c_uint32, P, P, P, P]),
            "gwo_block_step": (c_uint32, [P, P, c_uint32, P, c_uint32, c_uint32, P, P, P, P, c_uint64,
                                          POINTER(Params), P, P]),
            "gwo_compute_blocks": (c_uint32, [P, c_uint32, c_uint64, P, c_uint32]),
            "gwo_getblock": (c_uint32, [P, c_uint32, c_uint32]),
            "gwo_rmat_permute": (c_uint32, [c_uint32, c_uint32, c_uint64]),
            "gwo_rmat_edge": (None, [c_uint64, c_uint32, c_uint64, c_uint32, c_uint32, c_uint32, P, P]),
            "gwo_rmat_csr": (c_uint64, [c_uint32, c_uint64, c_uint64, c_uint32, c_uint32, c_uint32, P, P]),
            "gwo_expected_visits": (None, [P, P, c_uint32, c_uint32, c_uint32, c_uint32, c_double, P]),
            "gwo_simrank": (ctypes.c_float, [P, P, c_uint32, c_uint32, P]),
            "gwo_convert_text": (c_uint64, [ctypes.c_char_p, c_uint64, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def philox(ctr, key) -> list[int]:
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().gwo_philox4x32_10(_p(c), _p(k), _p(o))
    return [int(x) for x in o]


def continue_threshold(p: float) -> int:
    return lib().gwo_continue_threshold(p)


def prob_to_u32(x: float) -> int:
    """Quadrant threshold on the 32-bit draw scale (as the device generator)."""
    if x <= 0:
        return 0
    v = int(np.floor(x * 4294967296.0 + 0.5))
    return min(v, 0xFFFFFFFF)


def make_params(rule, L, jump_prob=0.15, njump=0, seed=42, max_hops=65535, rng=0) -> Params:
    return Params(rule, L, jump_prob, njump, seed & 0xFFFFFFFFFFFFFFFF, max_hops, rng)


def run_walks(rowptr, colidx, cur, *, rule, L, ids=None, src=None, hop0=None, jump_prob=0.15,
              njump=0, seed=42, max_hops=65535, counts=True, stride=0, closure=False, rng=0):
    """Runs every walk to its end (gw_oracle.h: gwo_run_walks)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    colidx = np.ascontiguousarray(colidx, dtype=np.uint32)
    if len(colidx) == 0:
        colidx = np.zeros(1, dtype=np.uint32)
    nv = len(rowptr) - 1
    cur = np.ascontiguousarray(cur, dtype=np.uint32)
    n = len(cur)
    src = cur.copy() if src is None else np.ascontiguousarray(src, dtype=np.uint32)
    ids = src.copy() if ids is None else np.ascontiguousarray(ids, dtype=np.uint32)
    hop0 = np.zeros(n, np.uint32) if hop0 is None else np.ascontiguousarray(
        np.broadcast_to(hop0, (n,)), dtype=np.uint32)
    prm = make_params(rule, L, jump_prob, njump or nv, seed, max_hops, rng)
    out = {}
    c = np.zeros(nv, np.uint32) if counts else None
    paths = np.full(n * stride, 0xFFFFFFFF, np.uint32) if stride else None
    plen = np.zeros(n, np.uint32)
    clo = np.zeros(1, np.uint64) if closure else None
    fcur = np.zeros(n, np.uint32)
    fhop = np.zeros(n, np.uint32)
    st = lib().gwo_run_walks(_p(rowptr), _p(colidx), nv, _p(cur), _p(ids), _p(src), _p(hop0), n,
                             ctypes.byref(prm), _p(c), _p(paths), stride, _p(plen), _p(clo), _p(fcur),
                             _p(fhop))
    out["status"] = st
    out["counts"] = c
    out["paths"] = paths.reshape(n, stride) if stride else None
    out["plen"] = plen
    out["closure"] = int(clo[0]) if closure else None
    out["final_cur"] = fcur
    out["final_hop"] = fhop
    return out


def compute_blocks(rowptr, blocksize_kb) -> np.ndarray:
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    out = np.zeros(len(rowptr) + 2, np.uint32)
    n = lib().gwo_compute_blocks(_p(rowptr), len(rowptr) - 1, blocksize_kb, _p(out), len(out))
    return out[:n].copy()


def rmat_csr(scale, edge_factor=16, seed=1, a=0.57, b=0.19, c=0.19):
    nv = 1 << scale
    m = edge_factor * nv
    rowptr = np.zeros(nv + 1, np.uint64)
    colidx = np.zeros(max(m, 1), np.uint32)
    kept = lib().gwo_rmat_csr(scale, m, seed, prob_to_u32(a), prob_to_u32(a + b),
                              prob_to_u32(a + b + c), _p(rowptr), _p(colidx))
    return rowptr, colidx[:kept].copy()


def expected_visits(rowptr, colidx, src, rule, L, alpha=0.15) -> np.ndarray:
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    colidx = np.ascontiguousarray(colidx, dtype=np.uint32)
    nv = len(rowptr) - 1
    out = np.zeros(nv, np.float64)
    lib().gwo_expected_visits(_p(rowptr), _p(colidx), nv, src, rule, L, alpha, _p(out))
    return out


def convert_text(text: bytes):
    """(rowptr u64[nv+1], colidx u32[ne]) as convert_to_csr builds them;
    raises ValueError naming the first line the reference rejects."""
    nv, ne = ctypes.c_uint32(), ctypes.c_uint64()
    bad = lib().gwo_convert_text(text, len(text), None, None, ctypes.byref(nv), ctypes.byref(ne))
    if bad:
        raise ValueError(f"line {bad} is not '<from> <to>' (or exceeds 1023 bytes)")
    rowptr = np.zeros(nv.value + 1, np.uint64)
    colidx = np.zeros(max(ne.value, 1), np.uint32)
    lib().gwo_convert_text(text, len(text), _p(rowptr), _p(colidx), None, None)
    return rowptr, colidx[: ne.value]


def simrank(paths_a, paths_b, R, L):
    """(the app's float estimate, per-level first-meeting pair counts)."""
    a = np.ascontiguousarray(paths_a, dtype=np.uint32).reshape(-1)
    b = np.ascontiguousarray(paths_b, dtype=np.uint32).reshape(-1)
    assert a.size == R * L and b.size == R * L
    meet = np.zeros(L, np.uint64)
    est = lib().gwo_simrank(_p(a), _p(b), R, L, _p(meet))
    return float(est), meet


def _chooser_coin(seed: int, superstep: int) -> float:
    """31-bit draw of Philox(seed, (superstep, "CHOS")) as the float quotient."""
    w = philox([superstep & 0xFFFFFFFF, superstep >> 32, 0x43484F53, 0],
               [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF])[0] >> 1
    return float(np.float32(np.float32(w) / np.float32(2147483647)))


def block_engine(rowptr, colidx, blocks, cur, *, rule, L, ids=None, src=None, hop0=None,
                 jump_prob=0.15, njump=0, seed=42, prob=0.2, max_hops=65535, max_supersteps=0, rng=0):
    """The reference's block loop (graphwalker.hpp:272-311) over stable pools.

    Pools hold walks in arrival order: the walks of a superstep are appended
    to their destination pools in the order of the executed pool.  The block
    choice follows chooseBlock (walk.hpp:245-252) with the coin drawn from
    Philox(seed, superstep).  Returns counts, superstep count and the pools
    (cur, id, src, hop per block) left when the loop stopped.
    """
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    colidx = np.ascontiguousarray(colidx if len(colidx) else np.zeros(1, np.uint32), dtype=np.uint32)
    blocks = np.ascontiguousarray(blocks, dtype=np.uint32)
    nv = len(rowptr) - 1
    nb = len(blocks) - 1
    cur = np.asarray(cur, np.uint32)
    n = len(cur)
    src = cur.copy() if src is None else np.asarray(src, np.uint32)
    ids = src.copy() if ids is None else np.asarray(ids, np.uint32)
    hop0 = np.zeros(n, np.uint32) if hop0 is None else np.broadcast_to(np.asarray(hop0, np.uint32), (n,)).copy()
    blk = np.searchsorted(blocks[1:], cur, side="right")
    pools = []
    for b in range(nb):
        m = blk == b
        pools.append([cur[m].copy(), ids[m].copy(), src[m].copy(), hop0[m].copy()])
    minstep = [min(int(p[3].min()), 0xFFFF) if len(p[0]) else 0xFFFF for p in pools]
    prm = make_params(rule, L, jump_prob, njump or nv, seed, max_hops, rng)
    counts = np.zeros(nv, np.uint32)
    status = 0
    superstep = 0
    walksum = n
    while walksum > 0 and (max_supersteps == 0 or superstep < max_supersteps):
        walknum = [len(p[0]) for p in pools]
        if _chooser_coin(seed, superstep) < np.float32(prob):
            mins, minp = 0xFFFF, 0
            for q in range(nb):
                if mins > minstep[q]:
                    mins, minp = minstep[q], q
            b = minp if walknum[minp] > 0 else int(np.argmax(walknum) if max(walknum) > 0 else 0)
        else:
            b = int(np.argmax(walknum)) if max(walknum) > 0 else 0
        c, i, s, h = (np.ascontiguousarray(x) for x in pools[b])
        m = len(c)
        dest = np.zeros(m, np.uint32)
        status |= lib().gwo_block_step(_p(rowptr), _p(colidx), nv, _p(blocks), nb, b, _p(c), _p(i), _p(s),
                                       _p(h), m, ctypes.byref(prm), _p(counts), _p(dest))
        pools[b] = [np.zeros(0, np.uint32) for _ in range(4)]
        minstep[b] = 0xFFFF
        forwarded = 0
        for d in np.unique(dest):
            if d == 0xFFFFFFFF:
                continue
            sel = dest == d
            pools[d] = [np.concatenate([pools[d][k], arr[sel]]) for k, arr in enumerate((c, i, s, h))]
            minstep[d] = min(minstep[d], int(h[sel].min()), 0xFFFF)
            forwarded += int(sel.sum())
        walksum = walksum - m + forwarded
        superstep += 1
    return {"counts": counts, "supersteps": superstep, "pools": pools, "status": status}
