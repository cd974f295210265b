#!/usr/bin/env python
"""Walk-steps/s of GraphWalker's raw-random-walk hot path on one or more B200s.

Workload (one "step"): R-MAT scale 24 (16,777,216 vertices, edge factor 16,
a/b/c/d = 0.57/0.19/0.19/0.05, self-loops dropped, duplicates kept, ids
permuted; graph seed 1), CSR split into 32 blocks by the reference's
compute_block rule and fully resident in HBM; one walk per vertex, fixed
length 10, uniform neighbour choice, the reference's 0.15 else-branch with
jump to a uniform vertex (RandomWalkwithJump), Philox stream seed 42, uint32
visit counts per vertex (the rwdomination sink).  A step clears the counts
and runs every walk to its end: exactly 16,777,216 x 10 = 167,772,160 walk
steps.

    python bench.py [--gpus N --steps K --warmup W]            # this engine
    python bench.py --impl reference [--steps K --warmup W]    # the reference's CPU engine

`value` is whole-job walk-steps/s with the walks and counts resident in HBM
(CUDA events on the launching stream, L2 flushed by a 256 MB write between
steps, max over ranks).  `e2e` is the same metric through the C-ABI call a
host program makes (gw_run_pools): 64-bit walk words copied from pinned host
memory and the counts copied back, every step.  Multi-GPU: the graph is
replicated, each rank runs its own full walk set (walk ids offset by rank,
weak scaling) and the visit counts are summed across ranks with one NCCL
all-reduce per step, inside the timed step.

At N = 1 the same line also carries, measured in the same run: `parity` (the
last timed step's counts against the reference engine's own, compiled from
source with rand_r routed to the same Philox stream), and the other
workloads as sub-objects -- `ppr1` (single-source PPR, R-MAT scale 20),
`msppr` (4096 queries at scale 26, batched vs plain, accuracy judged against
the FP64 series) and `serve` (Poisson arrivals at 1k/10k/50k queries/s,
continuous batching vs one query per superstep) and `ooc` (R-MAT scale 27,
edge factor 48, 257 blocks streamed from pinned host memory into 73 % as many
device slots).  --no-extras leaves those out.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "walk-steps/s"
FALLBACK_HBM_GBS = 6650.0
# Algorithmic DRAM bytes of the headline kernel, per graph layout.  A walk of
# L visits makes L - 1 moves (the move after its last visit is never observed):
#   csr:  per move one 32-B sector for the vertex record + one for the column id;
#   erec: per move one 32-B sector (the edge record moved along, or the vertex
#         record of a jump target) + one 32-B sector per walk for its start record.
BYTES_PER_MOVE = {"csr": 64, "erec": 32}
BYTES_PER_WALK = {"csr": 0, "erec": 32}
LAYOUT_MODE = {"auto": 2, "csr": 0, "erec": 1}  # EDGE_RECORDS_AUTO / _OFF / _ON


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--L", type=int, default=10)
    ap.add_argument("--nblocks", type=int, default=32)
    ap.add_argument("--graph-seed", type=int, default=1)
    ap.add_argument("--walk-seed", type=int, default=42)
    ap.add_argument("--aggregate", type=int, default=0, help="warp-aggregated counter atomics")
    ap.add_argument("--layout", choices=["auto", "csr", "erec"], default="auto",
                    help="graph layout of resident walks: edge records when they fit (auto), plain CSR, edge records")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-probe", action="store_true", help="skip the random-gather roof probe")
    ap.add_argument("--no-extras", action="store_true",
                    help="rawwalk at N=1: skip the single-source PPR, msppr and serving sub-objects")
    ap.add_argument("--cpu-sample-sec", type=float, default=15.0)
    ap.add_argument("--workload", choices=["rawwalk", "msppr", "serve", "ppr1", "ooc", "convert", "simrank",
                                           "gather", "walkonly"],
                    default="rawwalk",
                    help="rawwalk: the headline raw-random-walk step; msppr: batched vs plain multi-source PPR; "
                         "serve: Poisson-arrival PPR serving, continuous batching vs one query per launch; "
                         "gather: the random 32-B sector probe alone (small profiler captures); "
                         "walkonly: --steps resident walk launches at full occupancy, no autotuner, no extras "
                         "(small profiler captures)")
    ap.add_argument("--probe-mb", type=int, default=2048, help="gather: buffer size")
    ap.add_argument("--probe-loads", type=int, default=1 << 26, help="gather: loads per launch")
    ap.add_argument("--probe-host", action="store_true",
                    help="gather: the buffer in pinned host memory, read by the kernel over the host link")
    ap.add_argument("--sink", choices=["count", "none"], default="count",
                    help="walkonly: count visits per vertex (the headline's sink) or record nothing")
    ap.add_argument("--pool-budget-mb", type=int, default=0,
                    help="ooc: also run the streamed block loop with its walk pools held to this many MB of device "
                         "memory (gw_set_pool_budget), the rest spilled to host memory")
    ap.add_argument("--mapped-walks", default="auto",
                    help="ooc: gw_set_mapped_block_walks of the default streamed run ('auto' or a number)")
    ap.add_argument("--rng", choices=["philox", "native"], default="philox", help="walkonly: random stream")
    ap.add_argument("--hints", type=int, default=-1,
                    help="walkonly: explicit GW_HINT_* bits for the walk kernel (-1: the engine default)")
    ap.add_argument("--rates", default="1000,5000,10000,20000,50000", help="serve: arrival rates (queries/s)")
    ap.add_argument("--serve-sec", type=float, default=2.0, help="serve: seconds of arrivals per rate")
    ap.add_argument("--nmblocks", type=int, default=0,
                    help="ooc: device block slots (0: 73%% of the blocks, the share a 206 GB scale-30 graph keeps "
                         "resident on a 180 GB B200)")
    ap.add_argument("--queries", type=int, default=4096)
    ap.add_argument("--convert-sample-mb", type=int, default=512, help="convert: text prefix the reference parses")
    ap.add_argument("--topk", type=int, default=100)
    return ap.parse_args()


def blocksize_kb_for(scale: int, ef: int, nblocks: int) -> int:
    return math.ceil(ef * (1 << scale) * 4 / nblocks / 1024)


def workload_config(args, nblocks_actual=None) -> dict:
    return {"workload": f"raw random walks, R-MAT scale {args.scale} ef {args.edge_factor}, one walk per vertex, "
                        f"L={args.L}, jump rule, uint32 visit counts (rwdomination)",
            "graph": f"rmat(scale={args.scale}, ef={args.edge_factor}, a=0.57, b=0.19, c=0.19, seed={args.graph_seed})",
            "nvertices": 1 << args.scale, "walks_per_gpu": 1 << args.scale, "L": args.L,
            "nblocks": nblocks_actual if nblocks_actual is not None else args.nblocks,
            "blocksize_kb": blocksize_kb_for(args.scale, args.edge_factor, args.nblocks),
            "l2": "flushed between steps (256 MB write)",
            "parallelism": f"replicated graph, walks sharded, dp{args.gpus}"}


# Each arm names its random stream at the top level of its line, beside an
# identical `config`: the engine draws from Philox keyed on (seed, walk id,
# hop); the reference arm runs the reference unmodified, with glibc rand_r.
RNG_OURS = "philox4x32-10 keyed (seed {seed}, walk id, hop): the deterministic mode, bit-exact to the shimmed reference"
RNG_REFERENCE = ("glibc rand_r (native), seeded per block visit with walkid + dstId + hop + time(NULL) "
                 "(randomwalkwithjump.hpp:37), as the reference runs")


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str | None):
        self.proc = None
        self.path = None
        self.device_id = device_id

    def __enter__(self):
        try:
            self.path = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
            if self.device_id:
                cmd.insert(1, f"--id={self.device_id}")
            self.proc = subprocess.Popen(cmd, stdout=self.path, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict | None:
        if not self.proc or not self.path:
            return None
        rows = []
        for line in Path(self.path.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), float(parts[2]), parts[3:]))
            except ValueError:
                continue
        os.unlink(self.path.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[3][1:]) if v.lower().startswith("active")})
        loaded = [r for r in rows if r[2] > 250.0] or rows
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons}


def device_uuid(dev: int) -> str | None:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else f"GPU-{u}"
    except Exception:
        return None


def measured_peaks() -> tuple[float, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(layout: str) -> float | None:
    """DRAM bytes per walk launch from the committed ncu summary, if any."""
    return profile_field(layout, "dram_bytes_per_launch")


def profile_field(layout: str, key: str) -> float | None:
    f = ROOT / "profiles" / ("walk_resident_rmat24.json" if layout == "csr" else "walk_resident_erec_rmat24.json")
    if f.exists():
        try:
            return float(json.loads(f.read_text())[key])
        except Exception:
            return None
    return None


# --------------------------------------------------------------------------- reference arm
def write_reference_graph(tmp: Path, args, rowptr, colidx) -> tuple[str, int, int]:
    from graphwalker_b200 import formats
    base = str(tmp / f"rmat{args.scale}")
    kb = blocksize_kb_for(args.scale, args.edge_factor, args.nblocks)
    blocks = formats.write_graph(base, rowptr, colidx, kb)
    (tmp / "conf").mkdir(exist_ok=True)
    (tmp / "conf" / "graphwalker.cnf").write_text("# GraphWalker configuration (empty)\n")
    return base, kb, len(blocks) - 1


def write_reference_graph_c(tmp: Path, args) -> tuple[str, int]:
    """The benchmark graph for the reference arm, generated and written in the
    reference's on-disk layout by the C generator (oracle/_build/gw_oracle_rmat,
    the same seeded R-MAT stream the device generator reproduces bit for bit).
    It runs as its own process, so the arm loads no library of this repository;
    the reference computes the block range itself on its first run."""
    exe = ROOT / "oracle" / "_build" / "gw_oracle_rmat"
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing (built by `make -C oracle`)")
    base = str(tmp / f"rmat{args.scale}")
    subprocess.run([str(exe), str(args.scale), str(args.edge_factor), str(args.graph_seed), "0.57", "0.19", "0.19",
                    base], check=True, capture_output=True, timeout=1800)
    (tmp / "conf").mkdir(exist_ok=True)
    (tmp / "conf" / "graphwalker.cnf").write_text("# GraphWalker configuration (empty)\n")
    return base, blocksize_kb_for(args.scale, args.edge_factor, args.nblocks)


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_ref_bench(base, kb, nv, L, stride, warmup, steps, threads, cwd) -> list[tuple[int, float, int]]:
    """(visits, seconds, OpenMP threads left at the end) per timed run."""
    exe = ROOT / "oracle" / "_ref" / "gw_ref_bench"
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing (built by `make -C oracle ref` where the reference tree exists)")
    out = subprocess.run([str(exe), base, str(kb), str(nv), str(L), str(stride), str(warmup), str(steps),
                          "execthreads", str(threads)], cwd=cwd, capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(f"gw_ref_bench failed ({out.returncode}): {out.stderr[-500:]}")
    res = []
    for line in out.stdout.splitlines():
        f = line.split()
        if len(f) >= 10 and f[0] == "step":
            res.append((int(f[3]) * L, float(f[7]), int(f[9])))  # jump-rule walks make exactly L visits
    return res


def fallback_report(res, threads: int) -> dict:
    """Whether the reference's sticky single-thread fallback fired: exec_updates
    sets one OpenMP thread for a block with fewer than 100 walks and never
    restores it (graphwalker.hpp:260)."""
    fired = [i for i, r in enumerate(res) if threads > 1 and r[2] == 1]
    return {"fired": bool(fired), "runs_fired": len(fired), "runs": len(res), "execthreads": threads,
            "rule": "graphwalker.hpp:260 if(nwalks < 100) omp_set_num_threads(1), never undone within a run"}


def cpu_reference(args, base: str, kb: int, nv: int, tmp: Path, warmup: int, steps: int, budget_s: float) -> dict:
    """Times the reference engine on the host cores, on the graph files at
    `base`; the per-run sample (one walk on every `stride`-th vertex) is sized
    so that warmup + steps runs fit budget_s."""
    threads = host_cores()
    probe_stride = 64
    cal = run_ref_bench(base, kb, nv, args.L, probe_stride, 1, 1, threads, tmp)
    rate = cal[0][0] / max(cal[0][1], 1e-9)
    per_step = budget_s / max(1, warmup + steps)
    want_walks = max(1024, min(nv, int(rate * per_step / args.L)))
    stride = max(1, nv // want_walks)
    res = run_ref_bench(base, kb, nv, args.L, stride, warmup, steps, threads, tmp)
    nb = len(Path(base + "_GraphWalker", f"blocksize_{kb}KB.blockrange").read_text().split()) - 1
    tot_steps = sum(r[0] for r in res)
    tot_t = sum(r[1] for r in res)
    return {"value": tot_steps / tot_t, "unit": METRIC, "cores": threads, "kind": "reference",
            "sec_per_step": tot_t / len(res), "steps": len(res), "nblocks": nb,
            "single_thread_fallback": fallback_report(res, threads),
            "sample": f"the reference engine (graphwalker.hpp) + RandomWalkwithJump compiled -O3 from source, "
                      f"native rand_r, {threads} OpenMP threads, one walk on every {stride}-th vertex "
                      f"({nv // stride} walks x {args.L} hops per run) of the same scale-{args.scale} graph, "
                      f"blocks cached in RAM after the first run"}


def reference_parity(args, base: str, kb: int, blocks, nv: int, tmp: Path, gpu_counts) -> dict:
    """The timed step's visit counts against the reference engine itself.

    Runs GraphWalker's engine and RandomWalkwithJump, compiled from the
    reference's sources with its rand_r calls routed to the same Philox stream
    (oracle/_ref/gw_ref_shim_0), on the same graph files with the same walks:
    one per vertex, source field = start vertex (its Philox key).  Outside the
    timed region; `identical_counts` is the bit-for-bit comparison of all
    per-vertex counts."""
    import struct

    import numpy as np
    exe = ROOT / "oracle" / "_ref" / "gw_ref_shim_0"
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing (built by `make -C oracle ref` where the reference tree exists)")
    if nv > (1 << 24):
        raise ValueError("the walk word's 24-bit source field keys at most 2^24 walks")
    threads = host_cores()
    v = np.arange(nv, dtype=np.uint64)
    b64 = np.asarray(blocks, dtype=np.int64)
    blk = np.searchsorted(b64[1:], np.arange(nv, dtype=np.int64), side="right")
    rec = np.zeros(nv, dtype=[("b", "<u4"), ("pad", "<u4"), ("w", "<u8")])
    rec["b"] = blk
    rec["w"] = (v << np.uint64(40)) | ((v - b64[blk].astype(np.uint64)) << np.uint64(14))  # walk.hpp:69-73, hop 0
    wf, of = tmp / "parity_walks.bin", tmp / "parity_out.bin"
    with open(wf, "wb") as f:
        f.write(struct.pack("<Q", nv))
        f.write(rec.tobytes())
    del rec, v, blk
    t0 = time.perf_counter()
    subprocess.run([str(exe), base, str(kb), str(wf), str(of), str(args.L), f"{args.walk_seed:x}", str(nv), "0",
                    "0.2", "0", "0", "execthreads", str(threads)], cwd=tmp, check=True, capture_output=True,
                   timeout=1800)
    sec = time.perf_counter() - t0
    raw = of.read_bytes()
    status, nv_ref = struct.unpack_from("<II", raw, 0)
    ref = np.frombuffer(raw, np.uint32, nv_ref, 8)
    gpu = np.asarray(gpu_counts, dtype=np.uint32)
    diff = int(np.count_nonzero(ref != gpu)) if nv_ref == nv else nv
    return {"identical_counts": bool(diff == 0 and status == 0), "vertices_differing": diff, "walks": nv,
            "visits": int(ref.astype(np.int64).sum()), "reference_status": int(status), "sec": sec,
            "against": "the reference engine + RandomWalkwithJump compiled from source, rand_r routed to the same "
                       "Philox stream (gw_ref_shim_0), all walks of the timed step, counts of its last step"}


def cpu_reference_msppr(args, base: str, kb: int, nv: int, tmp: Path, walkspersource: int, budget_s: float) -> dict:
    """The reference engine with RandomWalkwithStop on msppr's placement
    (contiguous sources, a fixed number of walks each), sized to budget_s."""
    threads = host_cores()
    exe = ROOT / "oracle" / "_ref" / "gw_ref_bench"
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing (built by `make -C oracle ref` where the reference tree exists)")

    def run(numsources: int, warm: int):
        out = subprocess.run([str(exe), base, str(kb), str(nv), "20", "1", str(warm), "1", "execthreads",
                              str(threads), "msppr", "0", str(numsources), str(walkspersource)],
                             cwd=tmp, capture_output=True, text=True, timeout=1800)
        if out.returncode != 0:
            raise RuntimeError(out.stderr[-400:])
        f = [l.split() for l in out.stdout.splitlines() if l.startswith("step")][-1]
        return float(f[7]), int(f[5]), int(f[9])

    t_cal, _, _ = run(8, 1)
    numsources = max(8, min(4096, int(8 * budget_s / max(t_cal, 1e-6))))
    t, visits, thr_after = run(numsources, 1)
    return {"value": numsources / t, "unit": "queries/s", "cores": threads, "kind": "reference",
            "single_thread_fallback": fallback_report([(visits, t, thr_after)], threads),
            "sample": f"the reference engine + RandomWalkwithStop compiled -O3 from source, native rand_r, "
                      f"{threads} OpenMP threads, msppr placement: sources 0..{numsources - 1} x {walkspersource} "
                      f"walks (the mean budget), L<=20, a per-thread visit counter as sink ({visits} visits)"}


def reference_arm(args) -> None:
    """The reference's CPU engine on this box's host cores, on the headline
    workload.  Nothing of this repository's engine is loaded: the graph comes
    from the C generator (its own process) and the timed binary is the
    reference compiled from its sources."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    warm = max(1, args.warmup)
    with tempfile.TemporaryDirectory(prefix="gw_ref_") as td:
        tmp = Path(td)
        base, kb = write_reference_graph_c(tmp, args)
        r = cpu_reference(args, base, kb, 1 << args.scale, tmp, warm, args.steps, budget_s=150.0)
    line = {"metric": METRIC, "value": r["value"], "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": warm, "ms_per_step": r["sec_per_step"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(args, r["nblocks"]), "rng": RNG_REFERENCE,
            "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": r["cores"], "kind": "reference",
                             "sample": r["sample"]},
            "single_thread_fallback": r["single_thread_fallback"],
            "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- this engine
def our_arm(args) -> None:
    import numpy as np
    import torch
    import torch.distributed as dist

    import graphwalker_b200 as gw

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    kb = blocksize_kb_for(args.scale, args.edge_factor, args.nblocks)
    G = gw.Graph.rmat(args.scale, args.edge_factor, seed=args.graph_seed, blocksize_kb=kb, device=local)
    layout = "erec" if G.set_edge_records(LAYOUT_MODE[args.layout]) else "csr"
    nv, L = G.nv, args.L
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    # walk records resident in HBM: one walk per vertex, ids offset by rank
    v = torch.arange(nv, dtype=torch.int64, device="cuda")
    walks = torch.stack([v, v + rank * nv, v, torch.zeros_like(v)], dim=1).to(torch.int32).contiguous()
    del v
    counts = torch.zeros(nv, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    p = gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, L, seed=args.walk_seed, aggregate=bool(args.aggregate))

    # launch shape (CTAs per SM) timed on these walks before the warm-up
    tuned_ctas = G.walk_autotune(p, walks, nv)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    # A step = clear the counts, walk every walk to its end, and (N > 1) sum
    # the counts over the ranks: the path's one exchange is inside the step.
    for _ in range(max(3, args.warmup)):
        counts.zero_()
        G.walk_device(p, walks, nv, counts=counts, stream=sh)
        if world > 1:
            dist.all_reduce(counts)
    G.sync(sh)
    total_visits = int(counts.to(torch.int64).sum().item())
    expect = nv * L * world
    if total_visits != expect:
        raise RuntimeError(f"visit count {total_visits} != {expect}")

    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    with ClockSampler(device_uuid(local)) as clk:
        barrier()
        torch.cuda.synchronize()
        for k in range(K):
            flush.fill_(k & 0xFF)
            ev[k][0].record(stream)
            counts.zero_()
            ev[k][1].record(stream)
            G.walk_device(p, walks, nv, counts=counts, stream=sh)
            ev[k][2].record(stream)
            if world > 1:
                dist.all_reduce(counts)  # blocking form: the current stream waits for the reduction
            ev[k][3].record(stream)
        torch.cuda.synchronize()
        barrier()
    G.sync(sh)
    step_ms = sum(e[0].elapsed_time(e[3]) for e in ev) / K
    kern_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / K
    xchg_ms = sum(e[2].elapsed_time(e[3]) for e in ev) / K
    if world > 1:
        t = torch.tensor([step_ms, kern_ms, xchg_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms, kern_ms, xchg_ms = t.tolist()
    steps_per_launch = nv * L
    value = steps_per_launch * world / (step_ms * 1e-3)
    last_counts = counts.cpu().numpy().view(np.uint32).copy() if world == 1 else None

    # random-sector gather roof: an 8 GB buffer, far larger than L2
    gather_bps = red_ops_s = None
    if rank == 0 and not args.no_probe:
        buf = torch.empty(1 << 31, dtype=torch.int32, device="cuda")
        gather_bps = G.probe_gather(buf, buf.numel(), 1 << 28, iters=5)
        del buf
        # and the visit-counter roof: one red.add per visit into nv counters
        red_ops_s = G.probe_red(counts, nv, steps_per_launch, iters=5)
        torch.cuda.empty_cache()

    # e2e through the C-ABI host call (pinned words in, counts out)
    e2e = None
    if not args.no_e2e:
        e2e = e2e_run_pools(args, G, p, rank, world, K, barrier, last_counts)

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rowptr, colidx = G.export_csr()
            with tempfile.TemporaryDirectory(prefix="gw_ref_") as td:
                tmp = Path(td)
                base, kbw, _ = write_reference_graph(tmp, args, rowptr, colidx)
                del rowptr, colidx
                r = cpu_reference(args, base, kbw, nv, tmp, 1, 1, budget_s=args.cpu_sample_sec)
                cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample", "single_thread_fallback")}
                try:
                    parity = reference_parity(args, base, kbw, G.blocks, nv, tmp, last_counts)
                except Exception as exc:  # reported, never required
                    parity = {"identical_counts": None, "error": str(exc)[-300:]}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": host_cores(), "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if world > 1:
        dist.barrier(device_ids=[local])
        dist.destroy_process_group()
    G.close()
    del walks, counts, flush
    torch.cuda.empty_cache()
    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    moves = steps_per_launch - nv
    algo_bytes = BYTES_PER_MOVE[layout] * moves + BYTES_PER_WALK[layout] * nv
    achieved = algo_bytes / (kern_ms * 1e-3) / 1e9
    traffic = profile_traffic(layout)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": f"{peak_kind} HBM copy bandwidth",
            "bytes_per_move": BYTES_PER_MOVE[layout], "bytes_per_walk": BYTES_PER_WALK[layout],
            "moves_per_launch": moves,
            "algorithmic_bytes_per_launch": algo_bytes, "graph_layout": layout,
            "kernel": f"walk_resident_kernel<JUMP, VERTEX_COUNT, ER={'true' if layout == 'erec' else 'false'}>",
            "kernel_ms": kern_ms}
    if gather_bps:
        roof["gather_peak_gbs"] = gather_bps / 1e9
        roof["gather_frac"] = achieved / (gather_bps / 1e9)
        # the line-fill view: a random miss fills a 128-B line, so compare the
        # kernel's DRAM read rate with the probe's (its useful rate times the
        # DRAM sectors it reads per 32-B load, from the committed ncu summary)
        amp = profile_field(layout, "gather_probe_dram_sectors_per_load")
        if traffic and amp:
            roof["dram_gbs"] = traffic / (kern_ms * 1e-3) / 1e9
            roof["probe_dram_gbs"] = gather_bps / 1e9 * amp
            roof["line_fill_frac"] = roof["dram_gbs"] / roof["probe_dram_gbs"]
            roof["dram_bytes_per_step"] = traffic / steps_per_launch
            if red_ops_s:
                # the two resources a launch uses, each at its own probe's rate:
                # its line fills (DRAM) and its visit-counter updates (L2 atomics)
                fills_ms = traffic / (roof["probe_dram_gbs"] * 1e9) * 1e3
                reds_ms = steps_per_launch / red_ops_s * 1e3
                roof["counter_updates_per_s_probe"] = red_ops_s
                roof["fills_alone_ms"] = fills_ms
                roof["counter_updates_alone_ms"] = reds_ms
                roof["fills_plus_updates_frac"] = (fills_ms + reds_ms) / kern_ms
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
            "warmup": max(3, args.warmup), "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(args, G.nblocks), "rng": RNG_OURS.format(seed=args.walk_seed),
            "engine": {"graph_layout": layout, "autotuned_ctas_per_sm": tuned_ctas},
            "step_breakdown_ms": {"walk_kernel": kern_ms, "count_exchange": xchg_ms,
                                  "exchange": "NCCL all_reduce of the u32 counts" if world > 1 else "none (N=1)"},
            "roofline": roof, "cpu_baseline": cpu, "parity": parity, "e2e": e2e, "gpu_launches": K,
            "clocks": clk.summary(), "walk_steps_per_step": steps_per_launch * world}
    if world == 1 and not args.no_extras:
        # the other configs' workloads, each measured in this same run
        for key, fn in (("ppr1", ppr1_measure), ("msppr", msppr_measure),
                        ("serve", lambda a: serve_measure(a, rates="1000,10000,50000")), ("ooc", ooc_measure)):
            t0 = time.perf_counter()
            try:
                line[key] = fn(args)
            except Exception as exc:  # reported, never required
                line[key] = {"error": f"{type(exc).__name__}: {str(exc)[-300:]}"}
            line[key]["wall_s"] = time.perf_counter() - t0
            torch.cuda.empty_cache()
    print(json.dumps(line), flush=True)


def e2e_run_pools(args, G, p, rank: int, world: int, K: int, barrier, device_counts) -> dict:
    """The headline metric through the C-ABI host call a program makes
    (gw_run_pools): 64-bit walk words copied in from pinned host memory and the
    u32 counts copied back, every step."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    nv, L = G.nv, args.L
    vv = np.arange(nv, dtype=np.uint64)
    blocks = G.blocks.astype(np.int64)
    blk = np.searchsorted(blocks[1:], np.arange(nv), side="right")
    words_np = gw.encode(vv, vv - blocks[blk].astype(np.uint64), 0)
    offs_np = np.r_[0, np.cumsum(np.bincount(blk, minlength=G.nblocks))].astype(np.uint64)
    words = torch.from_numpy(words_np.view(np.int64)).pin_memory()
    offs = torch.from_numpy(offs_np.view(np.int64)).pin_memory()
    del vv, blk, words_np
    ids = None
    if rank:
        ids = torch.from_numpy((np.arange(nv, dtype=np.uint64) + rank * nv).astype(np.uint32).view(np.int32)).pin_memory()
    hcounts = [torch.zeros(nv, dtype=torch.int32).pin_memory() for _ in range(2)]
    idp = None if ids is None else ids.data_ptr()
    n_e2e = min(K, 50)

    def max_over_ranks(x):
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([x], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            x = t.item()
        return x

    # one call at a time: each returns with its counts on the host
    for _ in range(3):
        G.run_pools(p, words.data_ptr(), offs.data_ptr(), hcounts[0].data_ptr(), ids=idp)
    barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        G.run_pools(p, words.data_ptr(), offs.data_ptr(), hcounts[0].data_ptr(), ids=idp)
    sync_s = max_over_ranks((time.perf_counter() - t0) / n_e2e)

    # back-to-back steps, two in flight (gw_run_pools_submit / wait): step
    # k's count read-back overlaps step k + 1's copies in and walks; every
    # step still copies its words in and its counts out
    def pipelined(n):
        prev = None
        for k in range(n):
            t = G.run_pools_submit(p, words.data_ptr(), offs.data_ptr(), hcounts[k % 2].data_ptr(), ids=idp)
            if prev is not None:
                G.run_pools_wait(prev)
            prev = t
        G.run_pools_wait(prev)

    pipelined(3)
    barrier()
    t0 = time.perf_counter()
    pipelined(n_e2e)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / n_e2e)
    got = [h.numpy().view(np.uint32) for h in hcounts]
    for g in got:
        if int(g.astype(np.int64).sum()) != nv * L:
            raise RuntimeError("e2e visit count mismatch")
    out = {"value": nv * L * world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int(words.numel() * 8 + offs.numel() * 8 + (ids.numel() * 4 if ids is not None else 0)),
           "d2h_bytes_per_step": int(nv * 4), "ms_per_step": e2e_s * 1e3,
           "api": "gw_run_pools_submit / gw_run_pools_wait (C ABI, pinned host buffers), two steps in flight",
           "one_call_at_a_time": {"api": "gw_run_pools", "value": nv * L * world / sync_s, "ms_per_step": sync_s * 1e3}}
    if device_counts is not None:
        out["identical_to_device_step"] = bool(all(np.array_equal(g, device_counts) for g in got))
    # Within one call the count read-back cannot overlap the walks: any walk
    # may visit any vertex up to its last hop, so no count is final before
    # the last walk ends.  Its cost alone: the same 64 MB device-to-pinned-host
    # copy (hidden behind the next step when two steps are in flight).
    dcounts = torch.zeros(nv, dtype=torch.int32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d2h = []
    for _ in range(5):
        e0.record()
        hcounts[0].copy_(dcounts, non_blocking=True)
        e1.record()
        e1.synchronize()
        d2h.append(e0.elapsed_time(e1))
    out["count_readback_ms"] = statistics.median(d2h)
    return out


def msppr_queries(rp, nq: int, seed: int = 7):
    """Sources uniform over vertices with out-degree >= 1; budgets round(10^U(2,5))."""
    import numpy as np
    rng = np.random.default_rng(seed)
    deg = np.diff(rp.astype(np.int64))
    candidates = np.nonzero(deg > 0)[0]
    sources = rng.choice(candidates, nq).astype(np.uint32)
    budgets = np.round(10 ** rng.uniform(2, 5, nq)).astype(np.uint32)
    return sources, budgets


def extra_scale(args, default: int) -> int:
    """The graph scale of a non-headline workload: its config's own, unless
    --scale names another than the headline's 24."""
    return args.scale if args.scale != 24 else default


def msppr_measure(args) -> dict:
    """Batched multi-source PPR (one persistent launch for all queries) vs the
    plain per-query path, on one GPU: queries/s, same results, and the top-100
    accuracy of the largest queries judged against the FP64 power series."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    torch.cuda.set_device(0)
    scale = extra_scale(args, 26)
    kb = blocksize_kb_for(scale, args.edge_factor, args.nblocks)
    G = gw.Graph.rmat(scale, args.edge_factor, seed=args.graph_seed, blocksize_kb=kb)
    try:
        layout = "erec" if G.set_edge_records(LAYOUT_MODE[args.layout]) else "csr"
        rp, _ = G.export_csr()
        sources, budgets = msppr_queries(rp, args.queries)
        del rp
        L = 20
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, L, seed=args.walk_seed)
        tuned, tuned_chunk = G.ppr_autotune(p, sources[:256], budgets[:256])
        for _ in range(max(1, args.warmup)):
            G.ppr(p, sources, budgets, k=args.topk, batched=True)
        runs = []
        steps = max(1, args.steps)
        with ClockSampler(device_uuid(0)) as clk:
            for _ in range(steps):
                ids_b, cnt_b, st = G.ppr(p, sources, budgets, k=args.topk, batched=True)
                runs.append((st.ms_total, st.ms_clear, st.ms_walk, st.ms_topk))
        ms_med = statistics.median(r[0] for r in runs)
        G.ppr(p, sources, budgets, k=args.topk, batched=False)  # warm-up of the plain path
        ids_p, cnt_p, stp = G.ppr(p, sources, budgets, k=args.topk, batched=False)
        same = bool(np.array_equal(ids_b, ids_p) and np.array_equal(cnt_b, cnt_p))
        e2e = []
        for _ in range(3):
            t0 = time.perf_counter()
            G.ppr(p, sources, budgets, k=args.topk, batched=True)
            e2e.append(time.perf_counter() - t0)
        e2e_s = statistics.median(e2e)
        # top-100 accuracy of the largest-budget queries against the FP64 power
        # series, judged against the Monte Carlo noise of their budgets.  The
        # full per-vertex counts come from the same walks (walk j of the batch
        # has Philox id j) run through the resident kernel.
        prefix = np.r_[0, np.cumsum(budgets.astype(np.int64))]
        acc, mus = [], {}
        for q in np.argsort(-budgets.astype(np.int64), kind="stable")[:4]:
            src, B = int(sources[q]), int(budgets[q])
            mu = mus[int(q)] = G.expected_visits(p, src)
            j = torch.arange(prefix[q], prefix[q + 1], dtype=torch.int64, device="cuda")
            w = torch.stack([torch.full_like(j, src), j, torch.full_like(j, src), torch.zeros_like(j)], 1)
            w = w.to(torch.int32).contiguous()
            cnt = torch.zeros(G.nv, dtype=torch.int32, device="cuda")
            G.walk_device(gw.params(gw.RULE_STOP, gw.SINK_VERTEX_COUNT, L, seed=args.walk_seed), w, B, counts=cnt)
            G.sync()
            c = cnt.cpu().numpy().view(np.uint32)
            del w, cnt, j
            nz = np.flatnonzero(c)
            from_counts = accuracy.count_topk(nz, c[nz], args.topk)
            listed = ids_b[q][ids_b[q] != 0xFFFFFFFF]
            m = accuracy.measured_accuracy(mu, B, L, ids_b[q], counts=c, k=args.topk)
            m["query"] = int(q)
            m["batched_list_equals_counts_topk"] = bool(np.array_equal(listed, from_counts))
            acc.append(m)
        # native-RNG mode: the same batch, judged against the same FP64 series
        pn = gw.params(gw.RULE_STOP, gw.SINK_NONE, L, seed=args.walk_seed, rng=gw.RNG_NATIVE)
        G.ppr(pn, sources, budgets, k=args.topk, batched=True)
        nat_ms = []
        for _ in range(steps):
            ids_n, _, stn = G.ppr(pn, sources, budgets, k=args.topk, batched=True)
            nat_ms.append(stn.ms_total)
        nat_acc = [{"query": m["query"], **accuracy.measured_accuracy(mus[m["query"]], int(budgets[m["query"]]), L,
                                                                      ids_n[m["query"]], k=args.topk)} for m in acc]
        native = {"value": args.queries / (statistics.median(nat_ms) * 1e-3), "unit": "queries/s",
                  "ms_per_step": statistics.median(nat_ms), "accuracy_vs_fp64": nat_acc}
        cpu = None
        if not args.no_cpu_baseline:
            try:
                rp_h, ci_h = G.export_csr()
                with tempfile.TemporaryDirectory(prefix="gw_ref_") as td:
                    tmp = Path(td)
                    base, kbw, _ = write_reference_graph(tmp, argparse.Namespace(**{**vars(args), "scale": scale}),
                                                         rp_h, ci_h)
                    del rp_h, ci_h
                    cpu = cpu_reference_msppr(args, base, kbw, G.nv, tmp, int(round(float(budgets.mean()))),
                                              args.cpu_sample_sec)
            except Exception as exc:  # reported, never required
                cpu = {"value": None, "unit": "queries/s", "cores": host_cores(), "kind": "reference",
                       "sample": f"unavailable: {exc}"}
        return {"metric": "queries/s", "value": args.queries / (ms_med * 1e-3), "unit": "queries/s",
                "workload": "msppr", "n_gpus": 1, "steps": steps, "warmup": max(1, args.warmup),
                "ms_per_step": ms_med, "higher_is_better": True, "dtype": "u32", "data": "synthetic",
                "config": {"workload": f"multi-source PPR, R-MAT scale {scale} ef {args.edge_factor}, "
                                       f"{args.queries} queries, sources uniform over out-degree>=1, budgets "
                                       f"round(10^U(2,5)), stop rule p=0.15, L<=20, top-{args.topk}",
                           "walks_per_step": int(budgets.sum()), "autotuned_threads_per_sm": tuned,
                           "autotuned_walks_per_warp_grab": tuned_chunk, "graph_layout": layout},
                "breakdown_ms": {"clear": statistics.median(r[1] for r in runs),
                                 "walk": statistics.median(r[2] for r in runs),
                                 "topk": statistics.median(r[3] for r in runs)},
                "plain": {"value": args.queries / (stp.ms_total * 1e-3), "unit": "queries/s", "ms": stp.ms_total,
                          "launches": stp.launches},
                "speedup_vs_plain": stp.ms_total / ms_med, "identical_to_plain": same,
                "accuracy_vs_fp64": acc, "native_rng": native, "cpu_baseline": cpu,
                "e2e": {"value": args.queries / e2e_s, "unit": "queries/s", "ms_per_step": e2e_s * 1e3,
                        "api": "gw_ppr_run (host arrays in, top-k lists out)",
                        "h2d_bytes_per_step": int(args.queries * 8),
                        "d2h_bytes_per_step": int(args.queries * args.topk * 8)},
                "gpu_launches": int(st.launches) * steps, "clocks": clk.summary()}
    finally:
        G.close()


def msppr_arm(args) -> None:
    line = msppr_measure(args)
    line["scaling"], line["vs_baseline"] = "weak", None
    print(json.dumps(line), flush=True)


def serve_measure(args, rates: str | None = None) -> dict:
    """PPR serving on one GPU: Poisson arrivals at each rate, budgets
    Pareto(alpha=1.5, x_m=100) clipped to [100, 1e6], top-100 per query;
    continuous batching vs the plain one-query-per-superstep server."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    torch.cuda.set_device(0)
    scale = extra_scale(args, 26)
    G = gw.Graph.rmat(scale, args.edge_factor, seed=args.graph_seed,
                      blocksize_kb=blocksize_kb_for(scale, args.edge_factor, args.nblocks))
    try:
        rp, _ = G.export_csr()
        deg = np.diff(rp.astype(np.int64))
        cand = np.nonzero(deg > 0)[0]
        del rp, deg
        p = gw.params(gw.RULE_STOP, gw.SINK_NONE, 20, seed=args.walk_seed)
        rng = np.random.default_rng(11)
        G.ppr_autotune(p, rng.choice(cand, 64).astype(np.uint32), np.full(64, 2000, np.uint32))
        results = []
        with ClockSampler(device_uuid(0)) as clk:
            for rate in [float(r) for r in (rates or args.rates).split(",")]:
                n = max(200, int(rate * args.serve_sec))
                src = rng.choice(cand, n).astype(np.uint32)
                bud = np.clip(np.round(100.0 / rng.random(n) ** (1 / 1.5)), 100, 1_000_000).astype(np.uint32)
                gaps = rng.exponential(1e9 / rate, n)
                row = {"rate_qps": rate, "queries": n, "mean_budget": float(bud.mean())}
                lists = {}
                for name, mode in (("batched", gw._lib.SERVE_BATCHED), ("plain", gw._lib.SERVE_PLAIN)):
                    with G.serve(p, k=args.topk, mode=mode, table_slots=1 << 30) as S:
                        S.wait(S.submit(int(src[0]), 1000, 0), 60_000)  # warm-up
                        t0 = S.clock_ns() + 5_000_000
                        arrivals = t0 + np.cumsum(gaps).astype(np.int64)
                        tickets = [S.submit(int(s), int(b), i, int(a))
                                   for i, (s, b, a) in enumerate(zip(src, bud, arrivals))]
                        res = [S.wait(t, 600_000) for t in tickets]
                        st = S.stats()
                    tm = [r[2] for r in res]
                    lists[name] = np.stack([r[0] for r in res])
                    lat = np.array([x.done_ns - x.arrival_ns for x in tm], dtype=np.float64) / 1e6
                    span = (max(x.done_ns for x in tm) - int(arrivals[0])) / 1e9
                    row[name] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                                 "throughput_qps": n / span, "supersteps": int(st.supersteps)}
                # a query's draws depend only on (source, budget, stream): same lists either way
                row["identical_lists_batched_vs_plain"] = bool(np.array_equal(lists["batched"], lists["plain"]))
                results.append(row)
        best = max(results, key=lambda r: r["batched"]["throughput_qps"])
        return {"metric": "queries/s", "value": best["batched"]["throughput_qps"], "unit": "queries/s",
                "workload": "serve", "n_gpus": 1, "steps": len(results), "warmup": 1, "higher_is_better": True,
                "dtype": "u32", "data": "synthetic",
                "config": {"workload": f"PPR serving, R-MAT scale {scale}, Poisson arrivals, budgets Pareto(1.5, 100) "
                                       f"clipped to [100, 1e6], stop rule p=0.15, L<=20, top-{args.topk}, "
                                       f"{args.serve_sec} s of arrivals per rate"},
                "rates": results, "clocks": clk.summary()}
    finally:
        G.close()


def serve_arm(args) -> None:
    line = serve_measure(args)
    line["scaling"], line["vs_baseline"] = "weak", None
    print(json.dumps(line), flush=True)


def ppr1_measure(args) -> dict:
    """Single-source PPR (R-MAT scale 20, 16 blocks, 100,000 walks from vertex
    0, stop w.p. 0.15, a dangling vertex sends the walk back to its source,
    at most 20 hops): per-vertex visit counts and the top-100, with the L1
    error and top-100 overlap judged against the FP64 power series."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    from graphwalker_b200 import accuracy
    torch.cuda.set_device(0)
    scale = extra_scale(args, 20)
    B, L = 100_000, 20
    G = gw.Graph.rmat(scale, args.edge_factor, seed=args.graph_seed,
                      blocksize_kb=blocksize_kb_for(scale, args.edge_factor, 16))
    try:
        nv = G.nv
        # "vertex 0" of the R-MAT generator (all-zero quadrant bits: its hub) is
        # the vertex with the largest out-degree once ids are permuted
        rp, _ = G.export_csr()
        src = int(np.argmax(np.diff(rp.astype(np.int64))))
        del rp
        j = torch.arange(B, dtype=torch.int64, device="cuda")
        walks = torch.stack([torch.full_like(j, src), j, torch.full_like(j, src), torch.zeros_like(j)], 1)
        walks = walks.to(torch.int32).contiguous()
        counts = torch.zeros(nv, dtype=torch.int32, device="cuda")
        p = gw.params(gw.RULE_PPR, gw.SINK_VERTEX_COUNT, L, seed=args.walk_seed, aggregate=True)
        sh = torch.cuda.current_stream().cuda_stream
        for _ in range(max(3, args.warmup)):
            counts.zero_()
            G.walk_device(p, walks, B, counts=counts, stream=sh)
        G.sync(sh)
        steps = max(1, args.steps)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in ev:
            counts.zero_()
            a.record()
            G.walk_device(p, walks, B, counts=counts, stream=sh)
            b.record()
        G.sync(sh)
        ms = statistics.median(a.elapsed_time(b) for a, b in ev)
        c = counts.cpu().numpy().view(np.uint32).copy()
        nsteps = int(c.astype(np.int64).sum())
        # the same query through the C ABI (gw_ppr_run, host arrays in and out): warm calls
        api_dev, api_wall = [], []
        for i in range(3 + steps):
            t0 = time.perf_counter()
            ids, cnt, st = G.ppr(p, np.array([src], np.uint32), np.array([B], np.uint32), k=100)
            if i >= 3:
                api_wall.append((time.perf_counter() - t0) * 1e3)
                api_dev.append(st.ms_total)
        mu = G.expected_visits(p, src)
        acc = accuracy.measured_accuracy(mu, B, L, ids[0], counts=c, k=100)
        top_from_counts = accuracy.count_topk(np.arange(nv), c, 100)
        acc["top100_api_equals_counts"] = bool(np.array_equal(ids[0][ids[0] != 0xFFFFFFFF], top_from_counts))
        # native-RNG mode (one Philox block per two hops): timed the same way,
        # judged against the same FP64 series
        pn = gw.params(gw.RULE_PPR, gw.SINK_VERTEX_COUNT, L, seed=args.walk_seed, aggregate=True, rng=gw.RNG_NATIVE)
        for a_, b_ in ev:
            counts.zero_()
            a_.record()
            G.walk_device(pn, walks, B, counts=counts, stream=sh)
            b_.record()
        G.sync(sh)
        ms_native = statistics.median(a_.elapsed_time(b_) for a_, b_ in ev)
        cn = counts.cpu().numpy().view(np.uint32).copy()
        native = {"ms_per_step": ms_native, "walk_steps_per_s": int(cn.astype(np.int64).sum()) / (ms_native * 1e-3),
                  "accuracy_vs_fp64": accuracy.measured_accuracy(mu, B, L, accuracy.count_topk(np.arange(nv), cn, 100),
                                                                 counts=cn, k=100)}
        return {"metric": "walk-steps/s", "value": nsteps / (ms * 1e-3), "unit": "walk-steps/s", "workload": "ppr1",
                "n_gpus": 1, "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
                "higher_is_better": True, "dtype": "u32", "data": "synthetic",
                "config": {"workload": f"single-source PPR, R-MAT scale {scale} ef {args.edge_factor}, {B} walks "
                                       f"from the generator's vertex 0 (id {src} after permutation, the top "
                                       f"out-degree vertex), stop p=0.15, dangling->source, L<=20",
                           "walk_steps": nsteps},
                "queries_per_s": 1e3 / ms,
                "ppr_api": {"device_ms": statistics.median(api_dev), "wall_ms": statistics.median(api_wall),
                            "what": "gw_ppr_run, one query of the same walks, batch tag + walk + top-100, warm"},
                "accuracy_vs_fp64": acc, "native_rng": native, "gpu_launches": steps}
    finally:
        G.close()


def ppr1_arm(args) -> None:
    line = ppr1_measure(args)
    line["scaling"], line["vs_baseline"] = "weak", None
    print(json.dumps(line), flush=True)


def ooc_measure(args) -> dict:
    """Out-of-core raw random walks: the CSR held in pinned host memory as 256
    blocks, streamed into a bounded number of device block slots by the
    blocked engine (state-aware scheduling, double-buffered copies on a side
    stream); one walk per vertex, L = 10, 64-bit walk state resident.  The
    same walks also run with the graph resident (one launch, and the block
    loop), and all three give the same counts."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    torch.cuda.set_device(0)
    scale = extra_scale(args, 27)
    ef = args.edge_factor if args.edge_factor != 16 else 48
    nblocks = args.nblocks if args.nblocks != 32 else 256
    kb = blocksize_kb_for(scale, ef, nblocks)
    t0 = time.perf_counter()
    G = gw.Graph.rmat(scale, ef, seed=args.graph_seed, blocksize_kb=kb)
    gen_s = time.perf_counter() - t0
    try:
        nv, L = G.nv, args.L
        slots = args.nmblocks if args.nmblocks else max(1, (G.nblocks * 73) // 100)
        graph_bytes = (nv + 1) * 8 + G.ne * 4
        res, first, same = {}, None, True
        # the same walks (the context's pools, kept across runs) four ways:
        # one resident launch, the resident block loop, streamed blocks each
        # copied into a slot when chosen (findSubGraph), and streamed blocks
        # with the small pools' blocks read in place (the default)
        G.walks_clear()
        G.add_walks_at(np.arange(nv, dtype=np.uint32))
        # untimed first block loop: grows the block pools and loads the kernels
        t_first = time.perf_counter()
        G.run(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, L, seed=args.walk_seed, mode=gw.MODE_BLOCKED, prob=0.2))
        first_s = time.perf_counter() - t_first
        mapped_default = gw.MAPPED_AUTO if args.mapped_walks == "auto" else int(args.mapped_walks)
        modes = [("resident_one_launch", gw.RESIDENT_HBM, gw.MODE_RESIDENT, gw.MAPPED_AUTO, 0),
                 ("resident_blocked", gw.RESIDENT_HBM, gw.MODE_BLOCKED, gw.MAPPED_AUTO, 0),
                 ("streamed_blocked_copy_all", gw.STREAM_PINNED, gw.MODE_BLOCKED, 0, 0),
                 ("streamed_blocked", gw.STREAM_PINNED, gw.MODE_BLOCKED, mapped_default, 0)]
        if args.pool_budget_mb:
            modes.append(("streamed_blocked_pool_budget", gw.STREAM_PINNED, gw.MODE_BLOCKED, mapped_default,
                          args.pool_budget_mb << 20))
        for name, residency, mode, mapped, budget in modes:
            G.set_residency(residency, nmblocks=slots)
            G.set_mapped_block_walks(mapped)
            G.set_pool_budget(budget)
            st = G.run(gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT, L, seed=args.walk_seed, mode=mode, prob=0.2))
            counts = G.read_counts()
            if int(counts.astype(np.int64).sum()) != nv * L:
                raise RuntimeError(f"{name}: visit total differs from {nv * L}")
            if first is None:
                first = counts
            else:
                same = same and bool(np.array_equal(counts, first))
            res[name] = {"ms": st.ms_total, "walk_steps_per_s": nv * L / (st.ms_total * 1e-3),
                         "supersteps": int(st.supersteps), "block_loads": int(st.block_loads),
                         "h2d_GB": st.bytes_h2d / 1e9,
                         "h2d_GBps": st.bytes_h2d / (st.ms_total * 1e-3) / 1e9 if st.bytes_h2d else 0.0,
                         "blocks_read_in_place": {"supersteps": int(st.mapped_supersteps),
                                                  "walks": int(st.mapped_walks)},
                         "pools": {"budget_bytes": int(budget), "spilled": int(st.pools_spilled),
                                   "refilled": int(st.pools_refilled)},
                         "device_ms": {"walk": st.ms_walk, "partition": st.ms_partition,
                                       "copy_wait": st.ms_copy_wait}}
        link = host_link_gbps()
        for r in res.values():
            r["h2d_link_utilisation"] = r["h2d_GBps"] / link
        s = res["streamed_blocked"]
        return {"metric": "walk-steps/s", "value": s["walk_steps_per_s"], "unit": "walk-steps/s", "workload": "ooc",
                "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": s["ms"], "higher_is_better": True,
                "dtype": "u32", "data": "synthetic",
                "config": {"workload": f"out-of-core raw random walks, R-MAT scale {scale} ef {ef}, {G.nblocks} blocks "
                                       f"in pinned host memory, {slots} device block slots, one walk per vertex, "
                                       f"L={L}, jump rule", "graph_GB": graph_bytes / 1e9, "generate_s": gen_s,
                           "in_place_limit": args.mapped_walks},
                "host_link_GBps": link, "modes": res, "identical_counts_across_modes": same,
                "first_block_loop_wall_s": first_s,
                "speedup_vs_copy_all": res["streamed_blocked_copy_all"]["ms"] / s["ms"]}
    finally:
        G.close()


def host_link_gbps() -> float:
    """Host-to-device rate of one 1 GiB copy from pinned memory (best of 3),
    the denominator of the streamed runs' link utilisation."""
    import torch
    src = torch.empty(1 << 30, dtype=torch.uint8).pin_memory()
    dst = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
    best = 0.0
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dst.copy_(src, non_blocking=True)
        b.record()
        torch.cuda.synchronize()
        best = max(best, (1 << 30) / (a.elapsed_time(b) * 1e-3) / 1e9)
    del src, dst
    torch.cuda.empty_cache()
    return best


def ooc_arm(args) -> None:
    line = ooc_measure(args)
    line["scaling"], line["vs_baseline"] = "weak", None
    print(json.dumps(line), flush=True)


def edge_list_text(src, dst) -> "np.ndarray":
    """'<src> <dst>\n' lines of two CUDA integer tensors, formatted on the GPU
    (input preparation for the convert workload); returns host bytes as uint8."""
    import torch
    s, d = src.to(torch.int64), dst.to(torch.int64)

    def ndigits(x):
        n = torch.ones_like(x)
        p = 10
        for _ in range(9):
            n += (x >= p).to(torch.int64)
            p *= 10
        return n

    ns, nd = ndigits(s), ndigits(d)
    end = torch.cumsum(ns + nd + 2, 0)
    start = end - (ns + nd + 2)
    buf = torch.full((int(end[-1].item()),), 32, dtype=torch.uint8, device=s.device)
    for k in range(10):
        p10 = 10 ** k
        m = ns > k
        buf[start[m] + ns[m] - 1 - k] = (48 + (s[m] // p10) % 10).to(torch.uint8)
        m = nd > k
        buf[start[m] + ns[m] + nd[m] - k] = (48 + (d[m] // p10) % 10).to(torch.uint8)
    buf[end - 1] = 10
    return buf.cpu().numpy()


def convert_arm(args) -> None:
    """Graph preprocessing: a text edge list (an R-MAT graph, lines grouped by
    source as the reference requires) to the reference's preprocessed files,
    on the device (gw_convert_edgelist) against the reference's own
    convert_if_notexists compiled from source on a prefix of the same text."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    torch.cuda.set_device(0)
    scale = args.scale if args.scale != 24 else 23
    kb = blocksize_kb_for(scale, args.edge_factor, args.nblocks)
    with gw.Graph.rmat(scale, args.edge_factor, seed=args.graph_seed, blocksize_kb=kb) as G:
        rp, ci = G.export_csr()
    src = torch.repeat_interleave(torch.arange(len(rp) - 1, device="cuda"),
                                  torch.from_numpy(np.diff(rp.astype(np.int64))).cuda())
    text = edge_list_text(src, torch.from_numpy(ci.astype(np.int64)).cuda())
    del src
    torch.cuda.empty_cache()
    ne = len(ci)
    with tempfile.TemporaryDirectory(prefix="gw_conv_") as td:
        path = Path(td) / "rmat.txt"
        text.tofile(path)
        runs = []
        for _ in range(max(1, args.warmup) + max(1, args.steps)):
            runs.append(gw.convert_edgelist(str(path), kb))
        timed = runs[max(1, args.warmup):]
        st = sorted(timed, key=lambda r: r.ms_total)[len(timed) // 2]
        out_dir = Path(str(path) + "_GraphWalker")
        # the text names vertices up to its largest id; the generator's row pointer continues flat after it
        got_rp = np.fromfile(out_dir / "graphinfo" / "file_0.beg_pos", np.uint64)
        ok_full = (np.array_equal(got_rp, rp[: len(got_rp)]) and bool(np.all(rp[len(got_rp):] == ne))
                   and np.array_equal(np.fromfile(out_dir / "graphinfo" / "file_0.csr", np.uint32), ci))
        # the reference on a prefix of whole lines (a bounded sample), ours on the same prefix
        cpu, same = None, None
        if not args.no_cpu_baseline:
            exe = ROOT / "oracle" / "_ref" / "gw_ref_convert"
            cut = int(min(len(text), args.convert_sample_mb << 20))
            cut = int(np.flatnonzero(text[:cut] == 10)[-1]) + 1
            sample = Path(td) / "sample.txt"
            text[:cut].tofile(sample)
            ref = Path(td) / "sample_ref.txt"
            os.link(sample, ref)
            t0 = time.perf_counter()
            subprocess.run([str(exe), str(ref), str(kb)], check=True, capture_output=True)
            ref_s = time.perf_counter() - t0
            mine = gw.convert_edgelist(str(sample), kb)
            a, b = Path(str(sample) + "_GraphWalker"), Path(str(ref) + "_GraphWalker")
            same = all((a / f).read_bytes() == (b / f).read_bytes()
                       for f in ("graphinfo/file_0.beg_pos", "graphinfo/file_0.csr", "N.nvertices",
                                 "filesize_1024GB.filerange", f"blocksize_{kb}KB.blockrange"))
            cpu = {"value": mine.edges / ref_s, "unit": "edges/s", "cores": 1, "kind": "reference",
                   "sample": f"the reference's convert_if_notexists (conversions.hpp) compiled -O3 from source, "
                             f"single-threaded as written, on the first {cut} bytes ({mine.lines} lines) of the "
                             f"same text; {ref_s:.2f} s"}
    line = {"metric": "edges/s", "value": ne / (st.ms_total * 1e-3), "unit": "edges/s", "workload": "convert",
            "n_gpus": 1, "steps": max(1, args.steps), "warmup": max(1, args.warmup), "ms_per_step": st.ms_total,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"text edge list -> preprocessed CSR + block range, R-MAT scale {scale} "
                                   f"ef {args.edge_factor} ({len(text)} bytes, {ne} lines, grouped by source), "
                                   f"blocksize {kb} KB; the text file is in the page cache"},
            "text_GBps": len(text) / (st.ms_total * 1e-3) / 1e9,
            "breakdown_ms": {"read": st.ms_read, "device": st.ms_device, "write": st.ms_write},
            "identical_to_generator_csr": bool(ok_full), "identical_to_reference_on_sample": same,
            "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def simrank_arm(args) -> None:
    """Batched SimRank (apps/simrank.cpp semantics: R walks of L - 1 hops from
    each vertex under the restart rule, replica i from hop i*L; first-meeting
    reduction): queries/s of one gw_simrank_batch call against the reference's
    simrank app, unchanged, one query per process as it runs."""
    import numpy as np
    import torch

    import graphwalker_b200 as gw
    torch.cuda.set_device(0)
    R, L, nq = 1000, 11, args.queries
    kb = blocksize_kb_for(args.scale, args.edge_factor, args.nblocks)
    G = gw.Graph.rmat(args.scale, args.edge_factor, seed=args.graph_seed, blocksize_kb=kb)
    rng = np.random.default_rng(13)
    # the app asserts getblock(a) == getblock(b): pairs inside one block
    blocks = G.blocks.astype(np.int64)
    blk = rng.integers(0, G.nblocks, nq)
    lo, hi = blocks[blk], blocks[blk + 1]
    a = (lo + rng.integers(0, 1 << 62, nq) % (hi - lo)).astype(np.uint32)
    b = (lo + rng.integers(0, 1 << 62, nq) % (hi - lo)).astype(np.uint32)
    for _ in range(max(1, args.warmup)):
        G.simrank_batch(a, b, R, L, seed=args.walk_seed)
    times = []
    with ClockSampler(device_uuid(0)) as clk:
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            scores, meet = G.simrank_batch(a, b, R, L, seed=args.walk_seed)
            times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    cpu = None
    if not args.no_cpu_baseline:
        rowptr, colidx = G.export_csr()
        exe = ROOT / "oracle" / "_ref" / "simrank"
        with tempfile.TemporaryDirectory(prefix="gw_ref_") as td:
            tmp = Path(td)
            base, _, _ = write_reference_graph(tmp, args, rowptr, colidx)
            del rowptr, colidx
            wall = []
            for q in range(min(nq, 5)):
                t0 = time.perf_counter()
                r = subprocess.run([str(exe), "file", base, "a", str(a[q]), "b", str(b[q]), "R", str(R), "L", str(L),
                                    "blocksize_kb", str(kb)], cwd=tmp, capture_output=True, text=True, timeout=600)
                wall.append(time.perf_counter() - t0)
                if r.returncode != 0:
                    raise RuntimeError(r.stderr[-500:])
            cpu = {"value": 1.0 / statistics.median(wall), "unit": "queries/s", "cores": host_cores(),
                   "kind": "reference",
                   "sample": f"apps/simrank.cpp unchanged, compiled -O3 from source with native rand_r, one process "
                             f"per query as the app runs, {len(wall)} queries of the same batch "
                             f"(median {statistics.median(wall) * 1e3:.1f} ms each, graph files in the page cache)"}
    line = {"metric": "queries/s", "value": nq / t, "unit": "queries/s", "workload": "simrank", "n_gpus": 1,
            "steps": max(1, args.steps), "warmup": max(1, args.warmup), "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"batched SimRank, R-MAT scale {args.scale} ef {args.edge_factor}, {nq} pairs "
                                   f"inside one block each, R={R} walks per vertex, L={L}, decay 0.8",
                       "api": "gw_simrank_batch (host arrays in, scores out)"},
            "mean_score": float(np.mean(scores)), "pairs_meeting": int((meet.sum(1) > 0).sum()),
            "cpu_baseline": cpu, "clocks": clk.summary()}
    G.close()
    print(json.dumps(line), flush=True)


def gather_arm(args) -> None:
    """gw_probe_gather alone: `--probe-loads` loads of 4 B from distinct
    random 32-B sectors of a `--probe-mb` buffer (a warm-up launch and two
    timed ones), for profiler captures of the random-miss cost."""
    import torch

    import graphwalker_b200 as gw
    torch.cuda.set_device(0)
    with gw.Graph.rmat(10, 4, seed=1, blocksize_kb=64) as G:
        if args.probe_host:  # pinned host memory: its address is valid on the device
            buf = torch.zeros(args.probe_mb << 18, dtype=torch.int32).pin_memory()
        else:
            buf = torch.zeros(args.probe_mb << 18, dtype=torch.int32, device="cuda")
        bps = G.probe_gather(buf.data_ptr(), buf.numel(), args.probe_loads, iters=2)
    print(json.dumps({"workload": "gather", "buffer_MB": args.probe_mb, "loads": args.probe_loads,
                      "memory": "pinned host" if args.probe_host else "device",
                      "useful_GBps_32B": bps / 1e9, "loads_per_s": bps / 32}), flush=True)


def walkonly_arm(args) -> None:
    """`--steps` launches of the resident walk kernel over one walk per vertex
    (jump rule, counts), at full occupancy and without the autotuner, for
    profiler captures at a chosen --scale."""
    import torch

    import graphwalker_b200 as gw
    torch.cuda.set_device(0)
    with gw.Graph.rmat(args.scale, args.edge_factor, seed=args.graph_seed,
                       blocksize_kb=blocksize_kb_for(args.scale, args.edge_factor, args.nblocks)) as G:
        layout = "erec" if G.set_edge_records(LAYOUT_MODE[args.layout]) else "csr"
        nv = G.nv
        v = torch.arange(nv, dtype=torch.int64, device="cuda")
        walks = torch.stack([v, v, v, torch.zeros_like(v)], 1).to(torch.int32).contiguous()
        del v
        counts = torch.zeros(nv, dtype=torch.int32, device="cuda")
        p = gw.params(gw.RULE_JUMP, gw.SINK_VERTEX_COUNT if args.sink == "count" else gw.SINK_NONE, args.L,
                      seed=args.walk_seed, rng=gw.RNG_NATIVE if args.rng == "native" else gw.RNG_PHILOX,
                      cache_hints=None if args.hints < 0 else args.hints)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(max(1, args.steps))]
        for a, b in ev:
            counts.zero_()
            a.record()
            G.walk_device(p, walks, nv, counts=counts)
            b.record()
        G.sync()
        visits = int(counts.to(torch.int64).sum().item())
    print(json.dumps({"workload": "walkonly", "scale": args.scale, "graph_layout": layout, "rng": args.rng,
                      "hints": args.hints, "sink": args.sink,
                      "launch_ms": [a.elapsed_time(b) for a, b in ev], "visits": visits}), flush=True)


def main():
    args = parse_args()
    if args.workload == "gather" and args.impl != "reference":
        gather_arm(args)
        return
    if args.workload == "walkonly" and args.impl != "reference":
        walkonly_arm(args)
        return
    if args.workload == "simrank" and args.impl != "reference":
        simrank_arm(args)
        return
    if args.workload == "convert" and args.impl != "reference":
        convert_arm(args)
        return
    if args.workload == "ooc" and args.impl != "reference":
        ooc_arm(args)
        return
    if args.workload == "ppr1" and args.impl != "reference":
        ppr1_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    elif args.workload == "msppr":
        msppr_arm(args)
    elif args.workload == "serve":
        serve_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
