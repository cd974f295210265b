"""bench.py's reference arm, run on the CPU: it must time the reference's own
engine on the headline workload without loading any library of this
repository, and print the GPU arm's `config` so that the two lines compare
like for like."""
import json
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.skipif(
    not (ROOT / "oracle" / "_ref" / "gw_ref_bench").exists() or not (ROOT / "oracle" / "_build" / "gw_oracle_rmat").exists(),
    reason="the reference binaries are built by build() where the reference tree exists")

_RUN = """
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--scale", "12", "--steps", "2", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
maps = sorted({l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith(".so") and "{root}" in l})
print("MAPS " + json.dumps(maps))
"""


def test_reference_arm_is_clean_and_comparable():
    out = subprocess.run([sys.executable, "-c", _RUN.replace("{root}", str(ROOT))], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.splitlines()
    maps = json.loads(next(l for l in lines if l.startswith("MAPS "))[5:])
    assert maps == [], f"the reference arm loaded {maps}"
    line = json.loads(next(l for l in lines if l.startswith('{"metric"')))
    assert line["impl"] == "reference" and line["unit"] == "walk-steps/s" and line["value"] > 0
    assert "rand_r" in line["rng"]
    assert line["cpu_baseline"]["kind"] == "reference"
    assert set(line["single_thread_fallback"]) >= {"fired", "runs_fired", "runs", "execthreads"}
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    # the GPU arm's config for the same arguments
    sys.path.insert(0, str(ROOT))
    import bench
    sys_argv, sys.argv = sys.argv, ["bench.py", "--scale", "12", "--steps", "2", "--warmup", "1"]
    try:
        want = bench.workload_config(bench.parse_args(), line["config"]["nblocks"])
    finally:
        sys.argv = sys_argv
    assert line["config"] == want
