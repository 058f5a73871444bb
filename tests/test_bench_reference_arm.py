"""bench.py's reference arm (`--impl reference`) on the CPU: the reference's
own host-compiled path tracer timed on this machine's cores, printed as one
JSON line with the keys the bench contract asks for; rank > 0 under a
multi-process launch prints nothing and exits 0; scenes without a reference
counterpart print their `unavailable` line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref")


def run(args, env=None, timeout=240):
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    e.update(env or {})
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       env=e, timeout=timeout, cwd=ROOT)
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    return p.returncode, lines, p.stderr


@pytest.mark.skipif(not os.path.isdir(REF_LIB), reason="reference host build not present (build() makes it)")
def test_reference_arm_line():
    rc, lines, err = run(["--impl", "reference", "--scene", "cornell", "--steps", "1", "--warmup", "1",
                          "--reference-seconds", "1"])
    assert rc == 0, err[-2000:]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "Mpaths/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port") and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_nothing():
    rc, lines, err = run(["--impl", "reference", "--scene", "cornell", "--steps", "1", "--warmup", "1"],
                         env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert rc == 0, err[-2000:]
    assert lines == []


@pytest.mark.parametrize("scene", ["cache", "medium"])
def test_reference_arm_unavailable(scene):
    rc, lines, err = run(["--impl", "reference", "--scene", scene, "--steps", "1", "--warmup", "1"])
    assert rc == 0, err[-2000:]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unavailable"]


def test_profile_figures_the_bench_reads():
    """The DRAM figures the bench's roofline `traffic` keys come from are
    present in the committed ncu summaries and parse as numbers."""
    sys.path.insert(0, ROOT)
    import bench
    per_launch = bench._read_traffic("heightfield")
    per_query = bench._read_profile_value("k_rc_infer_heightfield", "dram_bytes_per_query")
    assert per_launch is not None and per_launch > 1e8
    assert per_query is not None and 96.0 <= per_query < 1000.0
