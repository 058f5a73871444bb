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


@pytest.mark.parametrize("scene", ["cache", "medium", "volume", "gdpt", "post", "rmse"])
def test_reference_arm_unavailable(scene):
    rc, lines, err = run(["--impl", "reference", "--scene", scene, "--steps", "1", "--warmup", "1"])
    assert rc == 0, err[-2000:]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unavailable"]


def test_recorded_ncu_figures_match_the_summaries():
    """The DRAM figures bench.py carries as recorded ncu traffic are the ones
    the committed ncu summaries state (bench.py itself reads no summary)."""
    sys.path.insert(0, ROOT)
    import bench

    def recorded(name, key):
        for line in open(os.path.join(ROOT, "profiles", name + ".md")):
            if line.strip().startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0].replace(",", ""))
        return None

    assert bench._read_traffic("heightfield") == recorded("k_extend_heightfield", "dram_bytes_per_launch")
    assert (bench.NCU_TRAFFIC["k_rc_infer heightfield"]["bytes_per_query"]
            == recorded("k_rc_infer_heightfield", "dram_bytes_per_query"))
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert "open(os.path.join(ROOT, \"profiles\"" not in src and ".md\")" not in src


@pytest.mark.skipif(not os.path.isdir(REF_LIB), reason="reference host build not present (build() makes it)")
def test_reference_arm_maps_no_library_code_and_prints_the_shared_config():
    """The reference arm's process maps the reference's host build and none of
    this library's shared objects, and its `config` is the dict the b200 arm
    prints for the same command line."""
    code = (
        "import runpy, sys, json\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--scene', 'cornell', '--steps', '2', '--warmup', '1',\n"
        "            '--reference-seconds', '1']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "libs = sorted({l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')})\n"
        "print('MAPPED ' + json.dumps(libs))\n")
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=e, timeout=240, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    mapped = json.loads([l for l in p.stdout.splitlines() if l.startswith("MAPPED ")][0][7:])
    ours = [m for m in mapped if m.startswith(ROOT)]
    assert ours and all("/oracle/_ref/" in m for m in ours), ours
    line = json.loads([l for l in p.stdout.splitlines() if l.startswith("{")][0])

    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(steps=2, warmup=1)
    desc = bench.make_scene("cornell", standalone=True)
    assert line["config"] == bench.path_config(bench.SCENES["cornell"], args, 1, desc)
