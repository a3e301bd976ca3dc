"""CPU test of bench.py's output contract through its reference arm, the
arm that runs without a GPU: one JSON line on stdout with the metric, the
value, the CPU-baseline record and an e2e record with no host-link bytes
(the reference's CPU path copies nothing to a device)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "frame256", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["unit"] == "Mpixel/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"].startswith("frame256")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port")
    assert d["e2e"] == {"value": d["value"], "unit": "Mpixel/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    # the reference's GPU kernel is timed beside it only where it can run
    import torch
    from oracle import refgpu
    assert ("reference_gpu" in d) == (torch.cuda.is_available() and refgpu.available())
    readings = cb["readings"]
    assert set(readings) == {"capped_all_cores", "unlimited_all_cores", "capped_one_core"}
    assert readings["capped_one_core"]["cores"] == 1
    assert all(r["value"] > 0 for r in readings.values())


def test_reference_arm_never_maps_this_library():
    """The reference arm times only the reference's code: it draws its
    workload with torch and must not load libncs_b200.so into its process."""
    code = (
        "import sys, os, io, contextlib\n"
        "sys.path.insert(0, %r)\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'frame256',\n"
        "            '--steps', '1', '--warmup', '0', '--no-compare-plain']\n"
        "import bench\n"
        "with contextlib.redirect_stdout(io.StringIO()):\n"
        "    rc = bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('MAPPED' if 'libncs_b200.so' in maps else 'CLEAN', rc)\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN 0", r.stdout
