"""bench.py's reference arm runs on the host cores alone (the reference's own
form_residual compiled as oracle/_ref): its one JSON line carries the
metric, config and the cpu_baseline / e2e objects the benchmark contract
asks for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the reference CPU build is absent
        assert isinstance(d["unavailable"], str) and d["unavailable"]
        return
    assert d["metric"] == "DOF-residual evals/s" and d["unit"] == "DOF/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1
    assert d["config"]["workload"] == "ns_mms_residual"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # the timed processes mapped no product library (their /proc/self/maps)
    assert d["product_libs_mapped"] == []
    # the same config object as the GPU arm's line
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.WORKLOAD
