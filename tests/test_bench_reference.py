"""The reference arm of bench.py (`--impl reference`) on the host cores.

The arm times the oracle's restatement of ASMBLE_DRIVER (the Fortran
reference cannot be compiled in this image) on the headline workload.  It
must print one JSON line with the arm's contract (impl, metric, unit, value,
config, cpu_baseline, an e2e with no host-device bytes) and must not load
this library's libfem25gpu.so in any of its processes: the timed work is the
reference's path only.  Runs on CPU (one bounded sample step, about 20 s)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_contract_and_no_product_library():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    out = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert out["impl"] == "reference"
    assert out["metric"] == bench.METRIC and out["unit"] == bench.UNIT
    assert out["value"] > 0 and out["higher_is_better"] is True
    assert out["steps"] == 1 and out["n_gpus"] == 1
    cfg = out["config"]
    assert cfg["systems_per_step"] == 512 and cfg["nelem"] == 48000
    base = out["cpu_baseline"]
    assert base["kind"] == "port" and base["cores"] >= 1 and base["value"] == out["value"]
    assert out["e2e"] == {"value": out["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    assert out["product_library_loaded"] is False
