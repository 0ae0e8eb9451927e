"""Host-side helpers of bench.py that shape its JSON line: the clock record
taken with nvidia-smi during the timed region (median SM clock, the maximum,
and which throttle reasons were active) and the workload description shared
by both arms.  CPU only: the nvidia-smi process is replaced by a file of
sampled rows."""
import os
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _Done:
    def terminate(self):
        pass

    def wait(self):
        return 0


def _clocks_from(rows):
    c = bench.Clocks.__new__(bench.Clocks)
    c.dev = 0
    c.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
    c.f.write("\n".join(rows) + "\n")
    c.f.flush()
    c.p = _Done()
    return c.stop()


def test_clock_record_median_and_reasons():
    na, act = "Not Active", "Active"
    rows = [f"0, {mhz}, 1965, 900.5, 0x0, {na}, {na}, {na}, {cap}"
            for mhz, cap in ((1965, na), (1950, act), (1965, na), (1800, act), (1965, na))]
    rec = _clocks_from(rows)
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"] and rec["samples"] == 5


def test_clock_record_reports_slowdowns_and_skips_bad_rows():
    na, act = "Not Active", "Active"
    rows = [f"0, 1200, 1965, 700.0, 0x8, {act}, {na}, {act}, {na}",
            "0, [N/A], [N/A], [N/A], [N/A]",
            f"0, 1300, 1965, 710.0, 0x8, {na}, {act}, {na}, {na}"]
    rec = _clocks_from(rows)
    assert rec["sm_mhz"] == 1250.0
    assert rec["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_clock_record_without_nvidia_smi():
    c = bench.Clocks.__new__(bench.Clocks)
    c.p = None
    rec = c.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]


def test_headline_config_names_the_workload():
    cfg = bench.headline_config(48000, 2302569, 247702329, 512)
    assert cfg["systems_per_step"] == 512 and cfg["nnz"] == 247702329
    assert "400x120" in cfg["workload"] and "512 complex128 CSR systems" in cfg["workload"]
    assert "L2" in cfg["l2"]
