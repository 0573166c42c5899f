"""Host-side pieces of bench.py's JSON line, checked without a GPU: the clock
record (median SM clock, throttle reasons) parsed from nvidia-smi samples, the
committed DRAM traffic per particle that `roofline.traffic` scales, the source
of the HBM peak, and the per-particle state bytes behind the algorithmic byte
count of the fused kernel."""
import json

import bench
from ckmpm_b200 import _capi as capi


class _FinishedProcess:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def test_clock_record_from_samples():
    s = bench.ClockSampler("0")
    s.proc = _FinishedProcess()
    s.lines = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 812.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, [N/A], 1965, 812.5, 0x0, Not Active, Not Active, Not Active, Not Active",
        "short, line",
        "",
    ]
    assert s.stop() == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    s = bench.ClockSampler("0")
    s.proc = _FinishedProcess()
    s.lines = ["0, 1200, 1965, 1000.0, 0x8, Active, Not Active, Active, Not Active"]
    assert s.stop()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert bench.ClockSampler("0").stop()["reasons"] == ["nvidia-smi unavailable"]


def test_committed_traffic_matches_the_profiles():
    table = json.loads((bench.ROOT / "profiles" / "traffic.json").read_text())
    for name in ("sand_column", "batched_256"):
        assert bench.committed_traffic(name) == table[name]["dram_bytes_per_particle"]
        per_launch = table[name]["dram_bytes_per_launch"]
        assert 100.0 < bench.committed_traffic(name) < 300.0 and per_launch > 1e8
    assert bench.committed_traffic("no_such_workload") is None


def test_hbm_peak_source(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_peak() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6548.5}))
    assert bench.measured_peak() == (6548.5, "measured")
    (tmp_path / "MEASURED_PEAKS.json").write_text("not json")
    assert bench.measured_peak() == (6650.0, "fallback")


def test_state_bytes_per_material():
    x, F, scalar = 12, 36, 4
    assert bench.STATE_BYTES == {
        capi.FIXED_COROTATED: x + F,
        capi.LINEAR: x + F + F,          # and the stored stress Q
        capi.DRUCKER_PRAGER: x + F + scalar,  # logJp
        capi.FLUID: x + scalar,          # J
        capi.VON_MISES: x + F + scalar,  # rigid flag
        capi.NACC: x + F + scalar,       # logJp
    }
