"""Host-side pieces of bench.py on the CPU: the clock record taken during the
timed region (median SM clock, throttle reasons, samples inside the window),
the roofline denominator, and the reference arm on ranks other than 0."""
import json
import os
import time
from types import SimpleNamespace

import pytest

import bench


class _Proc:
    def terminate(self):
        pass

    def wait(self):
        return 0


def _sampler(tmp_path, rows):
    """A ClockSampler whose nvidia-smi output is `rows` (no process runs)."""
    s = object.__new__(bench.ClockSampler)
    s.path = str(tmp_path / "clocks.csv")
    with open(s.path, "w") as f:
        for r in rows:
            f.write(r + "\n")
    s.f = open(os.devnull, "w")
    s.p = _Proc()
    return s


def _row(ts, sm, reasons=("Not Active",) * 4, mx=1965):
    stamp = time.strftime("%Y/%m/%d %H:%M:%S", time.localtime(ts)) + ".123"
    return ", ".join([stamp, str(sm), str(mx), "812.5", "0x0000000000000000"] + list(reasons))


def test_clock_record_inside_the_timed_window(tmp_path, monkeypatch):
    monkeypatch.setattr(bench.time, "sleep", lambda s: None)
    t0 = float(int(time.time()))
    rows = [_row(t0 - 30, 600, ("Active", "Not Active", "Not Active", "Not Active"))]   # before: ignored
    rows += [_row(t0 + k, 1965 if k != 2 else 1900) for k in range(5)]
    rows += [_row(t0 + 4, 1800, ("Not Active", "Not Active", "Not Active", "Active"))]
    rows += ["garbage line", ""]
    clk = _sampler(tmp_path, rows).stop(t0, t0 + 4)
    assert clk["samples"] == 6
    assert clk["sm_mhz"] == 1965.0 and clk["sm_max_mhz"] == 1965.0
    # only sw_power_cap was active inside the window; the hw_slowdown sample
    # thirty seconds earlier is outside it
    assert clk["reasons"] == ["sw_power_cap"]


def test_clock_record_names_every_slowdown_reason(tmp_path, monkeypatch):
    monkeypatch.setattr(bench.time, "sleep", lambda s: None)
    t0 = float(int(time.time()))
    rows = [_row(t0, 1200, ("Active", "Active", "Active", "Not Active"))]
    clk = _sampler(tmp_path, rows).stop(t0, t0 + 1)
    assert clk["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert clk["sm_mhz"] == 1200.0


def test_no_clock_record_without_samples(tmp_path, monkeypatch):
    monkeypatch.setattr(bench.time, "sleep", lambda s: None)
    assert _sampler(tmp_path, []).stop(0.0, 1.0) is None
    s = object.__new__(bench.ClockSampler)
    s.p = None
    assert s.stop(0.0, 1.0) is None


def test_roofline_denominator_is_the_measured_copy_bandwidth():
    peak, kind = bench.peaks()
    p = os.path.join(bench.ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        assert kind == "measured" and peak == pytest.approx(float(json.load(open(p))["hbm_gbs"]))
    else:
        assert (peak, kind) == (6650.0, "fallback")


def test_reference_arm_runs_on_rank_zero_only(capsys):
    args = SimpleNamespace(instances=4, steps=1, warmup=3)
    assert bench.run_reference(args, 2, 1) is None
    assert capsys.readouterr().out == ""


def test_reference_sample_fits_the_per_step_time():
    fields = [SimpleNamespace(n=n) for n in (1000, 5000, 200, 16000, 300, 9000)]
    # 0.02 s a step on 2 cores: 0.02 * 3e5 * 2 floe-steps
    s = bench.reference_sample(fields, 0.02, 2)
    assert [f.n for f in s] == [1000, 5000, 200, 16000, 300, 9000][:len(s)]
    assert 0 < sum(f.n for f in s) <= 0.02 * bench.ORACLE_RATE_PER_CORE * 2
    # a long step takes every instance; a sample never comes back empty
    assert len(bench.reference_sample(fields, 2.0, 4)) == len(fields)
    assert len(bench.reference_sample([SimpleNamespace(n=10 ** 9)], 0.05, 1)) == 1


def test_reference_arm_json_line(capsys):
    """The reference arm end to end on a 4-instance ensemble: one JSON line
    with the contract's keys, the CPU port timed on the host cores."""
    args = SimpleNamespace(instances=4, steps=2, warmup=3)
    bench.run_reference(args, 1, 0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == bench.UNIT
    assert line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["instances"] == 4


def test_cpu_baseline_stops_after_its_time():
    from godar_b200 import generators as gen
    fields = [gen.ensemble_member(i, n) for i, n in enumerate((600, 900, 400))]
    t = time.perf_counter()
    rate, procs, desc = bench.cpu_oracle_rate(fields, 1.0, 2)
    assert rate > 0 and procs == 2 and "3 of 3 ensemble instances" in desc
    assert time.perf_counter() - t < 60
