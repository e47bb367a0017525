"""Host-side measurement helpers of bench.py (no GPU): the algorithmic byte count the roofline
uses, the parsing of the nvidia-smi clock samples taken during the timed region, and the peak
lookup with its fallback."""

import json
import os
import tempfile

import numpy as np

import bench
from newton_b200 import scenes


def test_gate_configs_and_workload_configs():
    """Every gated workload has a tolerance; the config object is the same for both arms."""
    for wl in bench.WORKLOADS:
        g = bench.gate_config(wl)
        if wl == "cloth-on-boxes":
            assert g is None  # the gate is not available with self-contact
        else:
            assert g["tolerance"] > 0 and g["max_iterations"] == bench.GATE_CAP and g["residual"] == "sweep"
    model, _ = scenes.draped_cloth(n=16, device="cpu", height=0.904)
    cfg = bench.workload_config("draped-cloth", model, bench.gate_config("draped-cloth"))
    assert cfg["vertices"] == 256 and cfg["settle_steps"] == bench.SETTLE and cfg["residual_gate"]["norm"] == "mean"
    json.dumps(cfg)


def test_algorithmic_bytes_follow_the_per_element_formula():
    model, _ = scenes.hanging_cloth(seed=0, device="cpu")
    adj = model.soft_mesh_adjacency
    n_csr = (len(adj.v_adj_tris) + len(adj.v_adj_edges)) // 2
    V, T, E = model.particle_count, model.tri_count, model.edge_count
    expect = 60 * V + 44 * T + 32 * E + 8 * n_csr + 8 * (V + 1)
    assert bench.algorithmic_bytes_per_iteration(model) == expect
    # a regular grid: every triangle appears in 3 vertex rows; ~394 B per vertex-iteration at scale
    assert len(adj.v_adj_tris) // 2 == 3 * T
    per_vertex = expect / V
    assert 300.0 < per_vertex < 420.0


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _sampler_with(lines):
    s = bench.ClockSampler(0)
    fd, path = tempfile.mkstemp(suffix=".csv")
    with os.fdopen(fd, "w") as f:
        f.write("\n".join(lines) + "\n")
    s.path = path
    s.f = open(os.devnull, "w")
    s.proc = _FakeProc()
    return s


def test_clock_samples_give_median_max_and_active_reasons():
    rows = [
        "0, 1965, 1965, 700.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 701.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ]
    out = _sampler_with(rows).stop()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3,
                   "source": "nvidia-smi, 200 ms"}


def test_nvml_clock_samples_give_median_max_and_active_reasons():
    s = bench.ClockSampler(0)
    s.thread, s.stop_flag, s.max_mhz = _FakeThread(), False, 1965
    s.samples = [(1965, 0x0), (1950, 0x4), (1965, 0x0), (1200, 0x8 | 0x20)]
    out = s.stop()
    assert out == {"sm_mhz": 1957.5, "sm_max_mhz": 1965, "samples": 4, "source": "nvml, 1 ms",
                   "reasons": ["hw_slowdown", "sw_power_cap", "sw_thermal_slowdown"]}


class _FakeThread:
    def join(self, timeout=None):
        pass


def test_clock_samples_flag_the_rejecting_reasons():
    rows = ["0, 1200, 1965, 800.0, 0x0000000000000008, Active, Not Active, Active, Not Active"]
    out = _sampler_with(rows).stop()
    assert out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert out["sm_mhz"] == 1200.0


def test_clock_sampler_without_samples_reports_none():
    assert _sampler_with([]).stop() is None
    s = bench.ClockSampler(0)
    assert s.stop() is None  # never started


def test_measured_peaks_read_the_file_or_fall_back(tmp_path, monkeypatch):
    here = os.path.dirname(os.path.abspath(bench.__file__))
    p = os.path.join(here, "MEASURED_PEAKS.json")
    peaks = bench.measured_peaks()
    if os.path.exists(p):
        with open(p) as f:
            assert peaks == {"hbm_gbs": float(json.load(f)["hbm_gbs"]), "source": "measured"}
    else:
        assert peaks == {"hbm_gbs": 6650.0, "source": "fallback"}
    # the fallback when the file cannot be read
    monkeypatch.setattr(bench.os.path, "abspath", lambda _p: str(tmp_path / "bench.py"))
    assert bench.measured_peaks() == {"hbm_gbs": 6650.0, "source": "fallback"}
