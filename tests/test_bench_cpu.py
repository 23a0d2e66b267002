"""The host-side pieces of bench.py that go into its JSON line: the byte model
behind the roofline, the Curie-temperature fit, the guard on the Monte Carlo
comparison with the reference's own m(T), the reference arm's sample size and
the committed ncu traffic.  No GPU."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_byte_model_of_the_bench_workload():
    # compact 4-byte words, two materials, macrocell dipole, stored external field
    assert bench.byte_model(b_J=0, dipole=True) == {"predictor": 96, "corrector": 104}
    # 16-byte records carry the DMI vector per bond (12 B x 12 bonds)
    assert bench.byte_model(b_J=12, dipole=True) == {"predictor": 240, "corrector": 248}
    # without the stored field both passes regenerate the noise and the corrector reads the cell id
    assert bench.byte_model(b_J=0, dipole=True, noise_store=False) == {"predictor": 84, "corrector": 96}
    # no dipole field: no cell id in either pass
    assert bench.byte_model(b_J=0, dipole=False) == {"predictor": 92, "corrector": 104}


def test_tc_fit_recovers_a_power_law():
    T = np.arange(0.0, 1550.0, 50.0)
    tc = 1173.9
    m = np.where(T < tc, np.clip(1 - T / tc, 0, None) ** 0.35, 0.02)
    assert abs(bench._tc_fit(T, m) - tc) / tc < 1e-3


def test_mc_comparison_only_on_the_fixture_protocol():
    d = np.load(ROOT / "tests" / "golden" / "mc_sc50_curie.npz")
    T, ref, sweeps = d["T"], d["m_mean"], tuple(int(x) for x in d["sweeps"])
    tc_ref = bench._tc_fit(T, ref)
    got = bench.mc_reference_comparison(T, ref, tc_ref, sweeps)
    assert got["max_abs_m_dev"] == 0.0 and got["Tc_rel_dev"] == 0.0
    shifted = ref + 0.01
    assert abs(bench.mc_reference_comparison(T, shifted, tc_ref, sweeps)["max_abs_m_dev"] - 0.01) < 1e-12
    # another protocol (shorter sweeps, other temperatures) is not compared
    assert bench.mc_reference_comparison(T, ref, tc_ref, (500, 1000, 10)) is None
    assert bench.mc_reference_comparison(T[:-1], ref[:-1], tc_ref, sweeps) is None


@pytest.mark.parametrize("steps,L", [(20, 50), (150, 40), (300, 30), (2000, 20), (10**6, 20)])
def test_reference_sample_size(steps, L):
    assert bench.reference_sample_L(steps) == L


def test_committed_traffic_and_peak():
    t = json.loads((ROOT / "profiles" / "ncu_traffic.json").read_text())
    assert bench.traffic_from_profiles("predictor", "compact") == t["compact"]["predictor"]
    assert bench.traffic_from_profiles("predictor", "none") is None
    # measured traffic of the predictor is within 10 % of its byte model over 4M spins
    assert abs(t["compact"]["predictor"] / (96 * 4e6) - 1) < 0.1
    peak, kind = bench.measured_peak_hbm()
    if (ROOT / "MEASURED_PEAKS.json").exists():
        assert kind == "measured" and peak == json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
    else:
        assert kind == "fallback"


def test_workload_config_names_the_workload():
    c = bench.workload_config(100, 1)
    assert c["spins_per_gpu"] == 4_000_000 and c["cells"] == [100, 100, 100]
    assert "model" not in c and c["parallelism"] == "single GPU"
    assert bench.workload_config(100, 8)["parallelism"] == "replicas x8"
