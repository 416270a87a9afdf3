"""Host-side arithmetic of the bench line (no GPU): the roofline entries
(tensor flops, FP64 operations per QPE, HBM bytes over each class's event
time against the peaks) and the clock summary parsed from nvidia-smi rows."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture
def bench(monkeypatch):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    b = importlib.import_module("bench")
    monkeypatch.setattr(b, "_peaks", lambda: ({"hbm_gbs": 6400.0, "bf16_tflops": 1700.0,
                                                "bf16_tflops_sustained": 1400.0}, "measured"))
    monkeypatch.setattr(b, "_traffic", lambda: {"gemm": 1000, "quad_fp64_ops_per_qpe": 80.0})
    return b


CLASSES = {
    # work: flops (gemm), QPE (quad), bytes (trsv); ms summed over the launches
    "gemm": dict(launches=10, ms=20.0, work=7.0e12),
    "quad": dict(launches=4, ms=8.0, work=1.0e9),
    "trsv": dict(launches=5, ms=10.0, work=3.2e10),
    "other": dict(launches=100, ms=50.0, work=0.0),
}


def test_roofline_dominant_class_is_the_longest_of_ours(bench):
    r = bench.roofline(CLASSES)
    assert r["kernel"] == "gemm"           # "other" never counts as the dominant class
    # 7e12 / 10 launches = 7e11 flop per launch over 2 ms = 350 TFLOP/s
    assert r["achieved"] == pytest.approx(350.0)
    assert r["frac"] == pytest.approx(350.0 / 1400.0)
    assert r["bound"] == "tensor" and r["traffic"] == 1000
    assert r["ms_per_launch"] == pytest.approx(2.0)


def test_roofline_of_the_quadrature_uses_fp64_operations_per_qpe(bench):
    r = bench.roofline(CLASSES, "quad", fp64_peak=35.0)
    # 2.5e8 QPE per launch in 2 ms = 125 G QPE/s, times 80 operations = 10 TFLOP/s
    assert r["gqpe_per_s"] == pytest.approx(125.0)
    assert r["achieved"] == pytest.approx(10.0)
    assert r["frac"] == pytest.approx(10.0 / 35.0)
    assert r["bound"] == "fp64"


def test_roofline_of_an_hbm_class(bench):
    r = bench.roofline(CLASSES, "trsv")
    # 6.4e9 bytes per launch in 2 ms = 3200 GB/s of 6400
    assert r["achieved"] == pytest.approx(3200.0)
    assert r["frac"] == pytest.approx(0.5)
    assert r["bound"] == "hbm" and r["traffic"] is None


def test_roofline_of_a_missing_class(bench):
    assert bench.roofline(CLASSES, "panel") is None
    assert bench.roofline({"other": dict(launches=1, ms=1.0, work=0.0)}) is None


def test_clock_summary(bench):
    c = bench.ClockSampler(0)
    c.rows = [
        ["0", "1965", "1965", "700.1", "0x0000000000000004", "Not Active", "Not Active", "Not Active", "Active"],
        ["0", "1830", "1965", "990.0", "0x0000000000000004", "Not Active", "Not Active", "Not Active", "Active"],
        ["0", "1900", "1965", "950.0", "0x0000000000000000", "Not Active", "Not Active", "Not Active",
         "Not Active"],
    ]
    s = c.summary()
    assert s["sm_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
