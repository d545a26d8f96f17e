"""Host logic of bench.py that its headline numbers rest on, checked without a GPU: the time-to-1e-8-Ry rule
applied to a Davidson eigenvalue trace, the compact summary the bench prints last, and the local pass's
algorithmic bytes and flops per band."""
from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("_bench_logic", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_settle_time_is_the_first_time_after_which_every_value_stays_within_tolerance(bench):
    ref = np.array([1.0, 2.0])
    t = np.array([0.1, 0.2, 0.3, 0.4, 0.5])
    e = np.array([[1.1, 2.0], [1.0 + 5e-9, 2.0], [1.0 + 2e-8, 2.0], [1.0, 2.0 + 1e-9], [1.0, 2.0]])
    # within 1e-8 at 0.2, out again at 0.3, within from 0.4 on: the settle time is 0.4
    assert bench.settle_time((t, None, e), ref) == pytest.approx(0.4)
    # a trace whose last iterate is outside the tolerance never settles
    assert bench.settle_time((t, None, e[[0, 1, 3, 4, 2]]), ref) is None
    # an empty trace has no settle time
    assert bench.settle_time((np.array([]), None, np.zeros((0, 2))), ref) is None
    # every iterate within the tolerance: the first one
    assert bench.settle_time((t, None, np.tile(ref, (5, 1))), ref) == pytest.approx(0.1)


def test_summary_reports_medians_ratios_and_worst_cell(bench):
    line = {
        "value": 59770.4, "e2e": {"value": 37490.1},
        "roofline": {"frac": 0.3211, "mixed": {"frac": 0.2471}},
        "mixed": {"value": 96050.0},
        "nonlocal": {"ms_fp64": 1.162, "ms_fp64_cublas": 1.589},
        "davidson_216": {"fp64_s": 3.11, "mixed_s": 1.25, "speedup": 2.488, "fp64_to_1e-8_s": 3.0,
                         "mixed_to_1e-8_s": 1.05, "speedup_to_1e-8": 2.857, "fp64_err_ry": 7.6e-10,
                         "mixed_err_ry": 4.9e-10, "err_vs": "oracle fixture", "fp64_int8_s": 2.74,
                         "fp64_int8_to_1e-8_s": 2.65, "speedup_to_1e-8_vs_fp64_int8": 2.52},
        "serving": {"at_capacity": {"throughput_rps": 16.3, "p50_ms": 70.0, "p99_ms": 140.0, "n_shed": 3,
                                    "per_cell": {"a": {"p50_ms": 10.0, "p99_ms": 15.0},
                                                 "b": {"p50_ms": 100.0, "p99_ms": 250.0}}}},
        "cpu_baseline": {"value": 85.0, "cores": 16},
    }
    s = bench.summary_of(line)
    assert s["davidson_216"]["speedup_to_1e-8"] == pytest.approx(2.86, abs=0.01)
    assert s["davidson_216"]["speedup_to_1e-8_vs_fp64_int8"] == pytest.approx(2.52, abs=0.01)
    assert s["davidson_216"]["err_vs"] == "oracle fixture"
    sv = s["serving"]["at_capacity"]
    assert sv["p99_over_p50"] == pytest.approx(2.0) and sv["shed"] == 3
    assert sv["worst_cell_p99_over_p50"] == pytest.approx(2.5)
    assert s["nonlocal_ms_int8_vs_cublas"] == [pytest.approx(1.16, abs=0.01), pytest.approx(1.59, abs=0.01)]
    assert s["cpu_cores"] == 16


def test_local_pass_model_of_the_headline_cell(bench, pkg):
    """B_alg = b (3 npw + 4 S) + r N per band (S = sticks x nz, N = the grid) on the 64-atom cell: 19.9 MB per
    band in FP64, half of the complex bytes in FP32; the flops count two pruned 3-D transforms."""
    spec = pkg.synth.config(1)
    basis = pkg.pwdft.PWBasisK(spec.a, pkg.synth.make_cell(spec).latvec, spec.ecut, np.zeros((1, 3)), grid=spec.grid)
    b64 = bench.local_bytes_per_band(basis, 16, 8)
    b32 = bench.local_bytes_per_band(basis, 8, 4)
    assert b64 == pytest.approx(19.9e6, rel=0.01)
    assert b32 == pytest.approx(b64 / 2, rel=1e-12)
    assert bench.local_flops_per_band(basis) > 0
