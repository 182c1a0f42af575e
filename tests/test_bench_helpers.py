"""Host-side helpers of bench.py that need no GPU: the FP32-form E(k) error per
energy band of shells and the stage byte model."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_ek_error_bands():
    # peak shell 1.0; shells at 1e-1, 1e-3, 1e-5, 1e-7, 1e-9, 1e-11 of it
    e64 = np.array([1.0, 1e-1, 1e-3, 1e-5, 1e-7, 1e-9, 1e-11])
    rel = np.array([1e-9, 2e-9, 3e-8, 4e-7, 5e-6, 6e-5, 7e-4])
    e32 = e64 * (1.0 + rel)
    out = bench.ek_err_by_decade(e32, e64)
    assert list(out) == ["1e-2", "1e-4", "1e-6", "1e-8", "1e-10", "1e-12"]
    want = {"1e-2": 2e-9, "1e-4": 3e-8, "1e-6": 4e-7, "1e-8": 5e-6, "1e-10": 6e-5, "1e-12": 7e-4}
    for k, v in want.items():
        assert abs(out[k] - v) <= 1e-6 * v, (k, out[k], v)


def test_ek_error_bands_empty_band_is_none():
    e64 = np.array([1.0, 0.5])
    out = bench.ek_err_by_decade(e64.copy(), e64)
    assert out["1e-2"] == 0.0 and out["1e-4"] is None and out["1e-12"] is None


def test_stage_bytes_fp32_halves_the_work_fields():
    n = 512
    f64 = bench.stage_units(n, 0, True)
    f32 = bench.stage_units(n, 1, True)
    # the x pass and the y passes touch only work fields: half in the FP32 form
    for k in ("x_fused", "y_inverse", "y_forward", "z_forward"):
        assert abs(f32[k] - 0.5 * f64[k]) <= 1e-12 * f64[k]
    # the update reads and writes the FP64 state in both forms
    assert f32["update"] > 0.5 * f64["update"]
    assert abs(sum(f64.values()) - 27.9) < 0.1
