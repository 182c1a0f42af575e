"""Precision form: FP32 nonlinear-term transforms with an FP64 state,
integrator and reductions, against the FP64 path from the same state, per
statistic (E(k), energy, dissipation, velocity-derivative skewness)."""
import numpy as np
import pytest

from _cases import RN1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,dealias", [(128, 0), (64, 1)])
def test_fp32_transforms_track_fp64(n, dealias):
    from hit3d_b200 import Context, Params
    ctx = []
    for precision in (0, 1):
        c = Context(Params(nx=n, dealias=dealias, flow_type=1, kfmax=2, nu=1.0 / 1500.0, dt=0.002,
                           precision=precision))
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        ctx.append(c)
    for _ in range(4):
        for c in ctx:
            c.step(25)
        (e64, s64), (e32, s32) = ctx[0].stats(), ctx[1].stats()
        # shells holding more than 1e-8 of the peak: the nearly empty top shells of
        # this initial spectrum (1e-12 of the peak at 128^3) sit at the FP32
        # round-off floor, where a relative error says nothing
        mask = e64 > 1e-8 * e64.max()
        assert np.max(np.abs(e32[mask] - e64[mask]) / e64[mask]) < 1e-4
        assert abs(s32["energy"] - s64["energy"]) < 1e-8 * s64["energy"]
        assert abs(s32["eps_v"] - s64["eps_v"]) < 1e-7 * s64["eps_v"]
        assert abs(s32["skewness"] - s64["skewness"]) < 1e-6
    # the state stays FP64: the two runs differ, but only at FP32 round-off level
    f64, f32 = ctx[0].download_fields(), ctx[1].download_fields()
    assert 0 < np.abs(f32 - f64).max() < 1e-5 * np.abs(f64).max()
