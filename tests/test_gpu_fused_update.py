"""The z forward pass of the velocity products fused with the update and the
next step's z inverse (k_zfwd_update) against the separate z passes +
k_update_vel_23: the same state after several steps of one call (every step
but the first takes its z inverse from the previous step's fused pass),
pruned and unpruned, FP64 and FP32 transforms, forced and decaying, with
passive scalars, up to the 512^3 workload."""
import numpy as np
import pytest

from _cases import RN1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,precision,extra,prune", [
    (32, 0, {}, True),
    (64, 0, dict(flow_type=0), False),
    (64, 1, {}, True),
    (48, 0, dict(n_scalars=2, sc=[0.7, 1.0], scalar_type=[0, 1]), True),
    (128, 0, {}, True),
    (128, 1, {}, False),
    (256, 0, {}, True),
    (512, 0, dict(nu=1.0 / 3000.0, dt=2e-4), True),
    (512, 1, dict(nu=1.0 / 3000.0, dt=2e-4), True),
])
def test_fused_update_matches_separate_passes(n, precision, extra, prune):
    from hit3d_b200 import Context, Params
    kw = dict(nx=n, flow_type=1, kfmax=2, nu=1.0 / 800.0, dt=0.002, precision=precision)
    kw.update(extra)
    out = []
    for fused in (True, False):
        c = Context(Params(**kw))
        c.set_update_fusion(fused)
        c.set_pruning(prune)
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        c.step(4)
        out.append((c.download_fields(), c.download_rhs_old()))
        c.close()
    (f1, r1), (f0, r0) = out
    # the sums k.P are rounded in the same order on both paths
    for a, b in ((f1, f0), (r1, r0)):
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= 1e-14, err
