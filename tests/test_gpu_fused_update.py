"""The z forward pass of the velocity products fused with the update
(k_zfwd_update) against the separate z pass + k_update_vel_23: the same
state after several steps, pruned and unpruned, FP64 and FP32 transforms,
forced and decaying, with passive scalars."""
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
    for a, b in ((f1, f0), (r1, r0)):
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= 1e-14, err
