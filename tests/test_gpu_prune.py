"""2/3-rule pruning of the step's transforms gives bit-identical fields and is
used only when the state is zero beyond N/3."""
import numpy as np
import pytest

from _cases import RN1

pytestmark = pytest.mark.gpu

CASES = [
    (32, 0, {}),
    (48, 0, dict(n_scalars=2, sc=[0.7, 1.0], scalar_type=[0, 0])),
    (64, 0, {}),
    (128, 0, {}),
    (64, 1, dict(n_scalars=1, sc=[0.7], scalar_type=[0])),
    (128, 1, {}),
    (32, 0, dict(les_model=1)),
    (32, 0, dict(les_model=20)),
    (64, 1, dict(les_model=20)),
]


def _run(n, precision, extra, prune, steps=5):
    from hit3d_b200 import Context, Params
    from oracle import mlp_oracle as mo
    c = Context(Params(nx=n, flow_type=1, kfmax=2, nu=1.0 / 800.0, dt=0.002, precision=precision, **extra))
    if extra.get("les_model") == 20:
        c.les_set_mlp(mo.bf16_bits(mo.bf16_round(mo.init_params(4) * 0.05)), 4 * np.pi / n, clip=True, kernel=1)
    c.set_pruning(prune)
    c.init_velocity(RN1, 2, 4.0, 2.0)
    c.dealias_all()
    assert c.pruned == prune
    cour = c.step(steps)
    out = c.download_fields(), c.download_rhs_old(), cour
    c.close()
    return out


@pytest.mark.parametrize("n,precision,extra", CASES)
def test_pruned_step_is_bit_identical(n, precision, extra):
    a = _run(n, precision, extra, True)
    b = _run(n, precision, extra, False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_state_with_energy_beyond_the_cutoff_is_not_pruned():
    from hit3d_b200 import Context, Params
    c = Context(Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / 800.0, dt=0.002))
    c.init_velocity(RN1, 2, 4.0, 2.0)
    c.dealias_all()
    assert c.pruned
    f = c.download_fields()
    f[0, 0, 0, 2 * 15] = 1e-3              # kx = 15 > N/3: energy beyond the cutoff
    c.upload_fields(f)
    assert not c.pruned
    c.dealias_all()
    assert c.pruned
    c.upload_fields(f)
    c.step(2)
    ref = Context(Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / 800.0, dt=0.002))
    ref.set_pruning(False)
    ref.upload_fields(f)
    ref.step(2)
    assert np.array_equal(c.download_fields(), ref.download_fields())
