"""Every launch-shape variant of the fused x pass (the tuner's search space)
gives the same step: velocity, scalar and Smagorinsky operators, FP64 and FP32."""
import numpy as np
import pytest

from _cases import RN1, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32, 48, 64, 128])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("case", ["scalars", "les"])
def test_variants_agree(n, precision, case):
    from hit3d_b200 import Context, Params
    kw = dict(nx=n, flow_type=1, kfmax=2, nu=1.0 / 800.0, dt=0.002, precision=precision)
    if case == "scalars":
        kw.update(n_scalars=1, sc=[0.7], scalar_type=[0])
    else:
        kw.update(les_model=1)
    outs = []
    from hit3d_b200.gpu import N_VARIANTS
    for v in range(N_VARIANTS):
        c = Context(Params(**kw))
        c.set_variant(v)
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        c.step(3)
        outs.append(c.download_fields())
        c.close()
    tol = 1e-13 if precision == 0 else 1e-6
    for v in range(1, N_VARIANTS):
        assert relerr(outs[v], outs[0]) < tol, (v, relerr(outs[v], outs[0]))


@pytest.mark.parametrize("precision", [0, 1])
def test_one_pair_variants_at_512(precision):
    """At L = 512 variants 11, 12 and 13 take one row pair per CTA (the stage
    and split loops without index division; 13 with bulk-copy staging and the
    split in registers); they agree with variant 8 (two pairs per CTA) over two
    forced steps."""
    from hit3d_b200 import Context, Params
    kw = dict(nx=512, flow_type=1, kfmax=2, nu=1.0 / 3000.0, dt=2e-4, precision=precision)
    outs = {}
    for v in (8, 11, 12, 13, 14):
        c = Context(Params(**kw))
        c.set_variant(v)
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        c.step(2)
        outs[v] = c.download_fields()
        c.close()
    tol = 1e-13 if precision == 0 else 1e-6
    for v in (11, 12, 13, 14):
        assert relerr(outs[v], outs[8]) < tol, (v, relerr(outs[v], outs[8]))


def test_tuner_picks_a_valid_variant():
    from hit3d_b200 import Context, Params
    c = Context(Params(nx=64, flow_type=1, kfmax=2, nu=1.0 / 800.0, dt=0.002))
    from hit3d_b200.gpu import N_VARIANTS
    v, ms = c.autotune()
    assert 0 <= v < N_VARIANTS and len(ms) == N_VARIANTS and all(x > 0 for x in ms)
    assert ms[v] == min(ms)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n", [32, 48, 64, 128, 256, 512])
def test_column_tiles_agree(n, precision):
    """Every column-tile shape of the strided passes, the pipelined one (3)
    included, runs the same arithmetic per column: bit-identical steps."""
    from hit3d_b200 import Context, Params
    kw = dict(nx=n, flow_type=1, kfmax=2, nu=1.0 / 1000.0, dt=2e-4 * 512 / n, precision=precision)
    outs = {}
    tiles = (0, 1, 2, 3) if n <= 512 else (0, 3)
    for t in tiles:
        c = Context(Params(**kw))
        c.set_variant(12)
        c.set_column_tile(t)
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        c.step(2)
        outs[t] = c.download_fields()
        c.close()
    for t in tiles[1:]:
        assert np.array_equal(outs[t], outs[0]), t
