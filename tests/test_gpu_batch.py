"""Batched form: runs advanced together through one recorded CUDA graph give
the same fields as the same runs stepped one by one; subgrid-stress training
data agree with the oracle.

Runs of one size class step through batched launches (one launch per pass over
all the class's runs) with the fused x pass of variant 13; stepped one by one
with that variant they give bit-identical fields, and with any other variant
fields equal to rounding."""
import numpy as np
import pytest

from _cases import relerr

pytestmark = pytest.mark.gpu


def test_batch_graph_matches_independent_runs():
    from hit3d_b200 import Context, Params
    from hit3d_b200.batch import Batch, run_seed
    sizes = [32, 48, 64, 32]
    res = [1.0 / 300, 1.0 / 500, 1.0 / 700, 1.0 / 250]
    ps = [Params(nx=n, flow_type=1, kfmax=2, nu=nu, dt=0.004) for n, nu in zip(sizes, res)]
    b = Batch(ps)
    b.init()
    ref, ref_any = [], []
    for r, p in enumerate(ps):
        for variant, out in ((13, ref), (4, ref_any)):
            c = Context(p)
            c.set_variant(variant)
            c.init_velocity(run_seed(r), 2, 4.0, 2.0)
            c.dealias_all()
            c.step(12)
            out.append(c.download_fields())
            c.close()
    b.step(12, graph_steps=5)
    assert b.graph_launches == 2  # 1 eager Euler step, 2 x 5 in the graph, 1 eager
    for r in range(len(ps)):
        f = b.contexts[r].download_fields()
        assert np.array_equal(f, ref[r]), r
        assert relerr(f, ref_any[r]) < 1e-13, r
    b.close()


def test_batch_classes_of_uneven_sizes_with_lone_runs():
    """Classes of 3 x 32^3 (FP64), 2 x 48^3 (FP32) and lone runs that cannot join
    a class (phase shift, a passive scalar) in one batch: every run equals the
    same run stepped on its own."""
    from hit3d_b200 import Context, Params
    from hit3d_b200.batch import Batch, run_seed
    ps = [Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / (300 + 50 * r), dt=0.004) for r in range(3)]
    ps += [Params(nx=48, flow_type=1, kfmax=2, nu=1.0 / (400 + 50 * r), dt=0.003, precision=1) for r in range(2)]
    ps += [Params(nx=32, dealias=1, flow_type=1, kfmax=2, nu=1.0 / 300, dt=0.004),
           Params(nx=32, flow_type=0, nu=1.0 / 300, dt=0.004, n_scalars=1, sc=[0.7], scalar_type=[0])]
    b = Batch(ps)
    b.init()
    b.step(9, graph_steps=4)
    for r, p in enumerate(ps):
        c = Context(p)
        if r < 5:  # class runs use variant 13; lone runs keep their own (the default)
            c.set_variant(13)
        c.init_velocity(run_seed(r), 2, 4.0, 2.0)
        c.dealias_all()
        c.step(9)
        assert np.array_equal(b.contexts[r].download_fields(), c.download_fields()), r
        c.close()
    b.close()


def test_sgs_fields_match_oracle():
    from _cases import make_pair
    n = 32
    o, g = make_pair(n, dealias=0, flow_type=1, nu=1.0 / 200.0)
    o.step(2)
    g.step(2)
    delta = 4 * 2 * np.pi / n
    out = g.sgs_fields(4, delta)
    # the same quantities from the oracle's fields, in numpy
    G = o.filter_g(4, delta)
    Gc = G[..., 0::2] + 1j * G[..., 1::2]
    def inv(spec_c):
        a = np.zeros((n, n, n + 2))
        a[..., 0::2], a[..., 1::2] = spec_c.real, spec_c.imag
        o.fft3d(-1, a)
        return a[..., :n]
    def fwd(phys):
        a = np.zeros((n, n, n + 2))
        a[..., :n] = phys
        o.fft3d(1, a)
        return a[..., 0::2] + 1j * a[..., 1::2]
    U = [o.fields[c][..., 0::2] + 1j * o.fields[c][..., 1::2] for c in range(3)]
    u = [inv(U[c]) for c in range(3)]
    ub = [inv(Gc * U[c]) for c in range(3)]
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    tau = [inv(Gc * fwd(u[i] * u[j])) - ub[i] * ub[j] for i, j in pairs]
    # signed wavenumbers (+N/2 kept positive); oracle spectral arrays are [ky][kz][kx]
    ks = np.fft.fftfreq(n, 1.0 / n)
    ks[n // 2] = n // 2
    kx = np.arange(n // 2 + 1)
    Kd = [kx[None, None, :] * np.ones((n, n, 1)),      # d/dx
          ks[:, None, None] * np.ones((1, n, 1)),      # d/dy: ky on axis 0
          ks[None, :, None] * np.ones((n, 1, 1))]      # d/dz: kz on axis 1
    A = [inv(1j * Kd[j] * Gc * U[i]) for i in range(3) for j in range(3)]
    ref = ub + tau + A
    for q in range(18):
        assert relerr(out[q], ref[q]) < 2e-6, q


def test_batch_rerecords_graph_after_dt_change():
    """dt is baked into the recorded graph; changing it on a run's context between
    calls must take effect (the graph is re-recorded)."""
    from hit3d_b200 import Context, Params
    from hit3d_b200.batch import Batch, run_seed
    ps = [Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / 300, dt=0.004) for _ in range(2)]
    b = Batch(ps)
    b.init()
    b.step(6, graph_steps=5)
    for c in b.contexts:
        c.set_dt(0.002)
    b.step(10, graph_steps=5)
    assert b.graph_launches == 3
    for r, p in enumerate(ps):
        c = Context(Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / 300, dt=0.004))
        c.set_variant(13)
        c.init_velocity(run_seed(r), 2, 4.0, 2.0)
        c.dealias_all()
        c.step(6)
        c.set_dt(0.002)
        c.step(10)
        assert np.array_equal(b.contexts[r].download_fields(), c.download_fields())
        c.close()
    b.close()


def test_batch_refuses_a_learned_closure_run_without_weights():
    from hit3d_b200 import Hit3dError, Params
    from hit3d_b200.batch import Batch
    b = Batch([Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / 300, dt=0.004),
               Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / 300, dt=0.004, les_model=20)])
    b.init()
    with pytest.raises(Hit3dError, match="weights"):
        b.step(3, graph_steps=2)
    b.close()


def test_batch_autotune_picks_shapes_and_keeps_results():
    """The per-class tuner picks a staged x-pass variant (8-14) and a column
    tile (0-3) per size class without changing the state; afterwards every run
    equals the same run stepped on its own with that variant (the column tile
    does not change any run's arithmetic)."""
    from hit3d_b200 import Context, Params
    from hit3d_b200.batch import Batch, run_seed
    ps = [Params(nx=32, flow_type=1, kfmax=2, nu=1.0 / (300 + 100 * r), dt=0.004) for r in range(2)]
    ps.append(Params(nx=64, flow_type=1, kfmax=2, nu=1.0 / 600, dt=0.003))
    b = Batch(ps)
    b.init()
    f0 = [c.download_fields() for c in b.contexts]
    picks = b.autotune()
    assert b.nclasses == 2 and len(picks) == 2
    for v, tile, ms_v, ms_t in picks:
        assert 8 <= v <= 14 and 0 <= tile <= 3
        assert all(x > 0 for x in ms_v) and all(x > 0 for x in ms_t)
    for r, c in enumerate(b.contexts):
        assert np.array_equal(c.download_fields(), f0[r])
    b.step(7, graph_steps=3)
    cls = [0, 0, 1]
    for r, p in enumerate(ps):
        c = Context(p)
        c.set_variant(picks[cls[r]][0])
        c.init_velocity(run_seed(r), 2, 4.0, 2.0)
        c.dealias_all()
        c.step(7)
        assert np.array_equal(b.contexts[r].download_fields(), c.download_fields()), r
        c.close()
    b.close()
