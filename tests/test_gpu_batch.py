"""Batched form: runs advanced together through one recorded CUDA graph give
the same fields as the same runs stepped one by one; subgrid-stress training
data agree with the oracle."""
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
    ref = []
    for r, p in enumerate(ps):
        c = Context(p)
        c.init_velocity(run_seed(r), 2, 4.0, 2.0)
        c.dealias_all()
        c.step(12)
        ref.append(c.download_fields())
        c.close()
    b.step(12, graph_steps=5)
    assert b.graph_launches == 2  # 1 eager Euler step, 2 x 5 in the graph, 1 eager
    for r in range(len(ps)):
        assert np.array_equal(b.contexts[r].download_fields(), ref[r])
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
