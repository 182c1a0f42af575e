"""Learned subgrid closure on the GPU: the training kernels' loss and gradients and
the inference kernel against the numpy oracle, deterministic training, the LES
step with the network, and what the trained network gains over Smagorinsky."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

DELTA = 2 * 2 * np.pi / 32


def _mlp(w=None, seed=0):
    from hit3d_b200 import Mlp
    m = Mlp(seed=seed)
    if w is not None:
        m.params = np.asarray(w, dtype=np.float32)
    return m


def test_loss_and_gradient_match_oracle():
    A, tau = mo.synthetic_data(5000, seed=4)
    w = mo.bf16_round(mo.init_params(3)).astype(np.float64)
    m = _mlp(w)
    m.set_data(A, tau, DELTA)
    td = mo.deviatoric(tau)
    n1, n2 = m.norms()
    o1, o2 = mo.norms(A, td)
    assert abs(n1 - o1) <= 1e-6 * o1 and abs(n2 - o2) <= 1e-6 * o2
    idx = np.random.default_rng(1).choice(5000, 3000).astype(np.int32)
    for lam in (0.0, 0.8):
        loss, g = m.loss_grad(idx, lam)
        ol, og = mo.loss_grad(w, A[:, idx], td[:, idx], DELTA, float(np.float32(n1)), float(np.float32(n2)), lam)
        assert abs(loss - ol) <= 2e-5 * ol, (lam, loss, ol)
        assert np.abs(g - og).max() <= 2e-4 * np.abs(og).max(), (lam, np.abs(g - og).max(), np.abs(og).max())
    m.close()


def test_bf16_weights_are_the_rounded_parameters():
    w = mo.init_params(5).astype(np.float32)
    m = _mlp(w)
    assert np.array_equal(m.params, w)
    assert np.array_equal(m.bf16(), mo.bf16_bits(w))
    m.close()


@pytest.mark.parametrize("clip", [False, True])
def test_predict_matches_oracle(clip):
    A, _ = mo.synthetic_data(4000, seed=6)
    w = mo.bf16_round(mo.init_params(8)).astype(np.float64)
    m = _mlp(w)
    got = m.predict(A, DELTA, clip=clip)
    ref = mo.predict(w, A, DELTA, clip=clip)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    m.close()


def test_tensor_core_predict_matches_oracle():
    """Hidden layers on the tensor cores (bf16 activations, fp32 accumulation in
    TMEM), GELUs with the hardware tanh approximation: against the oracle with the
    same bf16 rounding of the activations and the exact tanh, on a ragged point
    count that spans several tiles per CTA.

    Bound: tanh.approx.f32 differs from tanh by up to about 2^-11, which moves an
    activation by far less than one bf16 step (2^-8 relative) but decides some
    bf16 roundings differently; a point's stress then moves by a fraction of a
    bf16 step.  Stated: 99.9 % of points within 2e-4 of the largest stress, every
    point within 2e-3 (measured on B200: median 1.6e-8, 99.9 % 5.1e-5, max
    3.8e-4)."""
    np_ = 300001
    A, _ = mo.synthetic_data(np_, seed=13)
    w = mo.bf16_round(mo.init_params(21)).astype(np.float64)
    m = _mlp(w)
    got = m.predict(A, DELTA, clip=False, kernel=1)
    ref = mo.predict(w, A, DELTA, act_bf16=True)
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max(axis=0) / scale
    print(f"tensor-core closure vs oracle: median {np.median(err):.2e}, 99.9 % {np.quantile(err, 0.999):.2e}, "
          f"max {err.max():.2e}")
    assert np.quantile(err, 0.999) < 2e-4 and err.max() < 2e-3, (np.quantile(err, 0.999), err.max())
    # and the fp32-activation kernel agrees to bf16 accuracy
    exact = m.predict(A, DELTA, clip=False, kernel=0)
    assert np.abs(exact - got).max() < 2e-2 * scale
    got_clip = m.predict(A, DELTA, clip=True, kernel=1)
    ref_clip = mo.predict(w, A, DELTA, clip=True, act_bf16=True)
    agree = np.all(np.abs(got_clip - ref_clip) <= 2e-3 * scale, axis=0)
    assert agree.mean() > 0.999
    m.close()


def test_training_reduces_loss_and_is_deterministic():
    A, tau = mo.synthetic_data(50000, seed=9)
    runs = []
    for _ in range(2):
        m = _mlp(seed=12)
        m.set_data(A, tau, DELTA)
        losses = m.train(300, batch=4096, lr=3e-3, lam=0.5, seed=21)
        runs.append((losses, m.params))
        m.close()
    losses = runs[0][0]
    assert np.all(np.isfinite(losses))
    assert losses[-30:].mean() < 0.25 * losses[:10].mean()
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


@pytest.mark.parametrize("kernel", [0, 1])
def test_les_step_with_smagorinsky_weights_matches_smagorinsky(kernel):
    """With g = (g1, 0, 0, 0, 0) the network is the Smagorinsky model; the LES step
    through the network must match les_model 1 with the same coefficient."""
    from _cases import RN1, relerr
    from hit3d_b200 import Context, Params
    n = 32
    dx = 2 * np.pi / n
    g1 = float(mo.bf16_round(np.float32(-2 * 0.18 ** 2 * dx * dx / DELTA ** 2)).item())
    cs = np.sqrt(-g1 * DELTA ** 2 / (2 * dx * dx))
    common = dict(nx=n, flow_type=1, kfmax=2, nu=1.0 / 2000.0, dt=0.005)
    a = Context(Params(les_model=1, c_smag=cs, **common))
    b = Context(Params(les_model=20, **common))
    w = mo.smagorinsky_params(0.0, dx, DELTA)
    w[-5] = g1
    b.les_set_mlp(mo.bf16_bits(w), DELTA, clip=True, kernel=kernel)
    for c in (a, b):
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        c.step(10)
    fa, fb = a.download_fields(), b.download_fields()
    assert relerr(fb, fa) < 1e-6
    # the model matters at this Reynolds number: no model gives a different field
    c = Context(Params(les_model=0, **common))
    c.init_velocity(RN1, 2, 4.0, 2.0)
    c.dealias_all()
    c.step(10)
    assert relerr(c.download_fields(), fa) > 1e-4


def test_learned_les_needs_weights():
    from hit3d_b200 import Context, Hit3dError, Params
    c = Context(Params(nx=32, les_model=20))
    with pytest.raises(Hit3dError, match="weights"):
        c.step(1)
    d = Context(Params(nx=32, les_model=1))
    with pytest.raises(Hit3dError, match="les_model 20"):
        d.les_set_mlp(np.zeros(mo.NPARAM, np.uint16), DELTA)


def test_learned_closure_beats_smagorinsky_a_priori():
    """Trained on box-filtered 64^3 DNS from the batched form, evaluated on a later,
    held-out state: the network's stress error is below the best-fit Smagorinsky
    model's and the reference's Cs = 0.18 model's."""
    from hit3d_b200.les import (LesExperiment, best_smagorinsky_g1, generate_training_data, sgs_samples,
                                smagorinsky_stress, stress_error, train_closure)
    from hit3d_b200 import Context
    ex = LesExperiment(n_dns=64, n_les=32, re=500.0, dt_dns=0.004, nruns=2, spinup=1.5, collect=0.5, nsnap=2,
                       stride=1, train_steps=800, batch=16384, lam=0.5)
    A, tau, f0, r0 = generate_training_data(ex, log=lambda *a: None)
    m, losses, _ = train_closure(ex, A, tau, log=lambda *a: None)
    g1 = best_smagorinsky_g1(A, tau, ex.delta)
    dns = Context(ex.dns_params())
    dns.upload_fields(f0)
    dns.upload_rhs_old(r0)
    dns.fov = 0
    dns.step(int(0.5 / ex.dt_dns))
    Ah, th = sgs_samples(dns, ex.delta, 1)
    e_net = stress_error(m.predict(Ah, ex.delta, clip=False), th)
    e_best = stress_error(smagorinsky_stress(Ah, 1.0, 1.0) * (g1 * ex.delta ** 2 / -2.0), th)
    e_ref = stress_error(smagorinsky_stress(Ah, 0.18, 2 * np.pi / ex.n_les), th)
    assert e_net < 0.9 * e_best and e_net < e_ref, (e_net, e_best, e_ref)
