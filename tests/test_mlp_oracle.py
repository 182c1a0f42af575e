"""CPU checks of the learned-closure oracle: the analytic gradient against finite
differences, the Smagorinsky special case, bf16 rounding."""
import numpy as np

from oracle import mlp_oracle as mo


def test_gradient_matches_finite_differences():
    A, tau = mo.synthetic_data(300, seed=3)
    td = mo.deviatoric(tau)
    n1, n2 = mo.norms(A, td)
    delta = 2 * np.pi / 32
    w = mo.init_params(7)
    for lam in (0.0, 0.7):
        loss, g = mo.loss_grad(w, A, td, delta, n1, n2, lam)
        rng = np.random.default_rng(11)
        coords = np.concatenate([rng.choice(mo.NPARAM, 60, replace=False), np.arange(mo.NPARAM - 5, mo.NPARAM)])
        h = 1e-6
        for q in coords:
            wp, wm = w.copy(), w.copy()
            wp[q] += h
            wm[q] -= h
            fd = (mo.loss_grad(wp, A, td, delta, n1, n2, lam)[0] - mo.loss_grad(wm, A, td, delta, n1, n2, lam)[0]) / (2 * h)
            assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g).max()), (lam, q, fd, g[q])


def test_smagorinsky_special_case():
    A, _ = mo.synthetic_data(100, seed=1)
    cs, dx, delta = 0.18, 2 * np.pi / 32, 2 * 2 * np.pi / 32
    tau = mo.predict(mo.smagorinsky_params(cs, dx, delta), A, delta)
    A3 = A.astype(np.float64).reshape(3, 3, -1)
    S = 0.5 * (A3 + A3.transpose(1, 0, 2))
    smag = np.sqrt(2 * np.einsum("ijp,ijp->p", S, S))
    ref = np.stack([-2 * (cs * dx) ** 2 * smag * S[i, j] for i, j in mo.PAIRS])
    assert np.abs(tau - ref).max() <= 1e-12 * np.abs(ref).max()
    # the Smagorinsky stress is purely dissipative, so clipping changes nothing
    assert np.array_equal(mo.predict(mo.smagorinsky_params(cs, dx, delta), A, delta, clip=True), tau)


def test_best_smagorinsky_recovers_coefficient():
    A, _ = mo.synthetic_data(500, seed=2)
    delta = 0.3
    w = mo.smagorinsky_params(0.15, 0.2, delta)
    tau = mo.predict(w, A, delta)
    assert abs(mo.best_smagorinsky(A, tau, delta) - w[-5]) <= 1e-12 * abs(w[-5])


def test_bf16_rounding():
    x = np.array([1.0, 1 + 2**-8, 1 + 3 * 2**-8, 1 + 2**-7, -2.5, 3.0e-3], dtype=np.float32)
    r = mo.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie to even
    assert r[2] == np.float32(1 + 2**-6)           # tie rounds up to even
    assert r[3] == np.float32(1 + 2**-7)           # representable
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) <= 2**-8 * 3.0e-3
    assert np.array_equal(mo.bf16_round(r), r)     # idempotent
