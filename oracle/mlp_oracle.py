"""CPU oracle of the learned subgrid closure -- TEST INFRASTRUCTURE ONLY.

A float64 numpy restatement of the network, features, loss and gradients that
the CUDA kernels of the product implement (the closure has no counterpart in the
reference; its fallback, the Smagorinsky model, follows m_les.f90:1142-1215).
Only tests/ import this module, as the checker of the kernels.

Parity status: unpinned against the reference (no counterpart); pinned by a
finite-difference check of the analytic gradient (tests/test_mlp_oracle.py) and by
the Smagorinsky special case g = (-2 Cs^2, 0, 0, 0, 0).

Conventions (shared with the kernels):
  A     (9, P) velocity gradients, A[3i+j] = d u_i / d x_j
  tau   (6, P) symmetric stresses in the order 11 12 13 22 23 33
  x     (6, P) inputs: tr s^2, tr r^2, tr s^3, tr s r^2, tr s^2 r^2, Delta*32/(2 pi)
  T     (5, 6, P) basis s, sr - rs, s^2 - tr(s^2)/3 I, r^2 - tr(r^2)/3 I, r s^2 - s^2 r
  tau_pred = Delta^2 |S|^2 sum_n g_n T_n,  |S| = sqrt(2 S:S),  s = S/|S|,  r = R/|S|
  params: W1[64][6] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[5][64] b4[5]
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 6, 64, 5
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
          ("W4", (NOUT, NH)), ("b4", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
FROB = np.array([1.0, 2.0, 2.0, 1.0, 2.0, 1.0])


def bf16_round(w) -> np.ndarray:
    """fp32 values rounded to the nearest bf16 (ties to even), returned as fp32."""
    b = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b >> 16) & 1) + 0x7FFF
    return (((b + r) & 0xFFFF0000).astype(np.uint32)).view(np.float32)


def bf16_bits(w) -> np.ndarray:
    return (bf16_round(w).view(np.uint32) >> 16).astype(np.uint16)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    out, o = {}, 0
    for name, s in SHAPES:
        k = int(np.prod(s))
        out[name] = w[o:o + k].reshape(s)
        o += k
    return out


def pack(d) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


GELU_A, GELU_B = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """GELU in its tanh form (Hendrycks and Gimpel 2016), the network's activation."""
    return 0.5 * z * (1.0 + np.tanh(GELU_A * (z + GELU_B * z ** 3)))


def gelu_d(z):
    t = np.tanh(GELU_A * (z + GELU_B * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_A * (1.0 + 3.0 * GELU_B * z * z)


def features(A, delta):
    """x (6,P), T (5,6,P), sbar (6,P), pref (P) from gradients A (9,P)."""
    A = np.asarray(A, dtype=np.float64).reshape(3, 3, -1)
    S = 0.5 * (A + A.transpose(1, 0, 2))
    R = 0.5 * (A - A.transpose(1, 0, 2))
    sbar = np.stack([S[i, j] for i, j in PAIRS])
    smag = np.sqrt(2.0 * np.einsum("ijp,ijp->p", S, S)) + 1e-30
    s = S / smag
    r = R / smag
    mm = lambda a, b: np.einsum("ikp,kjp->ijp", a, b)
    tr = lambda a: a[0, 0] + a[1, 1] + a[2, 2]
    s2, r2 = mm(s, s), mm(r, r)
    x = np.stack([tr(s2), tr(r2), tr(mm(s2, s)), tr(mm(s, r2)), tr(mm(s2, r2)),
                  np.full(smag.shape, delta * 32.0 / (2.0 * np.pi))])
    eye = np.eye(3)[:, :, None]
    basis = [s, mm(s, r) - mm(r, s), s2 - eye * tr(s2) / 3.0, r2 - eye * tr(r2) / 3.0, mm(r, s2) - mm(s2, r)]
    T = np.stack([np.stack([b[i, j] for i, j in PAIRS]) for b in basis])
    pref = delta * delta * smag * smag
    return x, T, sbar, pref


def _bf16_act(a):
    return bf16_round(a.astype(np.float32)).astype(np.float64)


def forward(w, x, act_bf16=False):
    """act_bf16: every layer's input rounded to bf16 (the features and the three
    hidden activations), as the tensor-core inference kernel feeds them to the
    MMAs of its four layers."""
    p = unpack(w)
    if act_bf16:
        x = _bf16_act(x)
    z1 = p["W1"] @ x + p["b1"][:, None]
    a1 = gelu(z1)
    if act_bf16:
        a1 = _bf16_act(a1)
    z2 = p["W2"] @ a1 + p["b2"][:, None]
    a2 = gelu(z2)
    if act_bf16:
        a2 = _bf16_act(a2)
    z3 = p["W3"] @ a2 + p["b3"][:, None]
    a3 = gelu(z3)
    if act_bf16:
        a3 = _bf16_act(a3)
    g = p["W4"] @ a3 + p["b4"][:, None]
    return g, (x, z1, a1, z2, a2, z3, a3)


def predict(w, A, delta, clip=False, act_bf16=False):
    x, T, sbar, pref = features(A, delta)
    g, _ = forward(w, x, act_bf16)
    tau = pref * np.einsum("np,ncp->cp", g, T)
    if clip:
        diss = -np.einsum("c,cp,cp->p", FROB, tau, sbar)
        tau = np.where(diss < 0, 0.0, tau)
    return tau


def deviatoric(tau):
    """Deviatoric part in the precision the library stores it (fp32)."""
    tau = np.asarray(tau, dtype=np.float64)
    tr = (tau[0] + tau[3] + tau[5]) / 3.0
    out = tau.copy()
    for c in (0, 3, 5):
        out[c] -= tr
    return out.astype(np.float32).astype(np.float64)


def norms(A, tau_dev):
    """(1/mean |tau|_F^2, 1/mean (tau:S)^2) over a data set."""
    A = np.asarray(A, dtype=np.float64).reshape(3, 3, -1)
    sbar = np.stack([0.5 * (A[i, j] + A[j, i]) for i, j in PAIRS])
    n2 = np.einsum("c,cp,cp->p", FROB, tau_dev, tau_dev)
    pi = -np.einsum("c,cp,cp->p", FROB, tau_dev, sbar)
    return 1.0 / n2.mean(), 1.0 / (pi * pi).mean()


def loss_grad(w, A, tau_dev, delta, inv_norm, inv_norm_p, lam):
    """Loss and gradient over all points of (A, tau_dev):
    L = inv_norm/P sum |tau_pred - tau|_F^2 + lam inv_norm_p/P sum (Pi_pred - Pi)^2."""
    x, T, sbar, pref = features(A, delta)
    g, (x, z1, a1, z2, a2, z3, a3) = forward(w, x)
    npt = x.shape[1]
    tp = pref * np.einsum("np,ncp->cp", g, T)
    e = tp - tau_dev
    ep = -np.einsum("c,cp,cp->p", FROB, tp, sbar) + np.einsum("c,cp,cp->p", FROB, tau_dev, sbar)
    loss = (inv_norm * np.einsum("c,cp,cp->", FROB, e, e) + lam * inv_norm_p * np.sum(ep * ep)) / npt
    a1n = np.einsum("c,cp,ncp->np", FROB, e, T)
    a2n = np.einsum("c,cp,ncp->np", FROB, sbar, T)
    d4 = (2.0 * inv_norm / npt) * pref * a1n + (-2.0 * lam * inv_norm_p / npt) * ep * pref * a2n
    p = unpack(w)
    d3 = (p["W4"].T @ d4) * gelu_d(z3)
    d2 = (p["W3"].T @ d3) * gelu_d(z2)
    d1 = (p["W2"].T @ d2) * gelu_d(z1)
    grad = {"W4": d4 @ a3.T, "b4": d4.sum(1), "W3": d3 @ a2.T, "b3": d3.sum(1), "W2": d2 @ a1.T, "b2": d2.sum(1),
            "W1": d1 @ x.T, "b1": d1.sum(1)}
    return float(loss), pack(grad)


def init_params(seed: int = 0) -> np.ndarray:
    """Random parameters for tests (not the library's initialisation)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, s in SHAPES:
        if name.startswith("W"):
            a = np.sqrt(6.0 / (s[0] + s[1])) * (0.1 if name == "W4" else 1.0)
            d[name] = rng.uniform(-a, a, s)
        else:
            d[name] = rng.uniform(-0.05, 0.05, s)
    return pack(d)


def smagorinsky_params(cs: float, dx: float, delta: float) -> np.ndarray:
    """Parameters whose prediction is the Smagorinsky stress -2 (Cs dx)^2 |S| S."""
    w = np.zeros(NPARAM)
    w[-NOUT] = -2.0 * cs * cs * dx * dx / (delta * delta)
    return w


def best_smagorinsky(A, tau_dev, delta):
    """Least-squares g1 of tau = g1 Delta^2 |S| S over a data set (in the Frobenius norm)."""
    x, T, sbar, pref = features(A, delta)
    m = pref * T[0]
    return float(np.einsum("c,cp,cp->", FROB, m, tau_dev) / np.einsum("c,cp,cp->", FROB, m, m))


def synthetic_data(P: int, seed: int = 0):
    """Random traceless gradients and stresses correlated with them (for gradient checks)."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((3, 3, P))
    tr = (A[0, 0] + A[1, 1] + A[2, 2]) / 3.0
    for i in range(3):
        A[i, i] -= tr
    S = 0.5 * (A + A.transpose(1, 0, 2))
    smag = np.sqrt(2.0 * np.einsum("ijp,ijp->p", S, S))
    tau = np.stack([-0.02 * smag * S[i, j] + 0.01 * rng.standard_normal(P) for i, j in PAIRS])
    return A.reshape(9, P).astype(np.float32), tau.astype(np.float32)
