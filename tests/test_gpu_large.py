"""1024^3: the largest grid the library supports on one GPU.  The forward
transform of a separable product of Fourier modes has exactly known
coefficients, and the inverse returns the field."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_transform_1024_separable_modes():
    from hit3d_b200 import Context, Params
    n = 1024
    c = Context(Params(nx=n))
    x = 2 * np.pi * np.arange(n) / n
    fx, gy, hz = np.cos(3 * x + 0.3), np.sin(5 * x), np.cos(7 * x)
    a = np.zeros((n, n, n + 2))                 # physical [z][y][x]
    a[..., :n] = hz[:, None, None] * gy[None, :, None] * fx[None, None, :]
    F = c.xfft3d(1, a)                          # Fourier [ky][kz][kx re/im]
    h = n / 2.0
    expect = {}
    for ky, gk in ((5, -1j * h), (n - 5, 1j * h)):
        for kz in (7, n - 7):
            expect[(ky, kz)] = h * np.exp(0.3j) * gk * h
    scale = abs(next(iter(expect.values())))
    for (ky, kz), v in expect.items():
        got = F[ky, kz, 6] + 1j * F[ky, kz, 7]
        assert abs(got - v) < 1e-12 * scale, (ky, kz, got, v)
        F[ky, kz, 6:8] = 0.0
    assert np.abs(F).max() < 1e-12 * scale
    for (ky, kz), v in expect.items():
        F[ky, kz, 6], F[ky, kz, 7] = v.real, v.imag
    back = c.xfft3d(-1, F)
    assert np.abs(back[..., :n] - a[..., :n]).max() < 1e-12
    c.close()
