"""xFFT3d parity: the sm_100a transform passes against the oracle's FFT
(x_fftw.f90:852-1085 conventions: unnormalised forward, 1/N^3 inverse, Fourier
layout (kx, kz, ky), imaginary parts of kx = 0 and kx = N/2 ignored by c2r)."""
import numpy as np
import pytest

from _cases import relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32, 48, 64, 128])
def test_forward_matches_oracle(n, oracle_mod):
    from hit3d_b200 import Context, Params
    rng = np.random.default_rng(n)
    o = oracle_mod.Oracle(n)
    g = Context(Params(nx=n))
    a = np.zeros((n, n, n + 2))
    a[:, :, :n] = rng.standard_normal((n, n, n))
    ref = a.copy()
    o.fft3d(1, ref)
    out = g.xfft3d(1, a)
    assert relerr(out, ref) < 1e-13


@pytest.mark.parametrize("n", [32, 48, 64, 128])
def test_inverse_matches_oracle(n, oracle_mod):
    """Includes a non-Hermitian kx = 0 plane and Nyquist column: both sides must
    drop the imaginary parts the way FFTW's c2r does."""
    from hit3d_b200 import Context, Params
    rng = np.random.default_rng(100 + n)
    o = oracle_mod.Oracle(n)
    g = Context(Params(nx=n))
    a = rng.standard_normal((n, n, n + 2))
    ref = a.copy()
    o.fft3d(-1, ref)
    out = g.xfft3d(-1, a)
    assert relerr(out[:, :, :n], ref[:, :, :n]) < 1e-13


@pytest.mark.parametrize("n", [256, 512])
def test_round_trip_large(n):
    """Size-independent property at full sizes: inverse(forward(x)) == x."""
    from hit3d_b200 import Context, Params
    rng = np.random.default_rng(7)
    g = Context(Params(nx=n))
    a = np.zeros((n, n, n + 2))
    a[:, :, :n] = rng.standard_normal((n, n, n))
    f = g.xfft3d(1, a)
    b = g.xfft3d(-1, f)
    assert relerr(b[:, :, :n], a[:, :, :n]) < 1e-13
    # Parseval on the half spectrum: sum x^2 = (1/N^3) sum_k w_k |X_k|^2
    X = f[..., 0::2] + 1j * f[..., 1::2]
    w = np.full(n // 2 + 1, 2.0)
    w[0] = w[-1] = 1.0
    lhs = np.sum(a[:, :, :n] ** 2)
    rhs = np.sum(w * np.abs(X) ** 2) / n ** 3
    assert abs(lhs - rhs) / lhs < 1e-12
