"""Pins of the FP64 CPU oracle, on the CPU.  The reference cannot be built here
and ships no golden vectors, so the oracle is checked against what can be
stated independently of it:

- the analytic RHS checks of the reference's own (uncalled) test routines,
  test_rhs_velocity (rhs_velocity.f90:430-553) and test_rhs_scalars
  (rhs_scalars.f90:504-594);
- numpy.fft for the 3-D real transform and the 1-D complex transform;
- a pure-Python integer restatement of RANDu (RANDu.f:12-52);
- the target spectra that init_velocity imposes (init_velocity.f90:150-237);
- the band forcing of force_velocity (m_force.f90:101-182) restated in numpy;
- exact properties: the 2/3-rule nonlinear term conserves energy, the pressure
  projection leaves a divergence-free field, and the les.gp means of the
  dynamic localization model for a uniform k_sgs (m_les.f90:876-892)."""
import math

import numpy as np
import pytest

import oracle
from _cases import RN1


def _grid(n):
    x = np.arange(n) * 2 * np.pi / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    return X, Y, Z


def _phys(n, f):
    """A physical field in the reference's array: [z][y][x] with two padding entries."""
    a = np.zeros((n, n, n + 2))
    a[..., :n] = f
    return a


def _wavenumbers(n):
    """akx per real entry (pairs), aky / akz per index (m_fields.f90 layout)."""
    akx = (np.arange(n + 2) // 2).astype(np.float64)
    k = np.arange(n, dtype=np.float64)
    aky = np.where(k <= n // 2, k, k - n)
    return akx, aky, aky.copy()


def _to_complex(f):
    """Reference Fourier layout [ky][kz][kx re/im] -> complex [ky][kz][kx]."""
    return f[..., 0::2] + 1j * f[..., 1::2]


def _shell32(k2):
    """nint(sqrt(real(k2, 4))): the single-precision shell index of the reference."""
    r = np.sqrt(np.asarray(k2, dtype=np.float32)).astype(np.float64)
    return np.floor(r + 0.5).astype(np.int64)


# --- transforms -----------------------------------------------------------------

@pytest.mark.parametrize("n", [16, 24, 40, 48])
def test_fft3d_matches_numpy(n):
    """xFFT3d(+1): unnormalised forward, e^{-i}, result in [ky][kz][kx re/im];
    xFFT3d(-1): the inverse with 1/N^3 (x_fftw.f90:850-1090)."""
    o = oracle.Oracle(n)
    rng = np.random.default_rng(n)
    f = rng.standard_normal((n, n, n))
    a = _phys(n, f)
    o.fft3d(1, a)
    want = np.fft.rfftn(f).transpose(1, 0, 2)
    got = _to_complex(a)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    o.fft3d(-1, a)
    assert np.abs(a[..., :n] - f).max() <= 1e-13 * np.abs(f).max()


@pytest.mark.parametrize("n", [8, 12, 20, 48, 96, 160])
def test_fft1d_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.abs(oracle.fft1d(x, -1) - np.fft.fft(x)).max() <= 1e-13 * n
    assert np.abs(oracle.fft1d(x, 1) - n * np.fft.ifft(x)).max() <= 1e-13 * n


# --- random numbers ---------------------------------------------------------------

def _randu_python(seed, count):
    """RANDu.f:12-52 in Python integers.  idum is recomputed from the caller's
    argument on every call; iv, iy and idum2 are saved between calls."""
    im1, im2, ia1, ia2, iq1, iq2, ir1, ir2, ntab = 2147483563, 2147483399, 40014, 40692, 53668, 52774, 12211, 3791, 32
    imm1 = im1 - 1
    ndiv = 1 + imm1 // ntab
    am, rnmx = 1.0 / im1, 1.0 - 1.2e-7
    st = {"idum2": 123456789, "iy": 0, "iv": [0] * ntab}

    def fdiv(a, b):                      # Fortran integer division truncates toward zero
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b >= 0) else -q

    def rnd(idum3):
        idum = int(math.floor(abs(idum3 / 987.0) + 0.5)) * (1 if idum3 >= 0 else -1)
        if idum <= 0:
            idum = max(-idum, 1)
            st["idum2"] = idum
            for j in range(ntab + 8, 0, -1):
                k = fdiv(idum, iq1)
                idum = ia1 * (idum - k * iq1) - k * ir1
                if idum < 0:
                    idum += im1
                if j <= ntab:
                    st["iv"][j - 1] = idum
        k = fdiv(idum, iq1)
        idum = ia1 * (idum - k * iq1) - k * ir1
        if idum < 0:
            idum += im1
        k = fdiv(st["idum2"], iq2)
        st["idum2"] = ia2 * (st["idum2"] - k * iq2) - k * ir2
        if st["idum2"] < 0:
            st["idum2"] += im2
        j = 1 + fdiv(st["iy"], ndiv)
        st["iy"] = st["iv"][j - 1] - st["idum2"]
        st["iv"][j - 1] = idum
        if st["iy"] < 1:
            st["iy"] += imm1
        return min(am * st["iy"], rnmx)

    rnd(-seed)
    return np.array([rnd(seed) for _ in range(count)])


@pytest.mark.parametrize("seed", [RN1, 93712139.0, 10765397.0, 987.0 * 5])
def test_randu_stream_is_exact(seed):
    got = oracle.randu_stream(seed, 3000)
    want = _randu_python(seed, 3000)
    assert np.array_equal(got, want)
    assert (got > 0).all() and (got < 1).all()


# --- initial spectrum -------------------------------------------------------------

@pytest.mark.parametrize("isp", [0, 1, 3])
def test_init_velocity_imposes_the_target_spectrum(isp):
    """init_velocity.f90:150-237: every shell 1..kmax carries the normalised
    target spectrum, binned as the reference bins it (real entries i < nx,
    kx = 0 halved, single-precision shell index)."""
    n, peak = 32, 4.0
    o = oracle.Oracle(n)
    o.init_velocity(RN1, isp_type=isp, peak_wavenum=peak)
    akx, aky, akz = _wavenumbers(n)
    k2 = akx[None, None, :] ** 2 + aky[:, None, None] ** 2 + akz[None, :, None] ** 2
    sh = _shell32(k2)[..., :n]
    w = np.where(akx[:n] == 0, 0.5, 1.0)[None, None, :]
    e = (o.fields[:3, ..., :n] ** 2).sum(axis=0) * w / float(n) ** 6
    kmax = o.kmax
    got = np.bincount(sh.ravel(), weights=e.ravel(), minlength=kmax + 2)[1:kmax + 1]
    k = np.arange(1, kmax + 1, dtype=np.float64)
    r = k / peak
    tgt = {0: k ** (-5.0 / 3.0), 1: r ** 3 / peak * np.exp(-3.0 * r),
           3: (2 * np.pi * r) ** 4 / (1 + (2 * np.pi * r) ** 2) ** 3}[isp]
    tgt = tgt / tgt.sum()
    assert np.abs(got - tgt).max() <= 1e-13
    # nothing outside shells 1..kmax, and the field is solenoidal
    full_sh = _shell32(k2)
    assert np.abs(o.fields[:3][:, (full_sh == 0) | (full_sh > kmax)]).max() == 0.0
    u = _to_complex(o.fields[:3])
    div = akx[0::2][None, None, :] * u[0] + aky[:, None, None] * u[1] + akz[None, :, None] * u[2]
    assert np.abs(div).max() <= 1e-12 * np.abs(u).max()


# --- right-hand sides -------------------------------------------------------------

@pytest.mark.parametrize("nu", [0.0, 0.01])
def test_rhs_velocity_analytic(nu):
    """test_rhs_velocity (rhs_velocity.f90:430-553): for u = (sin x, sin y, sin z)
    the RHS is -sin(x) (2 cos x + cos y + cos z + nu), and cyclically."""
    n = 16
    o = oracle.Oracle(n, nu=nu, flow_type=0)
    X, Y, Z = _grid(n)
    for m, f in enumerate((np.sin(X), np.sin(Y), np.sin(Z))):
        a = _phys(n, f)
        o.fft3d(1, a)
        o.fields[m] = a
    o.rhs()
    got = o.wrk[1:4].copy()
    for m in range(3):
        o.fft3d(-1, got[m])
    s = np.cos(X) + np.cos(Y) + np.cos(Z)
    want = [-np.sin(X) * (np.cos(X) + s + nu), -np.sin(Y) * (np.cos(Y) + s + nu),
            -np.sin(Z) * (np.cos(Z) + s + nu)]
    for m in range(3):
        assert np.abs(got[m][..., :n] - want[m]).max() <= 1e-13


def test_rhs_scalars_analytic():
    """test_rhs_scalars (rhs_scalars.f90:504-594): u = (sin x, sin 5y, sin 17z),
    phi = cos x, Sc = 1, nu = 0.5: RHS = -cos 2x - cos x (5 cos 5y + 17 cos 17z + nu).
    A scalar of initial type 1 carries no mean-gradient source."""
    n, nu = 54, 0.5
    o = oracle.Oracle(n, nu=nu, nscal=1, sc=(1.0,), scalar_type=(1,))
    o.set_flags(1, 1, 1)
    X, Y, Z = _grid(n)
    for m, f in enumerate((np.sin(X), np.sin(5 * Y), np.sin(17 * Z), np.cos(X))):
        a = _phys(n, f)
        o.fft3d(1, a)
        o.fields[m] = a
    o.rhs()
    r = o.wrk[4].copy()
    o.fft3d(-1, r)
    want = -np.cos(2 * X) - np.cos(X) * (5 * np.cos(5 * Y) + 17 * np.cos(17 * Z) + nu)
    assert np.abs(r[..., :n] - want).max() <= 1e-12


def test_two_thirds_nonlinear_term_conserves_energy():
    """For a solenoidal, 2/3-rule-truncated u the products are alias-free on the
    kept modes, so sum_k Re(u* . N) = 0 (N = -d(u_i u_j)/dx_j, nu = 0)."""
    n = 32
    o = oracle.Oracle(n, nu=0.0, flow_type=0)
    o.init_velocity(RN1, isp_type=1, peak_wavenum=4.0)
    o.dealias_all()
    o.rhs()
    akx, _, _ = _wavenumbers(n)
    w = np.where(akx == 0, 1.0, 2.0)[None, None, None, :]
    dot = (o.fields[:3] * o.wrk[1:4] * w).sum()
    scale = (np.abs(o.fields[:3]) * np.abs(o.wrk[1:4]) * w).sum()
    assert scale > 0 and abs(dot) <= 1e-13 * scale


def test_pressure_projection_is_divergence_free():
    """pressure.f90: u <- u - k (k.u)/k^2 leaves k.u = 0 and is idempotent."""
    n = 24
    o = oracle.Oracle(n)
    rng = np.random.default_rng(5)
    for m in range(3):
        a = _phys(n, rng.standard_normal((n, n, n)))
        o.fft3d(1, a)
        o.fields[m] = a
    o.pressure()
    akx, aky, akz = _wavenumbers(n)
    u = _to_complex(o.fields[:3])
    div = akx[0::2][None, None, :] * u[0] + aky[:, None, None] * u[1] + akz[None, :, None] * u[2]
    # the Nyquist planes carry modes whose +-N/2 ambiguity the projection does not resolve
    inner = (np.abs(aky) < n // 2)[:, None, None] & (np.abs(akz) < n // 2)[None, :, None] \
        & (akx[0::2] < n // 2)[None, None, :]
    assert np.abs(div[inner]).max() <= 1e-12 * np.abs(u).max()
    before = o.fields[:3].copy()
    o.pressure()
    assert np.abs(o.fields[:3] - before).max() <= 1e-13 * np.abs(before).max()


@pytest.mark.parametrize("kfmax", [2, 20])
def test_band_forcing_matches_numpy_restatement(kfmax):
    """force_velocity (m_force.f90:101-182): every real entry of shells 1..kfmax
    gains FAMP / E_band times itself, E_band binned as in the reference (any
    band the input file gives, m_parameters.f90:308)."""
    n, famp = 32, 0.5
    o0 = oracle.Oracle(n, flow_type=0, kfmax=kfmax, famp=famp)
    o1 = oracle.Oracle(n, flow_type=1, kfmax=kfmax, famp=famp)
    o0.init_velocity(RN1, isp_type=1, peak_wavenum=3.0)
    o0.dealias_all()
    o1.fields[:] = o0.fields
    o0.rhs()
    o1.rhs()
    akx, aky, akz = _wavenumbers(n)
    sh = _shell32(akx[None, None, :] ** 2 + aky[:, None, None] ** 2 + akz[None, :, None] ** 2)
    band = (sh > 0) & (sh <= kfmax)
    band[..., n:] = False
    w = np.where(akx == 0, 0.5, 1.0)[None, None, :]
    e_band = ((o0.fields[:3] ** 2).sum(axis=0) * w)[band].sum() / float(n) ** 6
    want = np.where(band[None], famp / e_band * o0.fields[:3], 0.0)
    got = o1.wrk[1:4] - o0.wrk[1:4]
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    assert o1.nforced() == int(band.sum())


def test_dlm_les_means_for_uniform_k_sgs():
    """les.gp of the dynamic localization model (m_les.f90:876-892) for k_sgs =
    0.1 everywhere: energy 0.1, dissipation 0.1^1.5 / Delta, B = 0 and production
    2 nu_t <S:S> with nu_t = 0.1 Delta sqrt(0.1) (Delta = dx)."""
    n = 32
    o = oracle.Oracle(n, les_model=2, flow_type=0, nu=1.0 / 2000.0)
    o.init_velocity(RN1, isp_type=1, peak_wavenum=4.0)
    o.dealias_all()
    o.fields[3] = 0.0
    o.fields[3, 0, 0, 0] = 0.1 * n ** 3
    o.rhs()
    st = o.les_stats()
    dx = 2 * np.pi / n
    u = _to_complex(o.fields[:3]).transpose(0, 2, 1, 3)            # [c][kz][ky][kx]
    kz = np.fft.fftfreq(n, 1.0 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1.0 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    kk = (kx, ky, kz)
    grad = [[np.fft.irfftn(1j * kk[j] * u[i], s=(n, n, n), axes=(0, 1, 2)) for j in range(3)] for i in range(3)]
    ss = sum((0.5 * (grad[i][j] + grad[j][i])) ** 2 for i in range(3) for j in range(3)).mean()
    nut = 0.1 * dx * math.sqrt(0.1)
    assert st["energy"] == pytest.approx(0.1, rel=1e-14)
    assert st["B"] == 0.0
    assert st["dissipation"] == pytest.approx(0.1 ** 1.5 / dx, rel=1e-13)
    assert st["production"] == pytest.approx(2 * nut * ss, rel=1e-12)


def test_lag_model_les_means_for_uniform_fields():
    """The lag model (les_model 3, m_les.f90:1629-1684) from its initial state
    k_sgs = 0.1, (B T_B) = (eps T_eps) = 0.05 (m_les.f90:474-479): B = 0.05 <|S|>
    with |S| = sqrt(2 S:S), eps = 0.05^1.5 / Delta (C_T = 1), production as for
    the DLM."""
    n = 32
    o = oracle.Oracle(n, les_model=3, flow_type=0, nu=1.0 / 2000.0)
    assert o.fields.shape[0] == 6
    assert o.fields[4, 0, 0, 0] == o.fields[5, 0, 0, 0] == 0.05 * n ** 3
    o.init_velocity(RN1, isp_type=1, peak_wavenum=4.0)
    o.dealias_all()
    o.rhs()
    st = o.les_stats()
    dx = 2 * np.pi / n
    u = _to_complex(o.fields[:3]).transpose(0, 2, 1, 3)
    kz = np.fft.fftfreq(n, 1.0 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1.0 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    kk = (kx, ky, kz)
    grad = [[np.fft.irfftn(1j * kk[j] * u[i], s=(n, n, n), axes=(0, 1, 2)) for j in range(3)] for i in range(3)]
    ss = sum((0.5 * (grad[i][j] + grad[j][i])) ** 2 for i in range(3) for j in range(3))
    nut = 0.1 * dx * math.sqrt(0.1)
    assert st["energy"] == pytest.approx(0.1, rel=1e-14)
    assert st["production"] == pytest.approx(2 * nut * ss.mean(), rel=1e-12)
    assert st["B"] == pytest.approx(0.05 * np.sqrt(2 * ss).mean(), rel=1e-12)
    assert st["dissipation"] == pytest.approx(0.05 ** 1.5 / dx, rel=1e-13)


def _gaussian_transfer(n, delta):
    """The test filter of m_filter_xfftw.f90:197-220 (Gaussian, values below 1e-20
    dropped) as the numpy rfftn of its kernel."""
    dx = 2 * np.pi / n
    d = np.minimum(np.arange(n), n - np.arange(n)) * dx
    Z, Y, X = np.meshgrid(d, d, d, indexing="ij")
    c1 = 6.0 / delta ** 2
    g = (np.sqrt(c1 / np.pi) ** 3 * dx ** 3) * np.exp(-c1 * (X ** 2 + Y ** 2 + Z ** 2))
    g[g < 1e-20] = 0.0
    return np.fft.rfftn(g)


@pytest.mark.parametrize("model,k0", [(4, 0.2), (6, 0.5)])
def test_dynamic_structure_model_against_numpy(model, k0):
    """m_les_dstm_vel_k_sources (m_les.f90:1697-1960) restated in numpy for the
    initial uniform k_sgs: tau_ij = 2 k / L_kk L_ij with L_ij = (u_i u_j)~ -
    u~_i u~_j; the velocity RHS gains -d tau_ij/dx_j on the 2/3-rule modes and
    the production is <-tau_ij du_i/dx_j>.  The mixed model (6) adds the
    eddy-viscosity stress with C_mixed nu_Smagorinsky and its transfer."""
    n = 32
    kw = dict(flow_type=0, nu=1.0 / 2000.0)
    o = oracle.Oracle(n, les_model=model, **kw)
    o.set_les_constants(c_mixed=0.25)
    o0 = oracle.Oracle(n, les_model=0, **kw)
    o0.init_velocity(RN1, isp_type=1, peak_wavenum=4.0)
    o0.dealias_all()
    o.fields[:3] = o0.fields[:3]
    assert o.fields[3, 0, 0, 0] == k0 * n ** 3
    o.rhs()
    o0.rhs()
    u_hat = _to_complex(o0.fields[:3]).transpose(0, 2, 1, 3)          # [c][kz][ky][kx]
    kz = np.fft.fftfreq(n, 1.0 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1.0 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    kk = (kx, ky, kz)
    inv = lambda f: np.fft.irfftn(f, s=(n, n, n), axes=(0, 1, 2))
    fwd = lambda f: np.fft.rfftn(f, axes=(0, 1, 2))
    G = _gaussian_transfer(n, 4 * 2 * np.pi / n)
    u = [inv(u_hat[i]) for i in range(3)]
    uf = [inv(G * u_hat[i]) for i in range(3)]
    L = [[inv(G * fwd(u[i] * u[j])) - uf[i] * uf[j] for j in range(3)] for i in range(3)]
    Lkk = L[0][0] + L[1][1] + L[2][2]
    F = 2 * k0 / np.maximum(Lkk, 1e-15)
    tau = [[F * L[i][j] for j in range(3)] for i in range(3)]
    grad = [[inv(1j * kk[j] * u_hat[i]) for j in range(3)] for i in range(3)]
    prod = -sum(grad[i][j] * tau[i][j] for i in range(3) for j in range(3)).mean()
    keep = (np.abs(kz) <= n // 3) & (np.abs(ky) <= n // 3) & (kx <= n // 3)
    vsrc = [np.where(keep, -sum(1j * kk[j] * fwd(tau[i][j]) for j in range(3)), 0) for i in range(3)]
    d = _to_complex(o.wrk[1:4] - o0.wrk[1:4]).transpose(0, 2, 1, 3)
    st = o.les_stats()
    if model == 4:
        for i in range(3):
            assert np.abs(d[i] - vsrc[i]).max() <= 1e-10 * np.abs(vsrc[i]).max()
        assert st["production"] == pytest.approx(prod, rel=1e-10)
        dx = 2 * np.pi / n
        assert st["dissipation"] == pytest.approx(k0 ** 1.5 / dx, rel=1e-13)
    else:
        S = [[0.5 * (grad[i][j] + grad[j][i]) for j in range(3)] for i in range(3)]
        ss = sum(S[i][j] ** 2 for i in range(3) for j in range(3))
        nut = 0.25 * (0.18 * 2 * np.pi / n) ** 2 * np.sqrt(2 * ss)
        eddy = [np.where(keep, sum(1j * kk[j] * fwd(2 * nut * S[i][j]) for j in range(3)), 0) for i in range(3)]
        for i in range(3):
            want = vsrc[i] + eddy[i]
            assert np.abs(d[i] - want).max() <= 1e-10 * np.abs(want).max()
        assert st["production"] == pytest.approx(prod + (2 * nut * ss).mean(), rel=1e-10)


def test_model_10_against_numpy():
    """les_model 10 (m_les.f90:2009-2392) restated in numpy at its initial state
    (B T_B) = (eps T_eps) = 0.1: k = 0.2, c = 2 k / L_kk, tau_ij = c L_ij -
    2 C_mixed nu_t S_ij (nu_t Smagorinsky's), the velocity RHS gains -d
    tau_ij/dx_j on the 2/3-rule modes; production <-c L:S + C_mixed nu_t^3 /
    (c_s dx)^4>, B = 0.1 <|S|>, dissipation 0.1^1.5 / dx."""
    n, cm = 32, 0.4
    kw = dict(flow_type=0, nu=1.0 / 2000.0)
    o = oracle.Oracle(n, les_model=10, **kw)
    o.set_les_constants(c_mixed=cm)
    o0 = oracle.Oracle(n, les_model=0, **kw)
    o0.init_velocity(RN1, isp_type=1, peak_wavenum=4.0)
    o0.dealias_all()
    o.fields[:3] = o0.fields[:3]
    o.rhs()
    o0.rhs()
    u_hat = _to_complex(o0.fields[:3]).transpose(0, 2, 1, 3)
    kz = np.fft.fftfreq(n, 1.0 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1.0 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    kk = (kx, ky, kz)
    inv = lambda f: np.fft.irfftn(f, s=(n, n, n), axes=(0, 1, 2))
    fwd = lambda f: np.fft.rfftn(f, axes=(0, 1, 2))
    dx = 2 * np.pi / n
    G = _gaussian_transfer(n, 4 * dx)
    u = [inv(u_hat[i]) for i in range(3)]
    uf = [inv(G * u_hat[i]) for i in range(3)]
    L = [[inv(G * fwd(u[i] * u[j])) - uf[i] * uf[j] for j in range(3)] for i in range(3)]
    Lkk = L[0][0] + L[1][1] + L[2][2]
    c = np.where(Lkk < 1e-10, 0.0, 2 * 0.2 / np.where(Lkk < 1e-10, 1.0, Lkk))
    grad = [[inv(1j * kk[j] * u_hat[i]) for j in range(3)] for i in range(3)]
    S = [[0.5 * (grad[i][j] + grad[j][i]) for j in range(3)] for i in range(3)]
    ss = sum(S[i][j] ** 2 for i in range(3) for j in range(3))
    cs = 0.18 * dx
    nut = cs ** 2 * np.sqrt(2 * ss)
    tau = [[c * L[i][j] - cm * 2 * nut * S[i][j] for j in range(3)] for i in range(3)]
    keep = (np.abs(kz) <= n // 3) & (np.abs(ky) <= n // 3) & (kx <= n // 3)
    vsrc = [np.where(keep, -sum(1j * kk[j] * fwd(tau[i][j]) for j in range(3)), 0) for i in range(3)]
    d = _to_complex(o.wrk[1:4] - o0.wrk[1:4]).transpose(0, 2, 1, 3)
    for i in range(3):
        assert np.abs(d[i] - vsrc[i]).max() <= 1e-10 * np.abs(vsrc[i]).max()
    st = o.les_stats()
    lds = sum(L[i][j] * S[i][j] for i in range(3) for j in range(3))
    assert st["energy"] == pytest.approx(0.2, rel=1e-14)
    assert st["production"] == pytest.approx((-c * lds + cm * nut ** 3 / cs ** 4).mean(), rel=1e-10)
    assert st["B"] == pytest.approx(0.1 * np.sqrt(2 * ss).mean(), rel=1e-12)
    assert st["dissipation"] == pytest.approx(0.1 ** 1.5 / dx, rel=1e-13)


def _scalar_field(n, seed):
    """A smooth scalar field inside the 2/3-rule cube, in the reference layout."""
    rng = np.random.default_rng(seed)
    X, Y, Z = _grid(n)
    f = sum(rng.standard_normal() * np.cos(a * X + b * Y + c * Z + rng.uniform(0, 6.28))
            for a, b, c in rng.integers(-4, 5, size=(10, 3)))
    a = _phys(n, f)
    return a


@pytest.mark.parametrize("model", [1, 10])
def test_les_scalar_fluxes_against_numpy(model):
    """Passive scalars under LES: les_model 1 adds d/dx_i (nu_t dphi/dx_i)
    (m_les.f90:1028-1091); les_model 10 adds d/dx_i (T tau_ij dphi/dx_j) with
    T = (c_s dx)^2 / nu_t (Harlow, m_les.f90:2191-2270); both on the 2/3-rule
    modes, restated in numpy against a run without LES."""
    n, cm = 32, 0.4
    kw = dict(flow_type=0, nu=1.0 / 2000.0, nscal=1, sc=(0.7,), scalar_type=(1,))
    o = oracle.Oracle(n, les_model=model, **kw)
    o.set_les_constants(c_mixed=cm)
    o0 = oracle.Oracle(n, les_model=0, **kw)
    o0.init_velocity(RN1, isp_type=1, peak_wavenum=4.0)
    a = _scalar_field(n, 3)
    o0.fft3d(1, a)
    o0.fields[3] = a
    o0.dealias_all()
    o.fields[:4] = o0.fields[:4]
    for x in (o, o0):
        x.set_flags(1, 1, 1)
        x.rhs()
    u_hat = _to_complex(o0.fields[:4]).transpose(0, 2, 1, 3)
    kz = np.fft.fftfreq(n, 1.0 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1.0 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    kk = (kx, ky, kz)
    inv = lambda f: np.fft.irfftn(f, s=(n, n, n), axes=(0, 1, 2))
    fwd = lambda f: np.fft.rfftn(f, axes=(0, 1, 2))
    dx = 2 * np.pi / n
    grad = [[inv(1j * kk[j] * u_hat[i]) for j in range(3)] for i in range(3)]
    S = [[0.5 * (grad[i][j] + grad[j][i]) for j in range(3)] for i in range(3)]
    cs = 0.18 * dx
    nut = cs ** 2 * np.sqrt(2 * sum(S[i][j] ** 2 for i in range(3) for j in range(3)))
    gphi = [inv(1j * kk[j] * u_hat[3]) for j in range(3)]
    if model == 1:
        flux = [nut * gphi[i] for i in range(3)]
    else:
        G = _gaussian_transfer(n, 4 * dx)
        u = [inv(u_hat[i]) for i in range(3)]
        uf = [inv(G * u_hat[i]) for i in range(3)]
        L = [[inv(G * fwd(u[i] * u[j])) - uf[i] * uf[j] for j in range(3)] for i in range(3)]
        Lkk = L[0][0] + L[1][1] + L[2][2]
        c = np.where(Lkk < 1e-10, 0.0, 2 * 0.2 / np.where(Lkk < 1e-10, 1.0, Lkk))
        tau = [[c * L[i][j] - cm * 2 * nut * S[i][j] for j in range(3)] for i in range(3)]
        smag = nut / cs ** 2
        T = np.where(np.abs(smag) < 1e-10, 0.0, 1.0 / np.where(np.abs(smag) < 1e-10, 1.0, smag))
        flux = [T * sum(tau[i][j] * gphi[j] for j in range(3)) for i in range(3)]
    keep = (np.abs(kz) <= n // 3) & (np.abs(ky) <= n // 3) & (kx <= n // 3)
    want = np.where(keep, sum(1j * kk[i] * fwd(flux[i]) for i in range(3)), 0)
    d = _to_complex(o.wrk[4] - o0.wrk[4]).transpose(1, 0, 2)
    assert np.abs(d - want).max() <= 1e-10 * np.abs(want).max()


@pytest.mark.parametrize("stype,peak", [(1, 4.0), (2, 3.0), (101, 4.0)])
def test_init_scalar_imposes_the_target_spectrum(stype, peak):
    """init_scalar_spectrum (init_scalars.f90:84-240): the scalar's shells carry
    the normalised spectrum (types 1 and 3: k^3 e^{-3k/kp}; 2: (2 pi k/kp)^4 /
    (1 + (2 pi k/kp)^2)^3), binned as the reference bins; modes beyond N/3 zero."""
    n = 32
    o = oracle.Oracle(n, nscal=1, sc=(1.0,), scalar_type=(stype,))
    if stype == 101:             # a reaction-type scalar has no spectrum of its own
        with pytest.raises(ValueError):
            o.init_scalar(0, 93712139.0, peak)
        return
    o.init_scalar(0, 93712139.0, peak)
    akx, aky, akz = _wavenumbers(n)
    k2 = akx[None, None, :] ** 2 + aky[:, None, None] ** 2 + akz[None, :, None] ** 2
    sh = _shell32(k2)[..., :n]
    w = np.where(akx[:n] == 0, 0.5, 1.0)[None, None, :]
    e = o.fields[3, ..., :n] ** 2 * w / float(n) ** 6
    kmax = o.kmax
    got = np.bincount(sh.ravel(), weights=e.ravel(), minlength=kmax + 2)[1:kmax + 1]
    r = np.arange(1, kmax + 1) / peak
    tgt = r ** 3 / peak * np.exp(-3 * r) if stype == 1 else (2 * np.pi * r) ** 4 / (1 + (2 * np.pi * r) ** 2) ** 3
    assert np.abs(got - tgt / tgt.sum()).max() <= 1e-13
    keep = ((np.abs(aky) <= n // 3)[:, None, None] & (np.abs(akz) <= n // 3)[None, :, None]
            & (akx <= n // 3)[None, None, :])
    assert np.abs(o.fields[3][~keep]).max() == 0.0


def test_init_scalar_randu_continues_the_velocity_stream():
    """The RANDu state is module state (RANDu.f:20-22): a scalar made after the
    velocity differs from one made by a fresh generator (iy carries over)."""
    n = 16
    a = oracle.Oracle(n, nscal=1, sc=(1.0,), scalar_type=(1,))
    b = oracle.Oracle(n, nscal=1, sc=(1.0,), scalar_type=(1,))
    a.init_velocity(RN1, isp_type=1)
    a.init_scalar(0, 93712139.0)
    b.init_scalar(0, 93712139.0)
    assert not np.array_equal(a.fields[3], b.fields[3])


def test_init_scalar_profiles():
    """init_scalar_space (init_scalars.f90:280-345): type 13 is sin(k_p x) with
    k_p = min(peak, N/8); type 11 a tanh slab in z with zero mean."""
    n = 32
    o = oracle.Oracle(n, nscal=2, sc=(1.0, 1.0), scalar_type=(13, 11))
    o.init_scalar(0, 1.0, 6.0)
    o.init_scalar(1, 1.0, 2.0)
    X, Y, Z = _grid(n)
    a = o.fields[3].copy()
    o.fft3d(-1, a)
    assert np.abs(a[..., :n] - np.sin(4.0 * X)).max() <= 1e-13
    b = o.fields[4].copy()
    o.fft3d(-1, b)
    assert abs(b[..., :n].mean()) <= 1e-14
    assert np.abs(b[..., :n] - b[:, :1, :1][..., :1]).max() <= 1e-13   # depends on z only
