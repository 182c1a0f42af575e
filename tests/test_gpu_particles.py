"""Particle parity (m_particles.f90:815-1230): trilinear and 4-point cubic (CINT)
interpolation of the level-n velocity, AB2 in grid units, periodic wrap-around."""
import numpy as np
import pytest

from _cases import make_pair, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme", [0, 1])
def test_particles_match_oracle(scheme):
    import oracle
    n = 32
    o, g = make_pair(n, dealias=0, flow_type=1, kfmax=2, nu=1.0 / 100.0, dt=0.01)
    rng = np.random.default_rng(11)
    npart = 5000
    xyz = 1.0 + rng.random((npart, 3)) * n
    g.particles_upload(xyz, None, scheme)
    xo = xyz.copy()
    uo = np.full((npart, 3), -999.0)
    for _ in range(5):
        up = np.zeros((3, n, n, n + 2))
        for c in range(3):
            a = np.ascontiguousarray(o.fields[c]).copy()
            o.fft3d(-1, a)
            up[c] = a
        oracle.particles_step(n, o_dt := 0.01, up, xo, uo, scheme)
        o.step(1)
        g.step(1)
    xg, ug = g.particles_download()
    assert relerr(ug, uo) < 1e-10
    assert np.abs(xg - xo).max() < 1e-9
    assert xg.min() >= 1.0 and xg.max() < n + 1.0


def test_lattice_init_counts():
    import oracle
    x = oracle.particles_lattice(256, 10 ** 6)
    assert x.shape == (10 ** 6, 3)
    assert x.min() >= 1.0 and x.max() < 257.0


@pytest.mark.parametrize("scheme", [0, 1])
def test_filtered_particle_velocity_matches_oracle(scheme):
    """particles_filter_size > 0 (m_particles.f90:759-766): the particles move
    with the velocity filtered by the Gaussian of that width
    (m_filter_xfftw.f90:197-220); the oracle filters and inverse-transforms."""
    import oracle
    n, delta = 32, 4.0 * 2 * np.pi / 32
    o, g = make_pair(n, dealias=0, flow_type=1, kfmax=2, nu=1.0 / 100.0, dt=0.01)
    rng = np.random.default_rng(5)
    npart = 3000
    xyz = 1.0 + rng.random((npart, 3)) * n
    g.particles_upload(xyz, None, scheme)
    g.particles_filter(delta)
    gf = o.filter_g(2, delta)
    xo = xyz.copy()
    uo = np.full((npart, 3), -999.0)
    for _ in range(4):
        up = np.zeros((3, n, n, n + 2))
        for c in range(3):
            a = np.ascontiguousarray(o.fields[c]).copy()
            o.apply_filter(gf, a)
            o.fft3d(-1, a)
            up[c] = a
        oracle.particles_step(n, 0.01, up, xo, uo, scheme)
        o.step(1)
        g.step(1)
    xg, ug = g.particles_download()
    assert relerr(ug, uo) < 1e-10
    assert np.abs(xg - xo).max() < 1e-9
    from hit3d_b200 import Hit3dError
    with pytest.raises(Hit3dError, match="too small"):
        g.particles_filter(2.0 * 2 * np.pi / 32)
