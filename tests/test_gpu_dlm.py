"""Dynamic localization model (les_model 2, m_les.f90:111-123, 1313-1621,
1041-1091): k_sgs transported as state field 3, nu_t = 0.1 Delta sqrt(k_sgs),
production, dissipation and turbulent diffusion of k_sgs, -2 nu_t S in the
velocity RHS; against the oracle, including the clipping of a negative k_sgs."""
import numpy as np
import pytest

from _cases import make_pair, relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32, 48])
def test_dlm_matches_oracle(n):
    o, g = make_pair(n, flow_type=1, les_model=2, nu=1.0 / 2000.0, dt=0.004, isp_type=2)
    assert g.download_fields().shape[0] == 4
    # m_les_dlm_k_init: k_sgs = 0.1 everywhere
    assert g.download_fields()[3, 0, 0, 0] == pytest.approx(0.1 * n ** 3, rel=1e-15)
    for _ in range(3):
        o.step(4)
        g.step(4)
        f = g.download_fields()
        assert relerr(f[:3], o.fields[:3]) < 1e-10
        assert relerr(f[3], o.fields[3]) < 1e-10
        # les.gp means of the last step (device block sums against the oracle's zero modes)
        gs, os_ = g.les_stats(), o.les_stats()
        assert gs["B"] == 0.0
        for k in ("energy", "production", "dissipation"):
            assert gs[k] == pytest.approx(os_[k], rel=1e-11), k
    assert relerr(g.download_rhs_old(), o.rhs_old) < 1e-9


def test_dlm_clips_negative_k_sgs_like_the_oracle():
    n = 32
    o, g = make_pair(n, flow_type=1, les_model=2, nu=1.0 / 2000.0, dt=0.004, isp_type=2)
    f = g.download_fields()
    f[3] = 0.0
    f[3, 0, 0, 0] = 0.1 * n ** 3
    f[3, 0, 0, 2] = 0.15 * n ** 3      # + 0.3 cos(x): k_sgs < 0 on part of the domain
    g.upload_fields(f)
    o.fields[:] = f
    o.step(1)
    g.step(1)
    got = g.download_fields()
    # the clipped field replaced the state: it now has modes beyond kx = 1
    assert np.abs(got[3, 0, 0, 4:8]).max() > 1e-3 * n ** 3
    assert relerr(got, o.fields) < 1e-10
    o.step(5)
    g.step(5)
    assert relerr(g.download_fields(), o.fields) < 1e-10


@pytest.mark.parametrize("n", [32, 48])
def test_lag_model_matches_oracle(n):
    """les_model 3: the DLM with the lag model for the dissipation; k_sgs,
    (B T_B) and (eps T_eps) are state fields 3, 4, 5."""
    o, g = make_pair(n, flow_type=1, les_model=3, nu=1.0 / 2000.0, dt=0.004, isp_type=2)
    f0 = g.download_fields()
    assert f0.shape[0] == 6
    assert f0[3, 0, 0, 0] == pytest.approx(0.1 * n ** 3, rel=1e-15)
    assert f0[4, 0, 0, 0] == f0[5, 0, 0, 0] == pytest.approx(0.05 * n ** 3, rel=1e-15)
    for _ in range(3):
        o.step(4)
        g.step(4)
        f = g.download_fields()
        for m in range(6):
            assert relerr(f[m], o.fields[m]) < 1e-10, m
        gs, os_ = g.les_stats(), o.les_stats()
        for k in ("energy", "production", "B", "dissipation"):
            assert gs[k] == pytest.approx(os_[k], rel=1e-11), k
    assert relerr(g.download_rhs_old(), o.rhs_old) < 1e-9


def test_les_stats_only_for_the_dynamic_localization_model():
    from hit3d_b200 import Context, Hit3dError, Params
    with Context(Params(nx=32, les_model=1)) as c:
        with pytest.raises(Hit3dError, match="les_models 2-7"):
            c.les_stats()


def test_dlm_rejects_what_it_does_not_support():
    from hit3d_b200 import Context, Hit3dError, Params
    with pytest.raises(Hit3dError, match="FP64"):
        Context(Params(nx=32, les_model=2, precision=1))
    with pytest.raises(Hit3dError, match="scalars"):
        Context(Params(nx=32, les_model=5, n_scalars=1, sc=[1.0], scalar_type=[0], c_t=1.0))


@pytest.mark.parametrize("model,nles", [(4, 1), (5, 3), (6, 1), (7, 3)])
def test_dynamic_structure_models_match_oracle(model, nles):
    """les_models 4-7 (m_les.f90:138-300, 1697-1960): the Dynamic Structure Model
    with the algebraic (4) or lag (5) dissipation, and the mixed models (6, 7)
    with C_mixed times the Smagorinsky viscosity; test filter Gaussian of width
    4 dx; parity of all fields and of the les.gp means."""
    n = 32
    o, g = make_pair(n, flow_type=1, les_model=model, nu=1.0 / 2000.0, dt=0.004, isp_type=2, c_t=0.8,
                     c_mixed=0.3)
    f0 = g.download_fields()
    assert f0.shape[0] == 3 + nles
    assert f0[3, 0, 0, 0] == pytest.approx((0.2 if model == 4 else 0.5) * n ** 3, rel=1e-15)
    for _ in range(3):
        o.step(3)
        g.step(3)
        f = g.download_fields()
        for m in range(3 + nles):
            assert relerr(f[m], o.fields[m]) < 1e-10, m
        gs, os_ = g.les_stats(), o.les_stats()
        for k in ("energy", "production", "B", "dissipation"):
            assert gs[k] == pytest.approx(os_[k], rel=1e-10, abs=1e-14), k
    assert relerr(g.download_rhs_old(), o.rhs_old) < 1e-9


def test_les_constants_are_required():
    from hit3d_b200 import Context, Hit3dError, Params
    with pytest.raises(Hit3dError, match="C_T"):
        Context(Params(nx=32, les_model=5, c_t=0.0))
    for m in (6, 7):
        with pytest.raises(Hit3dError, match="C_mixed"):
            Context(Params(nx=32, les_model=m))


def test_one_equation_mixed_model_matches_oracle():
    """les_model 10 (m_les.f90:303-358, 2009-2392): (B T_B) and (eps T_eps)
    transported, k = their sum, tau from the DSTM with C_mixed times the
    Smagorinsky stress; parity of the five fields and the les.gp means."""
    n = 32
    o, g = make_pair(n, flow_type=1, les_model=10, nu=1.0 / 2000.0, dt=0.004, isp_type=2, c_mixed=0.4)
    f0 = g.download_fields()
    assert f0.shape[0] == 5
    assert f0[3, 0, 0, 0] == f0[4, 0, 0, 0] == pytest.approx(0.1 * n ** 3, rel=1e-15)
    for _ in range(3):
        o.step(3)
        g.step(3)
        f = g.download_fields()
        for m in range(5):
            assert relerr(f[m], o.fields[m]) < 1e-10, m
        gs, os_ = g.les_stats(), o.les_stats()
        for k in ("energy", "production", "B", "dissipation"):
            assert gs[k] == pytest.approx(os_[k], rel=1e-10, abs=1e-14), k
    assert relerr(g.download_rhs_old(), o.rhs_old) < 1e-9


@pytest.mark.parametrize("model", [1, 2, 3, 10])
def test_les_with_passive_scalars_matches_oracle(model):
    """Passive scalars under LES: turbulent diffusion with nu_t (les_models 1-3,
    m_les.f90:1028-1091) or Harlow fluxes (10, m_les.f90:2191-2270), next to the
    LES fields, which follow the scalars in the state."""
    n = 32
    kw = dict(flow_type=1, les_model=model, nu=1.0 / 2000.0, dt=0.004, isp_type=2, nscal=2, sc=(0.7, 1.0),
              scalar_type=(0, 1), c_mixed=0.4)
    o, g = make_pair(n, **kw)
    f = g.download_fields()
    rng = np.random.default_rng(model)
    for s in (3, 4):   # smooth scalar fields inside the 2/3-rule cube
        f[s] = 0.0
        for _ in range(8):
            # kx >= 1: no Hermitian constraint to respect on the kx = 0 plane
            ky, kz, kx = rng.integers(-5, 6), rng.integers(-5, 6), rng.integers(1, 6)
            f[s, ky % n, kz % n, 2 * kx:2 * kx + 2] = rng.standard_normal(2) * n ** 3 * 0.01
    g.upload_fields(f)
    g.dealias_all()
    f = g.download_fields()
    o.fields[:] = f
    g.set_scalars_active(True)
    o.set_flags(1, 1, 1)
    for _ in range(3):
        o.step(3)
        g.step(3)
        got = g.download_fields()
        for m in range(got.shape[0]):
            assert relerr(got[m], o.fields[m]) < 1e-10, m
    if model != 1:
        gs, os_ = g.les_stats(), o.les_stats()
        for k in ("energy", "production", "B", "dissipation"):
            assert gs[k] == pytest.approx(os_[k], rel=1e-10, abs=1e-14), k


@pytest.mark.parametrize("model", [2, 10])
def test_idle_passive_scalars_next_to_les_fields(model):
    """Before TSCALAR the reference still advances the passive scalars when LES
    fields move, with a RHS of only the mean-gradient source and the LES fluxes
    (rhs_scalars.f90:28-36, 384-395, main.f90:132-146); then they start moving."""
    n = 32
    kw = dict(flow_type=1, les_model=model, nu=1.0 / 2000.0, dt=0.004, isp_type=2, nscal=2, sc=(0.7, 1.0),
              scalar_type=(0, 1), c_mixed=0.4)
    o, g = make_pair(n, **kw)
    f = g.download_fields()
    rng = np.random.default_rng(7)
    for s in (3, 4):
        f[s] = 0.0
        for _ in range(6):
            ky, kz, kx = rng.integers(-5, 6), rng.integers(-5, 6), rng.integers(1, 6)
            f[s, ky % n, kz % n, 2 * kx:2 * kx + 2] = rng.standard_normal(2) * n ** 3 * 0.01
    g.upload_fields(f)
    g.dealias_all()
    o.fields[:] = g.download_fields()
    g.set_scalars_active(False)
    o.set_flags(1, 1, 0)
    o.step(3)
    g.step(3)
    got = g.download_fields()
    for m in range(got.shape[0]):
        assert relerr(got[m], o.fields[m]) < 1e-10, m
    # the scalars start moving
    g.set_scalars_active(True)
    fl = list(o.flags())
    o.set_flags(fl[0], fl[1], 1)
    o.step(3)
    g.step(3)
    got = g.download_fields()
    for m in range(got.shape[0]):
        assert relerr(got[m], o.fields[m]) < 1e-10, m


def test_dynamic_structure_models_refuse_passive_scalars():
    from hit3d_b200 import Context, Hit3dError, Params
    with pytest.raises(Hit3dError, match="scalars"):
        Context(Params(nx=32, les_model=4, n_scalars=1, sc=[1.0], scalar_type=[0]))
