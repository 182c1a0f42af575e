"""Shared set-up for parity tests: matched oracle / GPU runs on the same inputs."""
from __future__ import annotations

import numpy as np

RN1 = 67748937.0  # RN1 of the reference's sample input (scripts/00_example.in:32)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def spectral_view(fields):
    """(nf, ky, kz, kx re/im) real array -> complex (nf, ky, kz, kx)."""
    return fields[..., 0::2] + 1j * fields[..., 1::2]


def make_pair(n, *, dealias=0, flow_type=0, kfmax=2, nu=1.0 / 400.0, dt=0.005, famp=0.5, nscal=0, sc=(),
              scalar_type=(), les_model=0, c_smag=0.18, precision=0, isp_type=1, peak=4.0, ir_exp=2.0,
              init="gpu", c_t=1.0, c_mixed=0.0):
    """Create an oracle and a GPU context holding the same initial state.

    init="gpu": velocity initialised by the GPU path, copied into the oracle.
    init="oracle": velocity initialised by the oracle, uploaded to the GPU."""
    import oracle
    from hit3d_b200 import Context, Params

    o = oracle.Oracle(n, nscal=nscal, dealias=dealias, flow_type=flow_type, kfmax=kfmax, nu=nu, dt=dt, famp=famp,
                      les_model=les_model, c_smag=c_smag, sc=sc, scalar_type=scalar_type)
    o.set_les_constants(c_t, c_mixed)
    p = Params(nx=n, dealias=dealias, flow_type=flow_type, kfmax=kfmax, nu=nu, dt=dt, famp=famp, n_scalars=nscal,
               sc=list(sc), scalar_type=list(scalar_type), les_model=les_model, c_smag=c_smag, precision=precision,
               c_t=c_t, c_mixed=c_mixed)
    g = Context(p)
    if init == "gpu":
        g.init_velocity(RN1, isp_type, peak, ir_exp)
        g.dealias_all()
        f = g.download_fields()
        o.fields[:] = f
    else:
        o.init_velocity(RN1, isp_type=isp_type, peak_wavenum=peak, ir_exp=ir_exp)
        o.dealias_all()
        g.upload_fields(np.ascontiguousarray(o.fields))
    return o, g


def seed_scalars(o, g, nscal, rng):
    """Give the scalars a smooth random spectral field (low modes only)."""
    n = o.n
    f = np.ascontiguousarray(o.fields).copy()
    for s in range(nscal):
        phys = np.zeros((n, n, n + 2))
        x = 2 * np.pi * np.arange(n) / n
        Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
        a = rng.standard_normal(6)
        phys[:, :, :n] = a[0] * np.sin(X + a[1]) + a[2] * np.cos(2 * Y + a[3]) + a[4] * np.sin(Z - Y + a[5])
        o.fft3d(1, phys)
        f[3 + s] = phys
    o.fields[:] = f
    g.upload_fields(np.ascontiguousarray(f))
