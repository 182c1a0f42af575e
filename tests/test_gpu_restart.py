"""Restart files packed and unpacked on the device (restart_io.f90:240-506):
the image equals the host writer's bytes, reads back through the oracle's
restart reader to the oracle's own fields, and loads back into a context."""
import os

import numpy as np
import pytest

from _cases import RN1, make_pair, seed_scalars, spectral_view

pytestmark = pytest.mark.gpu


def test_device_image_equals_host_writer(tmp_path):
    from hit3d_b200.restart import write_restart
    rng = np.random.default_rng(3)
    o, g = make_pair(32, dealias=0, flow_type=1, nu=1.0 / 300.0, dt=0.004, nscal=2, sc=(0.7, 1.0),
                     scalar_type=(0, 0))
    seed_scalars(o, g, 2, rng)
    g.set_scalars_active(True)
    g.step(3)
    f = g.download_fields()
    for nums in (2, 0):
        p = str(tmp_path / f"host_{nums}")
        write_restart(p, np.ascontiguousarray(f[:3 + nums]), 1.25, 0.004, nums)
        img = g.restart_image(1.25, 0.004, nums)
        assert img.tobytes() == open(p, "rb").read(), nums
    g.close()


def test_image_reads_back_through_the_oracle(tmp_path):
    """GPU and oracle advance the same state; the GPU's restart file, read by the
    oracle's restart_read restatement, equals the oracle's fields to 1e-10 per mode."""
    import oracle
    o, g = make_pair(64, dealias=0, flow_type=1, kfmax=2, nu=1.0 / 400.0, dt=0.004)
    o.step(5)
    g.step(5)
    path = str(tmp_path / "run.64.000005")
    with open(path, "wb") as fh:
        fh.write(g.restart_image(0.02, 0.004).tobytes())
    o2 = oracle.Oracle(64, dealias=0, flow_type=1, kfmax=2, nu=1.0 / 400.0, dt=0.004)
    t, dt, nums, nles = o2.read_restart(path)
    assert (t, dt, nums, nles) == (0.02, 0.004, 0, 0)
    for m in range(3):
        a, b = spectral_view(o2.fields[m]), spectral_view(o.fields[m])
        assert (np.abs(a - b) <= 1e-10 * np.abs(b) + 1e-12 * np.abs(b).max()).all(), m
    g.close()


def test_image_round_trip_and_scalar_counts():
    from hit3d_b200 import Context, Hit3dError, Params
    rng = np.random.default_rng(8)
    o, g = make_pair(32, dealias=0, flow_type=1, nu=1.0 / 300.0, dt=0.004, nscal=2, sc=(0.7, 1.0),
                     scalar_type=(0, 0))
    seed_scalars(o, g, 2, rng)
    f = g.download_fields()
    f[..., 32:] = 0.0  # the file carries no kx = N/2 pair; loading zeroes it
    img = g.restart_image(0.5, 0.004)
    h = Context(Params(nx=32, flow_type=1, nu=1.0 / 300.0, dt=0.004, n_scalars=2, sc=[0.7, 1.0], scalar_type=[0, 0]))
    assert h.restart_load(img) == (0.5, 0.004, 2, 0)
    assert np.array_equal(h.download_fields(), f)
    # a file with one scalar fills the second with zeros; one with three drops the third
    h.upload_fields(f + 1.0)
    assert h.restart_load(g.restart_image(0.5, 0.004, 1)) == (0.5, 0.004, 1, 0)
    got = h.download_fields()
    assert np.array_equal(got[:4], f[:4]) and np.abs(got[4]).max() == 0.0
    k = Context(Params(nx=32, flow_type=1, nu=1.0 / 300.0, dt=0.004, n_scalars=1, sc=[0.7], scalar_type=[0]))
    k.restart_load(img)
    assert np.array_equal(k.download_fields(), f[:4])
    wrong = Context(Params(nx=48))
    with pytest.raises(Hit3dError, match="Dimensions are different"):
        wrong.restart_load(img)
    with pytest.raises(Hit3dError, match="size"):
        h.restart_load(img[:-8])
    for c in (g, h, k, wrong):
        c.close()
