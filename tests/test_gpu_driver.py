"""The host main loop over the C-ABI (main.f90) and the device pieces it needs:
velocity_rescale, the truncated physical output of io_write_4, restart files."""
import os
import shutil

import numpy as np
import pytest

from _cases import make_pair, relerr

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("isp", [0, 1, 3])
def test_velocity_rescale_matches_oracle(isp):
    o, g = make_pair(32, dealias=0, flow_type=0)
    o.step(3)
    g.step(3)
    o.velocity_rescale(isp, 4.0)
    g.velocity_rescale(isp, 4.0)
    f = g.download_fields()
    for m in range(3):
        assert relerr(f[m], o.fields[m]) < 1e-10


def test_truncated_physical_fields_match_oracle():
    o, g = make_pair(32)
    kmax = 32 // 3
    phys = g.physical_fields(3, float(kmax) ** 2)
    n = 32
    ky = np.fft.fftfreq(n, 1.0 / n)
    ky[n // 2] = n // 2
    kx = np.repeat(np.arange(n // 2 + 1), 2)
    k2 = ky[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    for c in range(3):
        a = np.ascontiguousarray(o.fields[c]).copy()
        a[k2 > kmax ** 2] = 0.0
        o.fft3d(-1, a)
        assert relerr(phys[c][:, :, :n], a[:, :, :n]) < 1e-13


def test_driver_run_writes_reference_files(tmp_path):
    from hit3d_b200.driver import Simulation
    from hit3d_b200.restart import read_real4, read_restart
    wd = str(tmp_path)
    shutil.copy(os.path.join(GOLDEN, "decay64_.in"), os.path.join(wd, "decay64_.in"))
    sim = Simulation("decay64_", wd)
    sim.begin()
    reason = sim.run()
    assert reason == 0 and sim.itime == 20
    lines = [ln for ln in open(os.path.join(wd, "stat1.gp")) if not ln.lstrip().startswith("#")]
    assert len(lines) == 2 and lines[0].split()[0] == "10"
    es_blocks = open(os.path.join(wd, "es.gp")).read().count("# ITIME=")
    assert es_blocks == 2
    # the run log: format 9000 of main.f90 at every statistics step, then my_exit
    log = open(os.path.join(wd, "d0000.txt")).read().splitlines()
    assert [ln[:12] for ln in log[:2]] == ["ITIME=    10", "ITIME=    20"]
    assert log[1].rstrip().endswith("*") and "TIME=  0.1000" in log[1]
    assert log[-1] == "my_exit with reason    0"
    assert os.path.exists(os.path.join(wd, "sc01.gp")) and os.path.exists(os.path.join(wd, "es_02.gp"))
    u0 = read_real4(os.path.join(wd, "u.000000"))
    assert u0.shape == (64, 64, 64) and np.isfinite(u0).all()
    f, t, dt, nums, nles = read_restart(os.path.join(wd, "decay64_.64.000020"), 64, 2)
    assert nums == 2 and abs(t - 20 * 0.005) < 1e-12
    g = sim.ctx.download_fields()
    assert np.array_equal(f[..., :64], g[..., :64])


def test_stop_file_ends_the_run_with_a_restart(tmp_path):
    from hit3d_b200.driver import Simulation
    wd = str(tmp_path)
    shutil.copy(os.path.join(GOLDEN, "decay64_.in"), os.path.join(wd, "decay64_.in"))
    open(os.path.join(wd, "stop"), "w").close()
    sim = Simulation("decay64_", wd)
    sim.begin()
    assert sim.run() == 3 and sim.itime == 10
    assert os.path.exists(os.path.join(wd, "decay64_.64.000010"))


@pytest.mark.parametrize("model,nles", [(2, 1), (3, 3)])
def test_dlm_run_restarts_with_k_sgs(tmp_path, model, nles):
    """The dynamic localization models through the host loop: the restart file
    carries the LES fields (nles = 1 or 3, as restart_io.f90 writes them) and a
    run restarted from it continues with the same state."""
    from dataclasses import replace
    from hit3d_b200.driver import Simulation
    from hit3d_b200.params import read_input_file
    from hit3d_b200.restart import read_restart
    wd = str(tmp_path)
    cfg = read_input_file(os.path.join(GOLDEN, "decay64_.in"))
    cfg = replace(cfg, les_model=model, n_scalars=0, scalar_type=[], sc=[], ir_exp_sc=[], peak_wavenum_sc=[],
                  reac_sc=[], itmax=6, iprint1=3, iprint2=3, iwrite4=100, tmax=10.0)
    sim = Simulation("dlm64", wd, cfg=cfg)
    sim.begin()
    assert sim.run() == 0 and sim.itime == 6
    # les.gp at every statistics step: itime, time, mean k_sgs, production, B, dissipation
    rows = [ln.split() for ln in open(os.path.join(wd, "les.gp"))]
    assert [int(r[0]) for r in rows] == [3, 6] and all(len(r) == 6 for r in rows)
    assert float(rows[1][1]) == pytest.approx(5 * 0.005, rel=1e-6)
    assert (float(rows[1][4]) == 0.0) == (model == 2)       # B: only with the lag model
    assert float(rows[1][3]) > 0 and float(rows[1][5]) > 0
    f, t, dt, nums, nles_read = read_restart(os.path.join(wd, "dlm64.64.000006"), 64, 0, nles)
    assert nums == 0 and nles_read == nles and f.shape[0] == 3 + nles
    g = sim.ctx.download_fields()
    assert np.array_equal(f[..., :64], g[..., :64])
    sim2 = Simulation("dlm64", wd, cfg=replace(cfg, itmin=6))
    sim2.begin()
    assert np.array_equal(sim2.ctx.download_fields()[..., :64], g[..., :64])


def test_run_limit_ends_the_run_with_a_restart(tmp_path):
    """job_parameters.txt gives the run limit in minutes; the loop leaves with
    reason 2 at the first 10-step check within 5 minutes of it (main.f90)."""
    from hit3d_b200.driver import Simulation
    wd = str(tmp_path)
    shutil.copy(os.path.join(GOLDEN, "decay64_.in"), os.path.join(wd, "decay64_.in"))
    with open(os.path.join(wd, "job_parameters.txt"), "w") as fh:
        fh.write("4.0\n")
    sim = Simulation("decay64_", wd)
    assert sim.job_runlimit == 4.0
    sim.begin()
    assert sim.run() == 2 and sim.itime == 10
    assert os.path.exists(os.path.join(wd, "decay64_.64.000010"))


def test_non_finite_state_is_detected_on_the_device(tmp_path):
    """NaN and Inf planted in a host copy of the state are counted by the
    device reduction, and the host loop then ends with reason -2 and writes
    no restart."""
    from hit3d_b200.driver import Simulation
    wd = str(tmp_path)
    shutil.copy(os.path.join(GOLDEN, "decay64_.in"), os.path.join(wd, "decay64_.in"))
    sim = Simulation("decay64_", wd)
    sim.begin()
    assert sim.ctx.nonfinite() == 0
    f = sim.ctx.download_fields()
    good = f.copy()
    f[1, 5, 7, 9] = np.nan
    f[4, 0, 0, 0] = np.inf
    f[0, 63, 63, 65] = -np.inf
    sim.ctx.upload_fields(f)
    assert sim.ctx.nonfinite() == 3
    sim.ctx.upload_fields(good)
    assert sim.ctx.nonfinite() == 0
    f[2, 3, 3, 3] = np.nan
    sim.ctx.upload_fields(f)
    # the Courant maximum (fmax) passes over NaN, so the statistics step finds it
    assert sim.run() == -2 and sim.itime == 10
    assert not any(n.startswith("decay64_.64.") for n in os.listdir(wd))


def test_sidecar_runs_the_learned_closure_with_fixed_settings(tmp_path):
    """<run>.gpu.in turns an unmodified .in file into a learned-closure run in
    the FP32 form with a fixed launch shape and no pruning; the state equals a
    Context driven with the same settings directly."""
    from hit3d_b200 import Context
    from hit3d_b200.driver import Simulation
    from hit3d_b200.params import read_input_file
    from oracle import mlp_oracle as mo
    wd = str(tmp_path)
    # the sample input without its passive scalars (LES runs here carry none)
    text = open(os.path.join(GOLDEN, "decay64_.in")).read()
    text = text.replace("2\t\tnums, # of passive scalars", "0\t\tnums, # of passive scalars")
    with open(os.path.join(wd, "decay64_.in"), "w") as fh:
        fh.write(text)
    w = mo.bf16_bits(mo.bf16_round(mo.init_params(4) * 0.05))
    np.save(os.path.join(wd, "closure.npy"), w)
    delta = 4 * np.pi / 64
    with open(os.path.join(wd, "decay64_.gpu.in"), "w") as fh:
        fh.write(f"precision = 1\npruning = off\nvariant = 5\nles_model = 20\nles_mlp = closure.npy\n"
                 f"les_mlp_delta = {delta!r}\nles_mlp_kernel = 1\n")
    sim = Simulation("decay64_", wd)
    assert sim.cfg.les_model == 20 and sim.settings.precision == 1 and not sim.ctx.pruned
    sim.begin()
    assert sim.run(max_steps=4) is None and sim.itime == 4
    got = sim.ctx.download_fields()
    assert np.isfinite(got).all()

    cfg = read_input_file(os.path.join(wd, "decay64_.in"))
    cfg.les_model = 20
    c = Context(cfg.to_params(precision=1))
    c.set_pruning(False)
    c.set_variant(5)
    c.les_set_mlp(w, delta, clip=True, kernel=1)
    assert cfg.n_scalars == 0
    c.init_velocity(cfg.rn1, cfg.isp_type, cfg.peak_wavenum, float(cfg.ir_exp))
    c.fov = c.fos = 1
    c.dealias_all()
    c.step(4)
    assert np.array_equal(c.download_fields(), got)
    c.close()


def test_particles_through_the_host_loop(tmp_path):
    """The 'parts' task of the reference through the host loop: 27 lattice
    particles from time_p = 0, trajectories p.NNNN every step (nptot < 1000)
    and pt.<ext> every IWRITE4 steps and at the end."""
    from hit3d_b200 import particles as pt
    from hit3d_b200.driver import Simulation
    wd = str(tmp_path)
    text = open(os.path.join(GOLDEN, "decay64_.in")).read()
    text = text.replace("0\t\tnp, number of Largangian particles", "27\t\tnp, number of Largangian particles")
    text = text.replace("0.1\t\ttime_p, when to release the particles into the flow",
                        "0.0\t\ttime_p, when to release the particles into the flow")
    text = text.replace("20\t\tIWRITE4", "2\t\tIWRITE4")
    with open(os.path.join(wd, "decay64_.in"), "w") as fh:
        fh.write(text)
    sim = Simulation("decay64_", wd)
    assert sim.cfg.nptot == 27 and sim.cfg.starttime_particles == 0.0
    sim.begin()
    assert sim.run(max_steps=4) is None
    grid, uvw = sim.ctx.particles_download()
    assert grid.shape == (27, 3) and np.isfinite(uvw).all() and np.abs(uvw).max() > 0
    rows = open(os.path.join(wd, "p.0001")).read().splitlines()
    assert [int(r[:6]) for r in rows] == [1, 2, 3, 4]
    last = [float(rows[-1][11 + 16 * k: 11 + 16 * (k + 1)]) for k in range(7)]
    dx = 2 * np.pi / 64
    assert np.allclose(last[1:4], (grid[0] - 1.0) * dx, rtol=1e-7)
    assert np.allclose(last[4:7], uvw[0], rtol=1e-7, atol=1e-12)
    ip, g4, t4 = pt.read_pt(os.path.join(wd, "pt.000004"), 64)
    # the 'parts' task's TIME: the start of step 4
    assert np.array_equal(ip, np.arange(1, 28)) and abs(t4 - 3 * 0.005) < 1e-12
    assert np.allclose(g4, grid, rtol=0, atol=1e-10)
    assert os.path.exists(os.path.join(wd, "pt.000002"))


def test_restart_with_an_added_scalar_initialises_it(tmp_path):
    """restart_io.f90:419-432: a scalar the .in file adds to a restart file
    without it starts from its initial condition (type 1: a random field)."""
    from dataclasses import replace
    from hit3d_b200.driver import Simulation
    from hit3d_b200.params import read_input_file
    wd = str(tmp_path)
    cfg = read_input_file(os.path.join(GOLDEN, "decay64_.in"))
    cfg0 = replace(cfg, n_scalars=0, scalar_type=[], sc=[], ir_exp_sc=[], peak_wavenum_sc=[], reac_sc=[],
                   itmax=2, iprint1=2, iprint2=2, iwrite4=100)
    sim = Simulation("add64", wd, cfg=cfg0)
    sim.begin()
    assert sim.run() == 0
    cfg1 = replace(cfg, n_scalars=1, scalar_type=[1], sc=[0.7], ir_exp_sc=[4.0], peak_wavenum_sc=[3.0],
                   reac_sc=[0.0], itmin=2, itmax=4, iprint1=2, iprint2=2, iwrite4=100)
    sim2 = Simulation("add64", wd, cfg=cfg1)
    sim2.begin()
    f = sim2.ctx.download_fields()
    assert f.shape[0] == 4 and np.abs(f[3]).max() > 0
    assert np.array_equal(f[:3, ..., :64], sim.ctx.download_fields()[:3, ..., :64])
