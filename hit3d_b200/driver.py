"""Host main loop of the hydro task over the C-ABI (restates main.f90:22-300).

The reference's Fortran host keeps the input file, the restart layout, the seeds
and the statistics files; here the same host logic drives the device through
hit3d_b200.gpu.  Output files keep the reference's names and formats:
stat1.gp / stat2.gp / es.gp (m_stats.f90:150-185), scNN.gp / es_NN.gp
(m_stats.f90:66-80, 420-432), u./v./w./scNN. real*4 files (io_write_4.f90) and
<run_name>.64.<itime> restart files (restart_io.f90).  Exit reasons follow
my_exit.f90:23-62: 0 normal, 1 TMAX, 2 run limit, 3 user 'stop' file.  One
reason is added, -2: the state turned non-finite (a non-finite Courant number,
or the device count of non-finite modes at a statistics step); as for every
negative reason of my_exit.f90:58-61, no restart is written over good ones.
"""
from __future__ import annotations

import math
import os
import time as _time

import numpy as np

from .gpu import Context, les_fields
from .params import InputFileError, RunConfig, read_input_file
from .restart import read_restart_header, restart_name, write_real4
from . import particles as _pt
from .sidecar import GpuSettings, SidecarError, read_sidecar


def _fmt_e(x: float, w: int = 15, d: int = 6) -> str:
    """Fortran Ew.d edit descriptor (0.dddddE+xx form)."""
    if x == 0.0 or not math.isfinite(x):
        m, e = 0.0, 0
    else:
        e = int(math.floor(math.log10(abs(x)))) + 1
        m = x / 10.0 ** e
        if round(abs(m), d) >= 1.0:
            m /= 10.0
            e += 1
    s = f"{'-' if m < 0 else ''}0.{int(round(abs(m) * 10 ** d)):0{d}d}E{'+' if e >= 0 else '-'}{abs(e):02d}"
    return s.rjust(w)


# les_model_name of m_les.f90:56-352, the last column of the progress line
LES_MODEL_NAME = {1: " SM", 2: "DLM", 3: "DLL", 4: "DST", 5: "STL", 6: "MMA", 7: "MML", 10: "#10", 20: "MLP"}


class Simulation:
    """One run: the reference's hydro task with the state resident on the GPU."""

    def __init__(self, run_name: str, workdir: str = ".", cfg: RunConfig | None = None,
                 precision: int | None = None, device: int | None = None, job_runlimit_min: float = 12 * 60,
                 settings: GpuSettings | None = None):
        """cfg: the `.in` settings (read from workdir if None); settings: those of
        `<run_name>.gpu.in` (read from workdir if None); precision and device, when
        given, override the settings."""
        self.run_name = run_name
        self.wd = workdir
        self.cfg = cfg or read_input_file(os.path.join(workdir, run_name + ".in"))
        s = settings if settings is not None else read_sidecar(workdir, run_name)
        if precision is not None:
            s.precision = precision
        if device is not None:
            s.device = device
        self.settings = s
        if s.les_model is not None:
            self.cfg.les_model = s.les_model
            if s.les_model > 0:
                self.cfg.dealias = 0  # every LES model runs with the 2/3 rule (m_parameters.f90:416-420)
        c_t, c_mixed = self._les_constants()
        self.ctx = Context(self.cfg.to_params(precision=s.precision, device=s.device, c_smag=s.c_smag, c_t=c_t,
                                              c_mixed=c_mixed))
        if not s.pruning:
            self.ctx.set_pruning(False)
        if s.variant is not None:
            self.ctx.set_variant(s.variant)
        if self.cfg.les_model == 20:
            self._load_closure()
        self.time = 0.0
        self.itime = self.cfg.itmin
        self.int_scalars = False
        self.t0 = _time.time()
        self.job_runlimit = job_runlimit_min
        p = os.path.join(workdir, "job_parameters.txt")
        if os.path.exists(p):
            try:
                self.job_runlimit = float(open(p).read().split()[0])
            except (ValueError, IndexError):
                pass
        self.exit_reason = None
        self.log = []
        # Lagrangian particles (the reference's 'parts' task)
        self.int_particles = False
        self.ipart = None
        self.particles_time = 0.0

    def _out(self, line: str):
        """A line of the run log d0000.txt (the reference's unit `out`, m_io.f90:27);
        the progress line has format 9000 of main.f90:301-302."""
        self.log.append(line)
        with open(os.path.join(self.wd, "d0000.txt"), "a") as fh:
            fh.write(line + "\n")

    def _les_constants(self):
        """C_T of les_model 5 from c_t.in and C_mixed of les_models 6, 7, 10 from
        c_mixed.in, first value of the file, as m_les_init reads them
        (m_les.f90:189-207, 213-290, 314-335); a missing file stops the run,
        except for les_model 10, which then takes C_mixed = 0.5."""
        def first_value(name):
            path = os.path.join(self.wd, name)
            if not os.path.exists(path):
                raise InputFileError(f"Cannot find the file '{name}' (les_model {self.cfg.les_model})")
            try:
                return float(open(path).read().replace(",", " ").split()[0].replace("d", "e").replace("D", "e"))
            except (IndexError, ValueError) as e:
                raise InputFileError(f"bad value in {name}") from e
        m = self.cfg.les_model
        c_mixed = 0.0
        if m in (6, 7):
            c_mixed = first_value("c_mixed.in")
        elif m == 10:
            c_mixed = first_value("c_mixed.in") if os.path.exists(os.path.join(self.wd, "c_mixed.in")) else 0.5
        return (first_value("c_t.in") if m == 5 else 1.0), c_mixed

    def _load_closure(self):
        s = self.settings
        if s.les_mlp is None:
            raise SidecarError("les_model 20 (learned closure) needs les_mlp weights")
        path = s.les_mlp if os.path.isabs(s.les_mlp) else os.path.join(self.wd, s.les_mlp)
        w = np.load(path)
        if w.dtype != np.uint16:
            raise SidecarError(f"{path}: the closure weights must be bf16 bit patterns (uint16), got {w.dtype}")
        delta = s.les_mlp_delta if s.les_mlp_delta is not None else 2.0 * self.cfg.dx
        self.ctx.les_set_mlp(w, delta, clip=s.les_mlp_clip, kernel=s.les_mlp_kernel)

    # -- start-up (begin_new.f90 / begin_restart.f90) ---------------------------
    def begin(self):
        c = self.cfg
        if c.itmin == 0:
            self.time = 0.0
            self.itime = 0
            if c.tscalar <= 0.0 and c.n_scalars > 0:
                self.int_scalars = True
            self.ctx.init_velocity(c.rn1, c.isp_type, c.peak_wavenum, float(c.ir_exp))
            if c.n_scalars:
                self._init_scalars()
            self.io_write_4()
        else:
            self.itime = c.itmin
            path = os.path.join(self.wd, restart_name(self.run_name, c.itmin))
            # the header is checked on the host first, so that a bad file is
            # reported by name before anything reaches the device
            read_restart_header(path, c.nx)
            with open(path, "rb") as fh:
                self.time, dt, nums1, _ = self.ctx.restart_load(np.frombuffer(fh.read(), dtype=np.uint8))
            # scalars the .in file has beyond the file's count start from their
            # initial condition (restart_io.f90:419-432)
            for s in range(min(nums1, c.n_scalars), c.n_scalars):
                self.ctx.init_scalar(s, c.rn2, c.peak_wavenum_sc[s])
            if nums1 > 0 or c.tscalar <= self.time:
                self.int_scalars = c.n_scalars > 0
            if c.variable_dt:
                c.dt = 0.5 * dt
                self.ctx.set_dt(c.dt)
        self.ctx.set_scalars_active(self.int_scalars)
        self.ctx.fov = self.ctx.fos = 1
        self.ctx.dealias_all()
        if self.settings.variant is None:
            self.ctx.autotune()

    def _init_scalars(self):
        """init_scalars (init_scalars.f90:1-35): every passive scalar from RN2 by its type."""
        for s in range(self.cfg.n_scalars):
            self.ctx.init_scalar(s, self.cfg.rn2, self.cfg.peak_wavenum_sc[s])

    # -- particles (m_particles.f90) -------------------------------------------
    def _particles_start(self):
        """particles_init: pt.<ext> of the restart step, else <run_name>.pt, else the lattice;
        uploaded once TIME reaches starttime_particles (m_fields.f90:239-247)."""
        c = self.cfg
        n = c.nx
        pt = os.path.join(self.wd, f"pt.{c.itmin:06d}")
        if c.itmin > 0 and os.path.exists(pt):
            self.ipart, grid, _ = _pt.read_pt(pt, n)
        else:
            own = os.path.join(self.wd, self.run_name + ".pt")
            if os.path.exists(own):
                phys = _pt.read_run_pt(own, c.nptot)
                self.ipart = np.arange(1, c.nptot + 1, dtype=np.int32)
            else:
                self.ipart, phys = _pt.lattice(c.nptot, n)
            grid = _pt.to_grid(phys, n)
        self.ctx.particles_upload(grid, None, c.particles_tracking_scheme)
        if c.particles_filter_size > 0.0:
            self.ctx.particles_filter(c.particles_filter_size)
        self.int_particles = True

    def write_particles(self):
        """particles_restart_write_binary: pt.<ext>, with the 'parts' task's TIME, the
        time at the start of the step that moved the particles last (the hydro
        task hands it over before advancing, main.f90:124-128, 166-167)."""
        grid, _ = self.ctx.particles_download()
        _pt.write_pt(os.path.join(self.wd, f"pt.{self.file_ext()}"), self.ipart, grid, self.cfg.nx,
                     self.particles_time)

    # -- outputs ---------------------------------------------------------------
    def file_ext(self):
        return f"{self.itime:06d}"

    def io_write_4(self):
        c = self.cfg
        nout = 3 + (c.n_scalars if self.int_scalars else 0)
        phys = self.ctx.physical_fields(nout, float(c.kmax) ** 2)
        names = ["u", "v", "w"] + [f"sc{n + 1:02d}" for n in range(nout - 3)]
        for n, nm in enumerate(names):
            write_real4(os.path.join(self.wd, f"{nm}.{self.file_ext()}"), phys[n])

    @property
    def n_les(self) -> int:
        """LES-related transported fields of the dynamic localization models."""
        return les_fields(self.cfg.les_model)

    def write_restart(self):
        """restart_write_parallel: the file image is packed on the device
        (hit3d_gpu_restart_pack) and written as is, through a temporary name."""
        nums = self.cfg.n_scalars if self.int_scalars else 0
        path = os.path.join(self.wd, restart_name(self.run_name, self.itime))
        img = self.ctx.restart_image(self.time, self.cfg.dt, nums)
        with open(path + ".part", "wb") as f:
            f.write(img.tobytes())
        os.replace(path + ".part", path)

    def stat_main(self):
        es, st = self.ctx.stats()
        wd, it, t = self.wd, self.itime, self.time

        def append(name, header, line):
            path = os.path.join(wd, name)
            new = not os.path.exists(path)
            with open(path, "a") as fh:
                if new and header:
                    fh.write(header + "\n")
                fh.write(line + "\n")

        append("stat1.gp", " # 1.itime 2.time         3.energy       4.diss         5.eta          6.enstrophy    7.R_lambda",
               f"{it:8d}" + "".join(_fmt_e(x) for x in (t, st["energy"], st["eps_v"], st["eta"], st["enstrophy"],
                                                         st["re_lambda"])))
        append("stat2.gp", "# 1.itime  2.time         3.int LS       4. lambda      5.R_lambda1    6.tau_e        7.etakmax",
               f"{it:8d}" + "".join(_fmt_e(x) for x in (t, st["x_length"], st["lambda"], st["re_lambda1"],
                                                         st["tau_e"], st["etakmax"])))
        e1 = es * np.arange(1, len(es) + 1) ** 2 * 2.0 * self.cfg.nu
        with open(os.path.join(wd, "es.gp"), "a") as fh:
            fh.write("\n\n" + f"# ITIME={it:7d} TIME={_fmt_e(t, 17, 8)}\n")
            for k in range(len(es)):
                fh.write(f"{k + 1:4d}{_fmt_e(es[k])}{_fmt_e(e1[k])}\n")
        if self.int_scalars:
            for s in range(self.cfg.n_scalars):
                ss = self.ctx.scalar_stats(s)
                append(f"sc{s + 1:02d}.gp",
                       "# 1.itime 2.time          3.sc.diss       4. mean      5.variance    6.min     7.max",
                       f"{it:7d}" + "".join(_fmt_e(x) for x in (t, ss["diss"], ss["mean"], ss["variance"], ss["min"],
                                                                ss["max"])))
                with open(os.path.join(wd, f"es_{s + 1:02d}.gp"), "a") as fh:
                    fh.write("\n\n" + f"# ITIME={it:7d} TIME={_fmt_e(t, 17, 8)}\n")
                    for k, v in enumerate(ss["spectrum"]):
                        fh.write(f"{k + 1:4d}{_fmt_e(v)}\n")
        return es, st

    def _les_gp(self, it, t):
        """les.gp (m_les.f90:876-892): itime, the time at the start of the step,
        mean k_sgs, production, B and dissipation of that step's RHS."""
        ls = self.ctx.les_stats()
        vals = (t, ls["energy"], ls["production"], ls["B"], ls["dissipation"])
        with open(os.path.join(self.wd, "les.gp"), "a") as fh:
            fh.write(f"{it:6d} " + "".join(_fmt_e(x) for x in vals) + "\n")

    # -- time step control (my_dt.f90) ------------------------------------------
    def my_dt(self, courant):
        c = self.cfg
        courant_max = 0.1
        if c.flow_type <= 1:
            if courant < courant_max:
                c.dt = min(c.dt * 1.01, 0.01)
            else:
                c.dt = c.dt / 1.05
            if self.int_scalars and courant > 0.0:
                for s in c.sc:
                    c.dt = min(c.dt, c.dt * courant_max / courant / s)
        self.ctx.set_dt(c.dt)

    # -- main cycle (main.f90:87-288) -------------------------------------------
    def run(self, max_steps: int | None = None):
        c = self.cfg
        last = c.itmax if max_steps is None else min(c.itmax, self.itime + max_steps)
        while self.itime < last:
            self.itime += 1
            it = self.itime
            t = self.time
            if c.flow_type == 0 and c.trescale > 0.0 and \
                    math.floor((t - c.dt) / c.trescale) < math.floor(t / c.trescale):
                if math.floor(t / c.trescale) <= c.nrescale and it != 1:
                    self.ctx.velocity_rescale(c.isp_type, c.peak_wavenum, float(c.ir_exp))
                    self.ctx.fov = self.ctx.fos = 1
                    if it % c.iprint1 == 0:
                        self.stat_main()
            if c.nptot > 0 and not self.int_particles and t >= c.starttime_particles:
                self._particles_start()
            courant = self.ctx.step(1)
            self.particles_time = t
            if self.int_particles and len(self.ipart) < 1000:
                grid, uvw = self.ctx.particles_download()
                _pt.append_trajectories(self.wd, it, t, self.ipart, grid, uvw, c.nx)
            if self.int_particles and it % c.iwrite4 == 0:
                self.write_particles()
            if self.n_les > 0 and it % c.iprint1 == 0:
                self._les_gp(it, t)
            self.time += c.dt
            if not math.isfinite(courant) or \
                    (self.settings.nonfinite_check and it % c.iprint1 == 0 and self.ctx.nonfinite() > 0):
                self._out(f"ITIME={it:6d}   non-finite state")
                return self.exit(-2)
            if it % c.iprint2 == 0:
                self.write_restart()
            if c.variable_dt:
                self.my_dt(courant)
            if it % c.iprint1 == 0:
                el = int(_time.time() - self.t0)
                sym = "*" if it % c.iwrite4 == 0 else " "
                self._out(f"ITIME={it:6d}   TIME={self.time:8.4f}    DT={c.dt:8.5f}   Courn= {courant:6.4f}  "
                          f"CPU:({el // 3600:04d}:{el // 60 % 60:02d}:{el % 60:02d}) {sym} "
                          f"{LES_MODEL_NAME.get(c.les_model, '   ')}")
            if it % c.iprint1 == 0 or it % c.iwrite4 == 0:
                if self.time > c.tmax:
                    return self.exit(1)
                if c.n_scalars > 0 and not self.int_scalars and self.time > c.tscalar:
                    self.int_scalars = True
                    self._init_scalars()
                    self.ctx.set_scalars_active(True)
                if it % c.iprint1 == 0:
                    self.stat_main()
                if it % c.iwrite4 == 0:
                    self.io_write_4()
            if it % 10 == 0:
                if (_time.time() - self.t0) / 60.0 + 5 > self.job_runlimit:
                    return self.exit(2)
                if os.path.exists(os.path.join(self.wd, "stop")):
                    return self.exit(3)
        if max_steps is None or self.itime >= c.itmax:
            return self.exit(0)
        return None

    def exit(self, reason: int):
        """my_exit: a restart file is written for every reason >= 0."""
        self.exit_reason = reason
        self._out(f"my_exit with reason {reason:4d}")
        if reason >= 0:
            self.write_restart()
            if self.int_particles:
                self.write_particles()
        return reason


def main(argv=None):
    """`python -m hit3d_b200.driver <run_name> [--workdir D] [--precision 0|1] [--device I]`:
    read <run_name>.in and <run_name>.gpu.in, run to ITMAX/TMAX/stop/runlimit,
    write the reference's files.  --precision and --device override the .gpu.in file."""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("run_name")
    ap.add_argument("--workdir", default=".")
    ap.add_argument("--precision", type=int, choices=(0, 1), default=None)
    ap.add_argument("--device", type=int, default=None)
    a = ap.parse_args(argv)
    sim = Simulation(a.run_name, workdir=a.workdir, precision=a.precision, device=a.device)
    sim.begin()
    reason = sim.run()
    print(f"exit reason {reason} at ITIME={sim.itime}, TIME={sim.time:.6f}")
    return 0 if reason is not None and reason >= 0 else 1


if __name__ == "__main__":
    raise SystemExit(main())
