#!/usr/bin/env python
"""Benchmark of the HIT3DP pseudospectral timestep on B200.

Workload: forced DNS on a 512^3 grid (flow_type=1, Machiels band forcing KFMAX=2,
FAMP=0.5), Re = 3000, fixed dt, 2/3-rule dealiasing, FP64 spectral state, no
scalars or particles; initial velocity from the reference's RANDu/Box-Muller
generator (RN1 of scripts/00_example.in) shaped to E(k) ~ k^2 exp(-2 (k/4)^2).
Data are synthetic (generated in place); every field is ~1.1 GB, far larger than
the 126 MB L2, so no flush is needed between steps.

`value` = timesteps/s of the FP64 path with the state resident in HBM, timed
with CUDA events on the library's stream; `e2e` = the same through the C-ABI
with the host owning the fields (pinned host -> device upload, step, device ->
host download every step).  The FP32-nonlinear-term form is timed on the same
initial state and its E(k) is compared with the FP64 run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun (N > 1) every rank advances its own independent replica (the
single-GPU path does not shard); value = all ranks' steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 512
RE = 3000.0
DT = 0.0002  # Courant number about 0.1 in the developed flow, as the reference keeps it (my_dt.f90)
RN1 = 67748937.0
METRIC = "timesteps/s at 512^3 FP64 (forced DNS, 2/3 rule)"


def metric_name(n: int) -> str:
    """The headline metric, named for the grid actually run."""
    return METRIC.replace("512^3", f"{n}^3")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--e2e-steps", type=int, default=24,
                    help="host-buffer steps of the e2e leg (the pipeline fills and drains once per call)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-transform form")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-les", action="store_true", help="skip the learned-LES leg")
    ap.add_argument("--les-full", action="store_true",
                    help="a-posteriori test at 512^3 DNS -> 128^3 LES (minutes) instead of 128^3 -> 32^3")
    ap.add_argument("--les-only", action="store_true", help="only the learned-LES step rates (profiling runs)")
    ap.add_argument("--no-configs", action="store_true", help="skip the step rates of the other configurations")
    ap.add_argument("--configs-only", action="store_true", help="only the step rates of the other configurations")
    ap.add_argument("--config", default=None, choices=CONFIG_NAMES, help="with --configs-only: just this configuration")
    ap.add_argument("--config-steps", type=int, default=0, help="timed steps of --config forced_256 (default 20)")
    ap.add_argument("--cmp-every", type=int, default=50, help="FP32 vs FP64 statistics every this many steps")
    ap.add_argument("--cmp-points", type=int, default=10)
    ap.add_argument("--variant", type=int, default=-1,
                    help="fix the fused x-pass launch shape instead of tuning (profiling runs)")
    ap.add_argument("--update-fusion", type=int, default=-1, choices=(-1, 0, 1),
                    help="fuse the products' z pass with the update (1) or not (0); -1: the library default")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_context(n, precision, device):
    from hit3d_b200 import Context, Params
    p = Params(nx=n, dealias=0, flow_type=1, force_type=1, kfmax=2, famp=0.5, nu=1.0 / RE, dt=DT,
               precision=precision, device=device)
    return Context(p)


def stage_units(n, precision, pruned, fused=False):
    """Algorithmic bytes per step of each stage, in units of one unpadded complex
    half-spectrum field B1 = N^2 (N/2+1) * 16 bytes, velocity only, 2/3 rule.

    With 2/3-rule pruning a = (kc+1)/(N/2+1) of the kx columns and b = (2 kc+1)/N of
    the ky (or kz) indices are kept (kc = N/3): inverse passes read only kept
    indices along their axis and forward passes store only kept indices, and the
    update visits only the kept modes (a b^2).  Unpruned, the update still reads
    the products only at kept modes.  Work
    fields are half size in the FP32 form; the state stays FP64."""
    kc = n // 3
    a0, b0 = (kc + 1) / (n // 2 + 1), (2 * kc + 1) / n
    a, b = (a0, b0) if pruned else (1.0, 1.0)
    w = 0.5 if precision else 1.0
    return {
        "z_inverse": 3 * a * b * b + w * 3 * a * b,
        "y_inverse": w * (3 * a * b + 3 * a),
        "x_fused": w * (3 * a + 6 * a),
        "y_forward": w * (6 * a + 6 * a * b),
        "z_forward": w * (6 * a * b + 6 * a * b * b),
        # U, RO read and written, products read: at the kept modes only when pruned
        "update": (12 if not pruned else 12 * a0 * b0 * b0) + w * 6 * a0 * b0 * b0,
    } if not fused else {
        "z_inverse": 3 * a * b * b + w * 3 * a * b,
        "y_inverse": w * (3 * a * b + 3 * a),
        "x_fused": w * (3 * a + 6 * a),
        "y_forward": w * (6 * a + 6 * a * b),
        # the products' z pass inside the update kernel: products read along all z
        # (kept kx and ky), U and RO read and written at the kept modes
        "z_forward": 0.0,
        "update": w * 6 * a * b + (12 if not pruned else 12 * a0 * b0 * b0),
    }


def load_traffic():
    """Per-launch DRAM bytes of the dominant stage from the committed ncu summary."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.txt")) as f:
            for line in f:
                line = line.split("#")[0].split()
                if len(line) == 2:
                    out[line[0]] = float(line[1])
    except OSError:
        pass
    return out
# single launches per step of each stage (velocity only, 2/3 rule)
STAGE_LAUNCHES = {"z_inverse": 1, "y_inverse": 1, "x_fused": 1, "y_forward": 1, "z_forward": 1, "update": 1}




def timed_steps(torch, ctx, steps):
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    ctx.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1000.0


def host_cpu():
    """CPU model, physical cores and the threads this process may use."""
    model, cores = None, set()
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None and core is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None and core is not None:
            cores.add((phys, core))
    except OSError:
        pass
    try:
        threads = len(os.sched_getaffinity(0))
    except AttributeError:
        threads = os.cpu_count() or 1
    return {"cpu_model": model, "physical_cores": len(cores) or None, "threads": threads}


def oracle_run(n):
    """The oracle (C/OpenMP FP64 restatement of the reference step) on the host,
    initialised as the GPU run is: RANDu/Box-Muller from RN1, E(k) ~ k^2 exp(-2(k/4)^2)."""
    import oracle
    o = oracle.Oracle(n, nscal=0, dealias=0, flow_type=1, kfmax=2, nu=1.0 / RE, dt=DT, famp=0.5)
    o.init_velocity(RN1, isp_type=2, peak_wavenum=4.0, ir_exp=2.0)
    o.dealias_all()
    return o


def cpu_sample(n, warm=1, timed=2, budget_s=240.0):
    """Time the oracle at the workload's own grid: `warm` untimed steps (the first
    one is the first-order step), then up to `timed` steps, fewer only if the
    warm-up step says they would take longer than budget_s."""
    hc = host_cpu()
    o = oracle_run(n)
    t0 = time.perf_counter()
    o.step(max(1, warm))
    t_warm = (time.perf_counter() - t0) / max(1, warm)
    k = max(1, min(timed, int(budget_s / max(t_warm, 1e-9))))
    t0 = time.perf_counter()
    o.step(k)
    el = time.perf_counter() - t0
    del o
    return {"value": k / el, "unit": "timesteps/s", "cores": hc["threads"], "kind": "port",
            "cpu_model": hc["cpu_model"], "physical_cores": hc["physical_cores"], "steps_timed": k,
            "seconds": round(el, 2),
            "sample": f"{k} oracle steps at {n}^3 after {max(1, warm)} warm-up (OpenMP on {hc['threads']} threads of "
                      f"{hc['physical_cores']} physical cores, {hc['cpu_model']})"}


def les_leg(torch, args, dns_rate, dns32_rate, device):
    """Learned-closure LES at 128^3 against the 512^3 DNS: step rates, the
    simulated-time speedup at equal Courant number (dt_les = 4 dt_dns), and an
    a-posteriori spectrum test against filtered DNS."""
    from hit3d_b200 import Context, Params
    from hit3d_b200.les import LesExperiment, run_experiment
    from hit3d_b200 import gpu
    n_les, ratio = 128, 2.0
    dt_les = DT * args.n / n_les
    delta = ratio * 2.0 * np.pi / n_les
    out = {"grid": n_les, "dt_les": dt_les, "dt_dns": DT, "filter_width": delta}
    # step cost does not depend on the weight values: time with the Smagorinsky-
    # equivalent network g = (-2 Cs^2 dx^2 / Delta^2, 0, 0, 0, 0)
    nparam = int(gpu.lib().hit3d_mlp_nparam())
    w = np.zeros(nparam, dtype=np.float32)
    dx = 2.0 * np.pi / n_les
    w[nparam - 5] = -2.0 * 0.18 ** 2 * dx * dx / (delta * delta)
    bits = ((w.view(np.uint32).astype(np.uint64) + 0x7FFF + ((w.view(np.uint32) >> 16) & 1)) >> 16).astype(np.uint16)
    rates = {}
    # FP64 transforms, and the FP32-transform form (FP64 state and integrator)
    # with the learned closure and with Smagorinsky
    for name, model, kernel, prec in (("learned", 20, 1, 0), ("learned_cuda_cores", 20, 0, 0), ("smagorinsky", 1, 0, 0),
                                      ("learned_fp32_transforms", 20, 1, 1), ("smagorinsky_fp32_transforms", 1, 0, 1)):
        c = Context(Params(nx=n_les, dealias=0, flow_type=1, force_type=1, kfmax=2, famp=0.5, nu=1.0 / RE, dt=dt_les,
                           les_model=model, precision=prec, device=device))
        if model == 20:
            c.les_set_mlp(bits, delta, clip=True, kernel=kernel)
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        if args.variant >= 0:
            c.set_variant(args.variant)
        else:
            c.autotune()
        c.step(args.warmup)
        steps = max(args.steps, 50)
        t = timed_steps(torch, c, steps)
        rates[name] = steps / t
        if model == 20:
            prof = c.step_profile(3)
            out[name + "_stage_ms"] = {("closure" if k == "smagorinsky" else k): round(v / 3, 4)
                                       for k, v in prof.items() if v > 0}
        c.close()
    out["steps_per_s"] = rates
    if dns_rate:
        out["speedup_vs_dns_fp64"] = rates["learned"] * dt_les / (dns_rate * DT)
    if dns32_rate:
        out["speedup_vs_dns_fp32"] = rates["learned"] * dt_les / (dns32_rate * DT)
    if args.les_only:
        return out
    ex = (LesExperiment(n_dns=512, n_les=128, re=RE, dt_dns=0.00025, nruns=1, spinup=2.0, collect=0.5, nsnap=4,
                        window=1.0, nsample=5, stride=4, train_steps=2000) if args.les_full else
          LesExperiment(n_dns=128, n_les=32, re=1000.0, dt_dns=0.002, nruns=2, spinup=2.0, collect=1.0, nsnap=4,
                        window=1.5, nsample=6, stride=2, train_steps=1500))
    try:
        r = run_experiment(ex, device=device, log=lambda *a: None)
        out["aposteriori"] = {"dns_to_les": f"{ex.n_dns}^3 -> {ex.n_les}^3", "re": ex.re,
                              "mean_abs_log_spectrum_error": r["spectrum_error"],
                              "apriori_stress_error": r["apriori_stress_error"],
                              "speedup_vs_dns": r["speedup_vs_dns"]}
    except Exception as e:  # reported, never fatal to the bench line
        out["aposteriori"] = {"error": str(e)}
    return out


CONFIG_NAMES = ("decaying_64", "forced_256", "batched_96", "les_128")


def configs_leg(torch, args, device, only=None):
    """Step rates of the other configurations of the path (the per-configuration
    parity lives in tests/): 64^3 decaying; 256^3 forced with phase-shift
    dealiasing, two scalars and 10^6 CINT particles; the batched 96-run set;
    128^3 LES with each closure.  `only` runs one of CONFIG_NAMES."""
    from hit3d_b200 import Context, Params
    from hit3d_b200.batch import Batch, batched_runs
    out = {}

    def rate(c, steps):
        c.init_velocity(RN1, 2, 4.0, 2.0)
        c.dealias_all()
        if args.variant >= 0:
            c.set_variant(args.variant)
        else:
            c.autotune()
        c.step(args.warmup)
        t = timed_steps(torch, c, steps)
        return steps / t

    if only in (None, "decaying_64"):
        c = Context(Params(nx=64, dealias=0, flow_type=0, nu=1.0 / 400.0, dt=0.005, device=device))
        r = rate(c, 100)
        out["decaying_64"] = {"workload": "decaying DNS 64^3, Re=400, dt=0.005, 2/3 rule", "steps_per_s": r,
                              "grid_points_steps_per_s": r * 64 ** 3}
        c.close()

    if only in (None, "forced_256"):
        n = 256
        c = Context(Params(nx=n, dealias=1, flow_type=1, force_type=1, kfmax=2, famp=0.5, nu=1.0 / 1000.0, dt=0.001,
                           n_scalars=2, sc=[0.7, 1.0], scalar_type=[0, 0], device=device))
        c.set_scalars_active(True)
        # 100^3 = 10^6 particles on the reference's lattice of cell centres, in its
        # 1-based grid units (m_particles.f90:220-262, 314-319)
        g = (np.arange(100) + 0.5) * n / 100.0 + 1.0
        Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
        c.particles_upload(np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1), None, scheme=1)
        r = rate(c, args.config_steps or 20)
        prof = c.step_profile(2)
        out["forced_256"] = {
            "workload": "forced DNS 256^3, Re=1000, dt=0.001, phase shift, 2 scalars (Sc 0.7, 1.0), 10^6 CINT particles",
            "steps_per_s": r, "grid_points_steps_per_s": r * n ** 3,
            "stage_ms": {k: round(v / 2, 4) for k, v in prof.items() if v > 0}}
        c.close()

    if only in (None, "batched_96"):
        ps = batched_runs()
        b = Batch(ps)
        b.init()
        picks = b.autotune()
        # first-order step, then one chunk through the graph, so that the timed
        # region replays a graph recorded beforehand
        b.step(1 + 10, graph_steps=10)
        b.step(args.warmup, graph_steps=10)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.step(50, graph_steps=10)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        pts = sum(p.nx ** 3 for p in ps)
        out["batched_96"] = {"workload": "96 forced runs: 32 x 32^3, 32 x 48^3, 28 x 64^3, 4 x 128^3, one recorded graph",
                             "run_steps_per_s": len(ps) * 50 / t, "grid_points_steps_per_s": pts * 50 / t,
                             "size_classes": b.nclasses,
                             "tuned": [{"variant": v, "tile": tl, "x_ms": [round(x, 4) for x in mv],
                                        "columns_ms": [round(x, 4) for x in mt]} for v, tl, mv, mt in picks],
                             "graph_launches": b.graph_launches, "timing": "host clock around 50 steps (5 graph launches)"}
        b.close()

    if only in (None, "les_128"):
        les = {}
        for name, model in (("smagorinsky", 1), ("dynamic_localization", 2), ("dynamic_localization_lag", 3),
                            ("dynamic_structure", 4), ("dynamic_structure_lag", 5), ("mixed", 6), ("mixed_lag", 7),
                            ("one_equation_mixed", 10), ("learned", 20)):
            # C_T and C_mixed stand in for the values of c_t.in / c_mixed.in
            c = Context(Params(nx=128, dealias=0, flow_type=1, force_type=1, kfmax=2, famp=0.5, nu=1.0 / 6000.0,
                               dt=0.002, les_model=model, device=device, c_t=1.0, c_mixed=0.5))
            if model == 20:
                from hit3d_b200 import gpu
                nparam = int(gpu.lib().hit3d_mlp_nparam())
                w = np.zeros(nparam, dtype=np.float32)
                w[nparam - 5] = -2.0 * 0.18 ** 2 / 4.0
                bits = ((w.view(np.uint32).astype(np.uint64) + 0x7FFF + ((w.view(np.uint32) >> 16) & 1)) >> 16).astype(np.uint16)
                c.les_set_mlp(bits, 2 * 2.0 * np.pi / 128, clip=True, kernel=1)
            les[name] = rate(c, 50)
            c.close()
        out["les_128"] = {"workload": "LES 128^3, Re=6000, 2/3 rule", "steps_per_s": les}
    return out


def workload_name(n):
    return (f"forced DNS {n}^3, Re={RE:g}, dt={DT}, 2/3 rule, KFMAX=2, FAMP=0.5, "
            "E(k)~k^2 exp(-2(k/4)^2) RANDu init")


def run_reference(args):
    """The CPU implementation of the step (the oracle port: the reference itself
    needs a Fortran/MPI/FFTW toolchain that these machines lack) on this host's
    cores, on the same workload; one step of the arm is one oracle step."""
    rank, world, _ = dist_info()
    if rank != 0:
        return
    cs = cpu_sample(args.n, warm=args.warmup, timed=args.steps, budget_s=300.0)
    line = {"impl": "reference", "metric": metric_name(args.n), "value": cs["value"], "unit": "timesteps/s",
            "n_gpus": args.gpus, "steps": cs["steps_timed"], "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args.n), "grid": args.n},
            "cpu_baseline": cs,
            "e2e": {"value": cs["value"], "unit": "timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _sig(x, d=4):
    """Round floats to d significant digits, recursively."""
    if isinstance(x, float):
        return float(f"{x:.{d}g}")
    if isinstance(x, dict):
        return {k: _sig(v, d) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_sig(v, d) for v in x]
    return x


def max_over_ranks(dist, t, device="cuda"):
    """The job's time: the largest of every rank's t (seconds), by one
    all_reduce(MAX) of the timing scalar (dist None: one process, t itself).
    device: where the scalar lives for the backend (cuda for NCCL, cpu for gloo)."""
    if not dist:
        return t
    import torch
    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def ek_err_by_decade(e32, e64):
    """Largest relative E(k) error of the FP32 form per band of shells, banded by
    the shell's energy over the peak shell's: [1e-2, 1], [1e-4, 1e-2], ...,
    [1e-12, 1e-10]; None for a band without shells."""
    r = e64 / e64.max()
    rel = np.abs(e32 - e64) / np.where(e64 > 0, e64, 1.0)
    out = {}
    for d in range(0, 12, 2):
        m = (r <= 10.0 ** -d) & (r > 10.0 ** -(d + 2))
        out["1e-%d" % (d + 2)] = float(rel[m].max()) if m.any() else None
    return out


def summarize(line):
    """Compact summary of the bench line: the headline, the FP32 form, the
    other configurations, the learned LES and the CPU baseline."""
    s = {"fp64_steps_per_s": line["value"], "ms_per_step": line["ms_per_step"],
         "roofline_frac": line["roofline"]["frac"], "roofline_kernel": line["roofline"]["kernel"],
         "e2e_steps_per_s": (line.get("e2e") or {}).get("value"),
         "e2e_full_arrays_steps_per_s": ((line.get("e2e") or {}).get("full_arrays") or {}).get("value")}
    f = line.get("fp32_fft")
    if f:
        s["fp32"] = {"steps_per_s": f["value"], "speedup_vs_fp64": f["speedup_vs_fp64"],
                     "ek_max_rel_err_over_run": f.get("ek_max_rel_err_over_run"),
                     "ek_1e-4_crossed_at_step": f.get("ek_1e-4_crossed_at_step"),
                     "ek_max_rel_err_above_1e-6_over_run": f.get("ek_max_rel_err_above_1e-6_over_run"),
                     "ek_max_rel_err_above_1e-10_over_run": f.get("ek_max_rel_err_above_1e-10_over_run"),
                     "per_step": [[c["step"], c["ek_max_rel_err"], c["eps_rel_err"], c["skew_abs_err"]]
                                  for c in f.get("vs_fp64_every_%d_steps" % 50, [])]}
    oc = line.get("other_configs") or {}
    if "error" in oc:
        s["configs_error"] = oc["error"]
    for k, v in oc.items():
        if isinstance(v, dict) and "steps_per_s" in v and not isinstance(v["steps_per_s"], dict):
            s[k] = v["steps_per_s"]
    if "batched_96" in oc:
        b = oc["batched_96"]
        s["batched_96"] = {"run_steps_per_s": b["run_steps_per_s"],
                                "grid_points_steps_per_s": b["grid_points_steps_per_s"]}
    if "les_128" in oc:
        s["les_128_steps_per_s"] = oc["les_128"]["steps_per_s"]
    le = line.get("learned_les")
    if le:
        s["learned_les"] = {"steps_per_s": le.get("steps_per_s"),
                            "closure_ms": (le.get("learned_stage_ms") or {}).get("closure"),
                            "closure_ms_fp32_transforms": (le.get("learned_fp32_transforms_stage_ms") or {}).get("closure"),
                            "speedup_vs_dns_fp64": le.get("speedup_vs_dns_fp64")}
        ap = le.get("aposteriori") or {}
        if "mean_abs_log_spectrum_error" in ap:
            s["learned_les"]["aposteriori"] = {"case": ap["dns_to_les"], "error": ap["mean_abs_log_spectrum_error"]}
    c = line.get("cpu_baseline") or {}
    s["cpu_baseline_steps_per_s"] = c.get("value")
    return _sig(s)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if args.les_only:
        print(json.dumps({"learned_les": les_leg(torch, args, None, None, local)}), flush=True)
        return
    if args.configs_only:
        print(json.dumps({"other_configs": configs_leg(torch, args, local, only=args.config)}), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n = args.n
    B1 = n * n * (n // 2 + 1) * 16.0
    peak, peak_kind = peaks()

    ctx = make_context(n, 0, local)
    if args.update_fusion >= 0:
        ctx.set_update_fusion(bool(args.update_fusion))
    ctx.init_velocity(RN1, 2, 4.0, 2.0)
    ctx.dealias_all()
    fields0 = ctx.download_fields()
    if args.variant >= 0:
        ctx.set_variant(args.variant)
        variant, variant_ms = args.variant, []
    else:
        variant, variant_ms = ctx.autotune()

    # warm-up, then the timed region
    ctx.step(args.warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    with ClockSampler(local) as clk:
        t = timed_steps(torch, ctx, args.steps)
    launches = ctx.launches - launches0
    t = max_over_ranks(dist, t)
    value = world * args.steps / t
    ms = 1000.0 * t / args.steps
    es64, st64 = ctx.stats()

    # per-stage device time (separate, untimed steps) -> roofline of the dominant stage
    pruned = ctx.pruned
    prof = ctx.step_profile(3)
    prof = {k: v / 3 for k, v in prof.items()}
    units = stage_units(n, 0, pruned, fused=args.update_fusion == 1)
    top = max(units, key=lambda k: prof.get(k, 0.0))
    ach = units[top] * B1 / (prof[top] / 1000.0) / 1e9
    traffic = load_traffic().get(f"{n}:{top}")
    stage_gbs = {k: round(units[k] * B1 / (prof[k] / 1000.0) / 1e9, 1) for k in units if prof.get(k, 0) > 0}
    ideal = 240.0 * n ** 3  # bytes per step of the ideal single-pass model
    # e2e through the C-ABI with host-owned fields
    e2e = None
    if not args.no_e2e:
        h = torch.empty(fields0.size, dtype=torch.float64).pin_memory()
        hv = h.numpy().reshape(fields0.shape)
        hv[:] = fields0
        ho = torch.empty(fields0.size, dtype=torch.float64).pin_memory()
        hov = ho.numpy().reshape(fields0.shape)
        # warm-up of the pipelined path (staging buffers and copy streams); the
        # full download also leaves hov zero outside the 2/3-rule band
        ctx.step_host([hv], [hov], nsteps=1)
        stream = torch.cuda.ExternalStream(ctx.stream)

        def e2e_time(band_only):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            # every step: upload of that step's fields from pinned host memory,
            # the step, download of the new state; the next upload overlaps this
            # step and download (hit3d_gpu_step_host)
            ctx.step_host([hv] * args.e2e_steps, [hov] * args.e2e_steps, nsteps=1, band_only=band_only)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / 1000.0

        te_full = e2e_time(False)
        te = e2e_time(True)
        out = hov
        te = max_over_ranks(dist, te)
        te_full = max_over_ranks(dist, te_full)
        nbytes = ctx.step_host_bytes(3, True)
        e2e = {"value": world * args.e2e_steps / te, "unit": "timesteps/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": args.e2e_steps,
               "api": "hit3d_gpu_step_host, reference-layout host fields, band_only: the 2/3-rule band "
                      "(every |k_i| <= N/3) crosses PCIe, uploads overlapping downloads",
               "full_arrays": {"value": world * args.e2e_steps / te_full, "h2d_bytes_per_step": fields0.nbytes,
                               "d2h_bytes_per_step": fields0.nbytes}}
        del out

    # the FP64 trajectory for the per-statistic comparison, recorded before the
    # FP32 context is created so that only one context is resident at a time
    # (1024^3 does not hold both)
    ref_traj = []
    if not args.no_fp32:
        ctx.upload_fields(fields0)
        ctx.fov = ctx.fos = 1
        for k in range(args.cmp_points):
            ctx.step(args.cmp_every)
            ref_traj.append(ctx.stats())
    ctx.close()

    # FP32 nonlinear-term transforms, same initial state and step count
    fp32 = None
    if not args.no_fp32:
        c32 = make_context(n, 1, local)
        if args.update_fusion >= 0:
            c32.set_update_fusion(bool(args.update_fusion))
        c32.upload_fields(fields0)
        if args.variant >= 0:
            c32.set_variant(args.variant)
            v32, v32_ms = args.variant, []
        else:
            v32, v32_ms = c32.autotune()
        tile32, tile32_ms = getattr(c32, "column_tile", 0), getattr(c32, "column_ms", [])
        c32.step(args.warmup)
        if dist:
            dist.barrier()
        t32 = timed_steps(torch, c32, args.steps)
        t32 = max_over_ranks(dist, t32)
        es32, st32 = c32.stats()
        prof32 = c32.step_profile(3)
        mask = es64 > 1e-12 * es64.max()
        ek_err = float(np.max(np.abs(es32[mask] - es64[mask]) / es64[mask]))
        fp32 = {"value": world * args.steps / t32, "unit": "timesteps/s", "speedup_vs_fp64": (world * args.steps / t32) / value,
                "ek_max_rel_err_vs_fp64": ek_err, "eps_rel_err": abs(st32["eps_v"] - st64["eps_v"]) / st64["eps_v"],
                "skew_abs_err": abs(st32["skewness"] - st64["skewness"]),
                "stage_ms": {k: round(v / 3, 3) for k, v in prof32.items() if v > 0},
                "tuned_variant": v32, "variant_ms": [round(x, 3) for x in v32_ms],
                "column_tile": tile32, "column_ms": [round(x, 3) for x in tile32_ms]}
        # error per statistic against the FP64 path every cmp_every steps from the same state
        c32.upload_fields(fields0)
        c32.fov = c32.fos = 1
        cmp = []
        for k, (e64, s64) in enumerate(ref_traj):
            c32.step(args.cmp_every)
            e32, s32 = c32.stats()
            mk = e64 > 1e-12 * e64.max()
            rel = np.abs(e32 - e64) / np.where(e64 > 0, e64, 1.0)
            mk6 = e64 > 1e-6 * e64.max()
            cmp.append({"step": (k + 1) * args.cmp_every,
                        "ek_max_rel_err": float(np.max(rel[mk])),
                        # shells holding at least 1e-6 of the peak shell's energy
                        "ek_max_rel_err_above_1e-6": float(np.max(rel[mk6])),
                        "worst_shell": int(np.argmax(np.where(mk, rel, -1.0))) + 1,
                        "ek_err_by_decade": ek_err_by_decade(e32, e64),
                        "energy_rel_err": abs(s32["energy"] - s64["energy"]) / s64["energy"],
                        "eps_rel_err": abs(s32["eps_v"] - s64["eps_v"]) / s64["eps_v"],
                        "skew_abs_err": abs(s32["skewness"] - s64["skewness"]),
                        "courant": c32.courant})
        fp32["vs_fp64_every_%d_steps" % args.cmp_every] = cmp
        fp32["ek_max_rel_err_over_run"] = max(c["ek_max_rel_err"] for c in cmp) if cmp else None
        # the first compared step at which the E(k) error passes 1e-4 (None: not within the run)
        fp32["ek_1e-4_crossed_at_step"] = next((c["step"] for c in cmp if c["ek_max_rel_err"] > 1e-4), None)
        fp32["ek_max_rel_err_above_1e-6_over_run"] = max(c["ek_max_rel_err_above_1e-6"] for c in cmp) if cmp else None
        # every shell holding at least 1e-10 of the peak shell's energy
        fp32["ek_max_rel_err_above_1e-10_over_run"] = max(
            (v for c in cmp for k, v in c["ek_err_by_decade"].items() if k != "1e-12" and v is not None),
            default=None)
        c32.close()

    les = None
    if not args.no_les and world == 1:
        les = les_leg(torch, args, value, fp32["value"] if fp32 else None, local)
    configs = None
    if not args.no_configs and world == 1:
        try:
            configs = configs_leg(torch, args, local)
        except Exception as e:  # reported, never fatal to the bench line
            configs = {"error": str(e)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_sample(n)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "error": str(e)}

    if rank == 0:
        line = {
            "metric": metric_name(n), "value": value, "unit": "timesteps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(n),
                       "grid": n, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs > L2 (1.1 GB per field), no flush"},
            "grid_points_steps_per_s": value * n ** 3,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": top, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": units[top] * B1, "pruned_transforms": pruned},
            "step_roofline": {"ideal_bytes_per_step": ideal, "achieved_GBs": ideal / (ms / 1000.0) / 1e9,
                              "frac_of_peak": ideal / (ms / 1000.0) / 1e9 / peak,
                              "stage_model_bytes_per_step": sum(units.values()) * B1,
                              "stage_model_GBs": sum(units.values()) * B1 / (ms / 1000.0) / 1e9,
                              "stage_model_frac_of_peak": sum(units.values()) * B1 / (ms / 1000.0) / 1e9 / peak},
            "stage_ms": {k: round(v, 3) for k, v in prof.items() if v > 0},
            "stage_GBs": stage_gbs,
            "tuned_variant": variant, "variant_ms": [round(x, 3) for x in variant_ms],
            "column_tile": getattr(ctx, "column_tile", 0),
            "column_ms": [round(x, 3) for x in getattr(ctx, "column_ms", [])],
            "clocks": clk.summary(),
            "e2e": e2e,
            "fp32_fft": fp32,
            "learned_les": les,
            "other_configs": configs,
            "cpu_baseline": cpu,
        }
        # the figures a reader needs first, last on the line (a log tail keeps them)
        line["summary"] = summarize(line)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
