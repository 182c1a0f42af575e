"""Learned LES closure: training data from box-filtered DNS generated by the
batched form, training on the GPU, and the a-posteriori comparison of LES
spectra (learned closure, Smagorinsky, no model) against filtered DNS.

The reference has Smagorinsky (m_les.f90:1142-1215) and other eddy-viscosity
models; the learned closure has no counterpart there.  The exact subgrid stress
follows the Leonard-type form tau_ij = filter(u_i u_j) - filter(u_i) filter(u_j)
of m_les.f90:1847-1865.
"""
from __future__ import annotations

import time
from dataclasses import asdict, dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .batch import Batch, run_seed
from .gpu import LES_LEARNED, Context, Mlp, Params

PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
FROB = np.array([1.0, 2.0, 2.0, 1.0, 2.0, 1.0])


def sgs_samples(ctx: Context, delta: float, stride: int = 1, kind: int = 4):
    """Filtered gradients A (9, P) and exact stresses tau (6, P) of the current state,
    on every `stride`-th point per axis."""
    sub = ctx.sgs_samples(kind, delta, stride).reshape(18, -1)
    return np.ascontiguousarray(sub[9:18]), np.ascontiguousarray(sub[3:9])


def spectral_truncate(fields: np.ndarray, n_to: int) -> np.ndarray:
    """Fourier fields (nf, N, N, N+2) in the reference layout ([ky][kz][kx re/im]) of
    an N^3 run onto an n_to^3 grid: modes with |k_i| < n_to/2, rescaled for the
    unnormalised transform."""
    nf, N = fields.shape[0], fields.shape[1]
    n = int(n_to)
    if n > N:
        raise ValueError("can only truncate to a coarser grid")
    out = np.zeros((nf, n, n, n + 2))
    ks = np.arange(-(n // 2 - 1), n // 2)
    src, dst = ks % N, ks % n
    scale = (n / N) ** 3
    kx = n // 2  # complex kx columns 0..n/2-1 -> reals 0..n-1
    blk = fields[:, src][:, :, src][..., : 2 * kx]
    out[:, dst[:, None], dst[None, :], : 2 * kx] = blk * scale
    return out


def filtered_state(fields: np.ndarray, scratch: Context, delta: float, kind: int = 4) -> None:
    """Upload the truncated velocity into `scratch`, box-filter it and apply the 2/3 rule."""
    scratch.upload_fields(np.ascontiguousarray(spectral_truncate(fields[:3], scratch.n)))
    for f in range(3):
        scratch.filter_field(kind, delta, f)
    scratch.dealias_all()
    scratch.fov = 1


def log_spectrum_error(e: np.ndarray, e_ref: np.ndarray, kmin: int = 1, kmax: Optional[int] = None) -> float:
    """mean over shells k = kmin..kmax of |ln(E(k) / E_ref(k))| (E[k-1] is shell k)."""
    kmax = len(e_ref) if kmax is None else kmax
    a, b = e[kmin - 1:kmax], e_ref[kmin - 1:kmax]
    ok = (a > 0) & (b > 0)
    return float(np.mean(np.abs(np.log(a[ok] / b[ok])))) if ok.any() else float("inf")


def smagorinsky_stress(A: np.ndarray, cs: float, dx: float) -> np.ndarray:
    """-2 (Cs dx)^2 |S| S on gradient samples A (9, P) (m_les.f90:1142-1215)."""
    A3 = A.astype(np.float64).reshape(3, 3, -1)
    S = 0.5 * (A3 + A3.transpose(1, 0, 2))
    smag = np.sqrt(2.0 * np.einsum("ijp,ijp->p", S, S))
    return np.stack([-2.0 * (cs * dx) ** 2 * smag * S[i, j] for i, j in PAIRS])


def deviatoric(tau: np.ndarray) -> np.ndarray:
    t = tau.astype(np.float64).copy()
    tr = (t[0] + t[3] + t[5]) / 3.0
    for c in (0, 3, 5):
        t[c] -= tr
    return t


def stress_error(pred: np.ndarray, tau: np.ndarray) -> float:
    """Normalised mean-square error of deviatoric stresses (Frobenius)."""
    e = deviatoric(pred) - deviatoric(tau)
    t = deviatoric(tau)
    return float(np.einsum("c,cp,cp->", FROB, e, e) / np.einsum("c,cp,cp->", FROB, t, t))


def stress_correlation(pred: np.ndarray, tau: np.ndarray) -> float:
    a, b = deviatoric(pred), deviatoric(tau)
    num = np.einsum("c,cp,cp->", FROB, a, b)
    return float(num / np.sqrt(np.einsum("c,cp,cp->", FROB, a, a) * np.einsum("c,cp,cp->", FROB, b, b)))


def best_smagorinsky_g1(A: np.ndarray, tau: np.ndarray, delta: float) -> float:
    """Least-squares g1 of tau = g1 Delta^2 |S| S (Frobenius) over samples."""
    m = smagorinsky_stress(A, 1.0, 1.0) / -2.0 * delta * delta  # Delta^2 |S| S
    t = deviatoric(tau)
    return float(np.einsum("c,cp,cp->", FROB, m, t) / np.einsum("c,cp,cp->", FROB, m, m))


@dataclass
class LesExperiment:
    """A-posteriori test: LES at n_les of a forced DNS at n_dns (same forcing)."""
    n_dns: int = 128
    n_les: int = 32
    re: float = 1000.0
    dt_dns: float = 0.002
    famp: float = 0.5
    kfmax: int = 2
    ratio: float = 2.0          # filter width / LES grid spacing
    nruns: int = 2              # DNS runs of the batch that generate training data
    spinup: float = 2.0         # time before training snapshots
    collect: float = 1.0        # training snapshots spread over this time
    nsnap: int = 4
    window: float = 1.0         # a-posteriori window after the last snapshot
    nsample: int = 5
    stride: int = 2
    train_steps: int = 1500
    batch: int = 16384
    lr: float = 1e-3
    lam: float = 1.0            # weight of the dissipation term of the loss
    clip: bool = True
    kernel: int = 1             # inference on the tensor cores (1) or the CUDA cores (0)
    cs: float = 0.18
    seed: int = 5
    graph_steps: int = 20

    @property
    def delta(self) -> float:
        return self.ratio * 2.0 * np.pi / self.n_les

    @property
    def dt_les(self) -> float:
        return self.dt_dns * self.n_dns / self.n_les

    def dns_params(self) -> Params:
        return Params(nx=self.n_dns, dealias=0, flow_type=1, force_type=1, kfmax=self.kfmax, famp=self.famp,
                      nu=1.0 / self.re, dt=self.dt_dns)

    def les_params(self, model: int) -> Params:
        return Params(nx=self.n_les, dealias=0, flow_type=1, force_type=1, kfmax=self.kfmax, famp=self.famp,
                      nu=1.0 / self.re, dt=self.dt_les, les_model=model, c_smag=self.cs)


def _steps(t: float, dt: float) -> int:
    return max(1, int(round(t / dt)))


def generate_training_data(ex: LesExperiment, log=print):
    """Run the batched DNS through spin-up and the collection window; return
    (A, tau, the last state and old RHS of run 0, timings)."""
    b = Batch([ex.dns_params() for _ in range(ex.nruns)])
    b.init(isp_type=2, peak=4.0, ir_exp=2.0)
    t0 = time.perf_counter()
    b.step(_steps(ex.spinup, ex.dt_dns), graph_steps=ex.graph_steps)
    As, taus = [], []
    per = _steps(ex.collect / ex.nsnap, ex.dt_dns)
    for s in range(ex.nsnap):
        b.step(per, graph_steps=ex.graph_steps)
        for c in b.contexts:
            A, tau = sgs_samples(c, ex.delta, ex.stride)
            As.append(A)
            taus.append(tau)
    t_dns = time.perf_counter() - t0
    f0 = b.contexts[0].download_fields()
    r0 = b.contexts[0].download_rhs_old()
    b.close()
    A = np.concatenate(As, axis=1)
    tau = np.concatenate(taus, axis=1)
    log(f"training data: {A.shape[1]} points from {ex.nruns} runs x {ex.nsnap} snapshots ({t_dns:.1f} s)")
    return A, tau, f0, r0


def train_closure(ex: LesExperiment, A: np.ndarray, tau: np.ndarray, device: int = 0, log=print):
    m = Mlp(device=device, seed=ex.seed)
    m.set_data(A, tau, ex.delta)
    t0 = time.perf_counter()
    losses = m.train(ex.train_steps, batch=ex.batch, lr=ex.lr, lam=ex.lam, seed=ex.seed + 1)
    dt = time.perf_counter() - t0
    log(f"training: {ex.train_steps} Adam steps, loss {losses[:20].mean():.4f} -> {losses[-50:].mean():.4f} ({dt:.1f} s)")
    return m, losses, dt


def run_experiment(ex: LesExperiment, device: int = 0, log=print) -> Dict:
    A, tau, f0, r0 = generate_training_data(ex, log)
    m, losses, t_train = train_closure(ex, A, tau, device, log)
    w16 = m.bf16()
    g1_best = best_smagorinsky_g1(A, tau, ex.delta)
    del A, tau

    dns = Context(ex.dns_params())
    dns.upload_fields(f0)
    dns.upload_rhs_old(r0)
    dns.fov = 0
    ref = Context(ex.les_params(0))
    models = {"learned": LES_LEARNED, "smagorinsky": 1, "none": 0}
    les = {}
    for name, model in models.items():
        c = Context(ex.les_params(model))
        if model == LES_LEARNED:
            c.les_set_mlp(w16, ex.delta, clip=ex.clip, kernel=ex.kernel)
        filtered_state(f0, c, ex.delta)
        les[name] = c

    dns_per = _steps(ex.window / ex.nsample, ex.dt_dns)
    les_per = _steps(ex.window / ex.nsample, ex.dt_les)
    errs: Dict[str, List[float]] = {k: [] for k in models}
    spectra: Dict[str, List[List[float]]] = {k: [] for k in list(models) + ["filtered_dns"]}
    kc = ref.kmax
    wall = {k: 0.0 for k in list(models) + ["dns"]}
    for s in range(ex.nsample):
        t0 = time.perf_counter()
        dns.step(dns_per)
        wall["dns"] += time.perf_counter() - t0
        filtered_state(dns.download_fields(), ref, ex.delta)
        e_ref, _ = ref.stats()
        spectra["filtered_dns"].append(e_ref.tolist())
        for name, c in les.items():
            try:
                t0 = time.perf_counter()
                c.step(les_per)
                wall[name] += time.perf_counter() - t0
                e, _ = c.stats()
                ok = bool(np.all(np.isfinite(e)))
            except Exception as exc:  # a blown-up LES is reported, not raised
                log(f"{name}: {exc}")
                e, ok = np.full(kc, np.nan), False
            spectra[name].append(e.tolist())
            errs[name].append(log_spectrum_error(e, e_ref, 1, kc) if ok else float("inf"))

    # a-priori errors on held-out data: the DNS at the end of the window
    Ah, th = sgs_samples(dns, ex.delta, ex.stride)
    pred = m.predict(Ah, ex.delta, clip=ex.clip, kernel=ex.kernel)
    dx_les = 2.0 * np.pi / ex.n_les
    apriori = {
        "learned": stress_error(pred, th),
        "smagorinsky": stress_error(smagorinsky_stress(Ah, ex.cs, dx_les), th),
        "best_smagorinsky": stress_error(smagorinsky_stress(Ah, 1.0, 1.0) * (g1_best * ex.delta ** 2 / -2.0), th),
        "corr_learned": stress_correlation(pred, th),
        "corr_smagorinsky": stress_correlation(smagorinsky_stress(Ah, ex.cs, dx_les), th),
    }
    for c in list(les.values()) + [dns, ref]:
        c.close()
    m.close()
    res = {
        "setup": asdict(ex),
        "delta": ex.delta,
        "dt_les": ex.dt_les,
        "kc": kc,
        "spectrum_error": {k: float(np.mean(v)) for k, v in errs.items()},
        "spectrum_error_per_sample": errs,
        "apriori_stress_error": apriori,
        "train_loss_first": float(np.mean(losses[:20])),
        "train_loss_last": float(np.mean(losses[-50:])),
        "train_seconds": t_train,
        "ms_per_step": {k: 1000.0 * v / ((dns_per if k == "dns" else les_per) * ex.nsample) for k, v in wall.items()},
        "spectra": spectra,
    }
    # simulated time per wall-clock second, LES over DNS
    res["speedup_vs_dns"] = {k: (ex.dt_les / res["ms_per_step"][k]) / (ex.dt_dns / res["ms_per_step"]["dns"])
                             for k in models}
    log("a-posteriori mean |ln E/E_fdns| over k=1..%d: " % kc +
        ", ".join(f"{k} {v:.4f}" for k, v in res["spectrum_error"].items()))
    log("a-priori stress error: " + ", ".join(f"{k} {v:.4f}" for k, v in apriori.items()))
    log("ms per step: " + ", ".join(f"{k} {v:.3f}" for k, v in res["ms_per_step"].items()) +
        "; speedup vs DNS (simulated time per second): " +
        ", ".join(f"{k} {v:.1f}" for k, v in res["speedup_vs_dns"].items()))
    return res


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    for f in LesExperiment.__dataclass_fields__.values():
        ap.add_argument("--" + f.name.replace("_", "-"), type=type(f.default) if f.type != "bool" else int,
                        default=f.default)
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    ex = LesExperiment(**{k: (bool(v) if isinstance(LesExperiment.__dataclass_fields__[k].default, bool) else v)
                          for k, v in vars(a).items() if k != "out"})
    res = run_experiment(ex)
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)


if __name__ == "__main__":
    main()
