"""Host side of the Lagrangian particles (the reference's 'parts' task).

Restates the file handling of m_particles.f90: the initial positions
(particles_init, m_particles.f90:157-337: the restart file pt.<ext>, else
<run_name>.pt, else a cubic lattice of round(nptot^(1/3))^3 particles), the
binary restart pt.<ext> (particles_restart_write_binary / _read_binary,
m_particles.f90:558-744) and the per-particle trajectory files p.NNNN written
every step when nptot < 1000 (m_particles.f90:1424-1434).  Positions are kept
in the reference's grid units (1-based, x / dx + 1); the device interpolates
and advances them inside each time step.
"""
from __future__ import annotations

import math
import os
import struct

import numpy as np


class ParticleFileError(ValueError):
    """An unreadable particle file (the reference stops with my_exit(-1))."""


def lattice(nptot: int, n: int):
    """particles_init's internal lattice: npthird^3 particles at the cell centres
    of an npthird^3 lattice over [0, 2 pi)^3, npthird the integer cube root of
    nptot rounded to the nearer cube (m_particles.f90:195-226)."""
    npthird = int(float(nptot) ** (1.0 / 3.0))
    if nptot - npthird ** 3 >= (npthird + 1) ** 3 - nptot:
        npthird += 1
    total = min(npthird ** 3, 2 ** 30)
    step = 2.0 * math.pi / npthird
    g = (np.arange(npthird) + 0.5) * step
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    phys = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)[:total]
    return np.arange(1, total + 1, dtype=np.int32), phys


def to_grid(phys: np.ndarray, n: int) -> np.ndarray:
    """Physical positions, wrapped into [0, 2 pi), to grid units x / dx + 1
    (m_particles.f90:256-300)."""
    two_pi = 2.0 * math.pi
    p = np.array(phys, dtype=np.float64)
    out = (p < 0.0) | (p >= two_pi)
    p[out] = p[out] - two_pi * np.floor(p[out] / two_pi)
    return p / (two_pi / n) + 1.0


def read_run_pt(path: str, nptot: int) -> np.ndarray:
    """<run_name>.pt: nptot lines of x y z (list-directed)."""
    try:
        vals = np.array(open(path).read().replace(",", " ").split(), dtype=np.float64)
    except ValueError as e:
        raise ParticleFileError(f"{path}: bad number") from e
    if vals.size < 3 * nptot:
        raise ParticleFileError(f"{path}: {vals.size // 3} positions for nptot = {nptot}")
    return vals[: 3 * nptot].reshape(nptot, 3)


# pt.<ext>: nptot as the reference's default integer (8 bytes with -i8), then
# per particle ipart (integer*4) and x, y, z (real*8), then TIME (real*8)
def write_pt(path: str, ipart: np.ndarray, grid: np.ndarray, n: int, time: float) -> None:
    dx = 2.0 * math.pi / n
    rec = np.zeros(len(ipart), dtype=[("i", "<i4"), ("x", "<f8", 3)])
    rec["i"] = ipart
    rec["x"] = (np.asarray(grid) - 1.0) * dx
    with open(path, "wb") as fh:
        fh.write(struct.pack("<q", len(ipart)))
        fh.write(rec.tobytes())
        fh.write(struct.pack("<d", float(time)))


def read_pt(path: str, n: int):
    """(ipart, grid positions, time) of a pt.<ext> file."""
    data = open(path, "rb").read()
    if len(data) < 8:
        raise ParticleFileError(f"{path}: truncated header")
    (nptot,) = struct.unpack_from("<q", data, 0)
    need = 8 + nptot * 28 + 8
    if nptot <= 0 or len(data) < need:
        raise ParticleFileError(f"{path}: truncated ({len(data)} bytes for {nptot} particles)")
    rec = np.frombuffer(data, dtype=[("i", "<i4"), ("x", "<f8", 3)], count=nptot, offset=8)
    (time,) = struct.unpack_from("<d", data, 8 + nptot * 28)
    return rec["i"].copy(), to_grid(rec["x"], n), time


def _e16_8(x: float) -> str:
    """Fortran E16.8."""
    if x == 0.0 or not math.isfinite(x):
        m, e = 0.0, 0
    else:
        e = int(math.floor(math.log10(abs(x)))) + 1
        m = x / 10.0 ** e
        if round(abs(m), 8) >= 1.0:
            m /= 10.0
            e += 1
    s = f"{'-' if m < 0 else ''}0.{int(round(abs(m) * 1e8)):08d}E{'+' if e >= 0 else '-'}{abs(e):02d}"
    return s.rjust(16)


def append_trajectories(workdir: str, itime: int, time: float, ipart: np.ndarray, grid: np.ndarray,
                        uvw: np.ndarray, n: int) -> None:
    """p.NNNN: itime, rank, time, x, y, z, u, v, w per line, format (i6.6,x,i4,12e16.8)."""
    dx = 2.0 * math.pi / n
    for k, ip in enumerate(ipart):
        xyz = (grid[k] - 1.0) * dx
        line = f"{itime:06d} {0:4d}" + "".join(_e16_8(v) for v in (time, *xyz, *uvw[k]))
        with open(os.path.join(workdir, f"p.{int(ip):04d}"), "a") as fh:
            fh.write(line + "\n")
