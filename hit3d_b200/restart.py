"""Restart files and real*4 field files in the reference's byte layouts.

Restart file <run_name>.64.<itime:06d> (restart_io.f90:240-334, read :341-506):
  header: 5 x int32 (nx, ny, nz_all, nums, nles) + 2 x float64 (TIME, DT) = 36 bytes;
  then, per variable, the Fourier array's first nx of its nx+2 rows (the kx = N/2
  pair is dropped) as float64 in (x, y, z) column-major order.
Real*4 file (write_tmp4.f90:14-33): 3 x int32 (nx, ny, nz) then float32 data.
All little-endian as written on x86 hosts.
"""
from __future__ import annotations

import os
import struct

import numpy as np

HEADER = struct.Struct("<5i2d")


class RestartError(ValueError):
    pass


def restart_name(run_name: str, itime: int) -> str:
    return f"{run_name}.64.{itime:06d}"


def write_restart(path: str, fields: np.ndarray, time: float, dt: float, nums: int, nles: int = 0) -> None:
    """fields: (nvar, nz, ny, nx+2) C-ordered Fourier arrays, nvar = 3 + nums + nles."""
    nvar, nz, ny, nx2 = fields.shape
    nx = nx2 - 2
    if nvar != 3 + nums + nles:
        raise RestartError("number of variables does not match nums + nles")
    tmp = path + ".part"
    with open(tmp, "wb") as f:
        f.write(HEADER.pack(nx, ny, nz, nums, nles, float(time), float(dt)))
        for n in range(nvar):
            f.write(np.ascontiguousarray(fields[n, :, :, :nx], dtype="<f8").tobytes())
    os.replace(tmp, path)


def read_restart_header(path: str, nx: int):
    """Header of a restart file, checked against the grid and the file size:
    (nx, ny, nz, nums, nles, time, dt)."""
    size = os.path.getsize(path)
    if size < HEADER.size:
        raise RestartError(f"{path}: truncated header")
    with open(path, "rb") as f:
        h = HEADER.unpack(f.read(HEADER.size))
    nx1, ny1, nz1, nums1, nles1 = h[:5]
    if (nx1, ny1, nz1) != (nx, nx, nx):
        raise RestartError(f"Dimensions are different: input file {nx}^3, restart file {nx1} {ny1} {nz1}")
    if nums1 < 0 or nles1 < 0:
        raise RestartError("corrupt header (negative counts)")
    if size != HEADER.size + (3 + nums1 + nles1) * nx * nx * nx * 8:
        raise RestartError(f"{path}: size {size} does not match its header")
    return h


def read_restart(path: str, nx: int, n_scalars: int, n_les: int = 0):
    """Return (fields (3 + n_scalars + n_les, nx, nx, nx + 2), time, dt, nums_in_file, nles_in_file).

    Dimension mismatches are errors; the scalar count follows the input file:
    extra scalars in the file are dropped, missing ones come back as zeros for
    the caller to initialise (restart_io.f90:408-448)."""
    size = os.path.getsize(path)
    if size < HEADER.size:
        raise RestartError(f"{path}: truncated header")
    with open(path, "rb") as f:
        nx1, ny1, nz1, nums1, nles1, time, dt = HEADER.unpack(f.read(HEADER.size))
        if (nx1, ny1, nz1) != (nx, nx, nx):
            raise RestartError(f"Dimensions are different: input file {nx}^3, restart file {nx1} {ny1} {nz1}")
        if nums1 < 0 or nles1 < 0:
            raise RestartError("corrupt header (negative counts)")
        per = nx * nx * nx * 8
        if size != HEADER.size + (3 + nums1 + nles1) * per:
            raise RestartError(f"{path}: size {size} does not match its header")
        nread = 3 + min(n_scalars, nums1)
        out = np.zeros((3 + n_scalars + n_les, nx, nx, nx + 2))
        for n in range(nread):
            f.seek(HEADER.size + n * per)
            out[n, :, :, :nx] = np.frombuffer(f.read(per), dtype="<f8").reshape(nx, nx, nx)
        for n in range(min(n_les, nles1)):
            f.seek(HEADER.size + (3 + nums1 + n) * per)
            out[3 + n_scalars + n, :, :, :nx] = np.frombuffer(f.read(per), dtype="<f8").reshape(nx, nx, nx)
    return out, time, dt, nums1, nles1


def write_real4(path: str, phys: np.ndarray) -> None:
    """phys: (nz, ny, nx+2) physical array; writes the first nx of every row."""
    nz, ny, nx2 = phys.shape
    nx = nx2 - 2
    with open(path, "wb") as f:
        f.write(struct.pack("<3i", nx, ny, nz))
        f.write(np.ascontiguousarray(phys[:, :, :nx], dtype="<f4").tobytes())


def read_real4(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        nx, ny, nz = struct.unpack("<3i", f.read(12))
        return np.frombuffer(f.read(), dtype="<f4").reshape(nz, ny, nx)
