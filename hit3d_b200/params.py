"""Reader of the reference's positional input file <run_name>.in.

Restates read_input_file (m_parameters.f90:172-512) with Fortran list-directed
semantics: each READ takes as many values as it asks for, continuing onto the
next line when a line has too few, and then skips the rest of its last line;
a bare READ skips one line.  Derived values follow m_parameters_init
(kmax, m_parameters.f90:123-131), nu = 1/RE, dt < 0 meaning a fixed step
(m_parameters.f90:275-284) and PE = nu/Sc (m_parameters.f90:451).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

from .gpu import Params


class InputFileError(ValueError):
    """Raised where the reference stops with 'An error was encountered while reading input file'."""


@dataclass
class RunConfig:
    nx: int = 0
    ny: int = 0
    nz_all: int = 0
    itmin: int = 0
    itmax: int = 0
    iprint1: int = 1
    iprint2: int = 1
    iwrite4: int = 1
    tmax: float = 0.0
    trescale: float = 0.0
    nrescale: int = 0
    tscalar: float = 0.0
    flow_type: int = 0
    re: float = 1.0
    dt: float = 0.0
    variable_dt: bool = False
    isp_type: int = 0
    ir_exp: int = 0
    peak_wavenum: float = 1.0
    force_type: int = 1
    kfmax: int = 0
    famp: float = 0.0
    dealias: int = 0
    det_rand: int = 0
    rn1: float = 0.0
    rn2: float = 0.0
    rn3: float = 0.0
    nptot: int = 0
    particles_tracking_scheme: int = 0
    starttime_particles: float = 0.0
    particles_filter_size: float = 0.0
    les_model: int = 0
    n_scalars: int = 0
    scalar_type: List[int] = field(default_factory=list)
    sc: List[float] = field(default_factory=list)
    ir_exp_sc: List[float] = field(default_factory=list)
    peak_wavenum_sc: List[float] = field(default_factory=list)
    reac_sc: List[float] = field(default_factory=list)

    @property
    def nu(self) -> float:
        return 1.0 / self.re

    @property
    def dx(self) -> float:
        return 2.0 * (4.0 * math.atan(1.0)) / self.nx

    @property
    def kmax(self) -> int:
        if self.dealias == 0:
            return self.nx // 3
        return int(math.floor(self.nx / 3.0 * math.sqrt(2.0)))

    @property
    def pe(self) -> List[float]:
        return [self.nu / s for s in self.sc]

    def to_params(self, precision: int = 0, device: int = 0, c_smag: float = 0.18, c_t: float = 1.0,
                  c_mixed: float = 0.0) -> Params:
        return Params(nx=self.nx, dealias=self.dealias, flow_type=self.flow_type, force_type=self.force_type,
                      kfmax=self.kfmax, n_scalars=self.n_scalars, precision=precision, les_model=self.les_model,
                      scalar_type=list(self.scalar_type), device=device, nu=self.nu, dt=self.dt, famp=self.famp,
                      c_smag=c_smag, sc=list(self.sc), c_t=c_t, c_mixed=c_mixed, reac_sc=list(self.reac_sc))


class _ListDirected:
    """Fortran list-directed reads over the lines of a text file."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0

    def skip(self):
        if self.pos >= len(self.lines):
            raise InputFileError("unexpected end of input file")
        self.pos += 1

    def line(self) -> str:
        if self.pos >= len(self.lines):
            raise InputFileError("unexpected end of input file")
        s = self.lines[self.pos]
        self.pos += 1
        return s

    def read(self, *types):
        vals = []
        while len(vals) < len(types):
            if self.pos >= len(self.lines):
                raise InputFileError("unexpected end of input file")
            toks = self.lines[self.pos].replace(",", " ").split()
            self.pos += 1
            for t in toks:
                if len(vals) == len(types):
                    break
                vals.append(t)
        out = []
        for v, ty in zip(vals, types):
            try:
                if ty is int:
                    out.append(int(v))
                else:
                    out.append(float(v.replace("d", "e").replace("D", "e")))
            except ValueError as e:
                raise InputFileError(f"bad value {v!r} in input file") from e
        return out[0] if len(out) == 1 else out


def parse_input(text: str, numprocs: int = 1) -> RunConfig:
    r = _ListDirected(text)
    c = RunConfig()
    r.skip(); r.skip(); r.skip()
    c.nx, c.ny, c.nz_all = r.read(int, int, int)
    r.skip()
    if c.nz_all % numprocs:
        raise InputFileError(f"wrong nz_all: {c.nz_all} should be divisible by numprocs {numprocs}")
    c.itmin = r.read(int)
    c.itmax = r.read(int)
    c.iprint1 = r.read(int)
    c.iprint2 = r.read(int)
    c.iwrite4 = r.read(int)
    r.skip()
    c.tmax = r.read(float)
    # TRESCALE, NRESCALE; a missing NRESCALE means one rescale if TRESCALE > 0
    save = r.pos
    toks = r.line().replace(",", " ").split()
    try:
        c.trescale = float(toks[0])
    except (IndexError, ValueError) as e:
        raise InputFileError("bad TRESCALE") from e
    try:
        c.nrescale = int(toks[1])
    except (IndexError, ValueError):
        c.nrescale = 1 if c.trescale > 0.0 else 0
    del save
    c.tscalar = r.read(float)
    r.skip()
    c.flow_type = r.read(int)
    r.skip()
    c.re = r.read(float)
    dt = r.read(float)
    c.variable_dt = dt >= 0.0
    c.dt = -dt if dt < 0.0 else dt
    r.skip()
    c.isp_type = r.read(int)
    c.ir_exp = r.read(int)
    c.peak_wavenum = r.read(float)
    r.skip()
    c.force_type = r.read(int)
    c.kfmax = r.read(int)
    c.famp = r.read(float)
    r.skip()
    c.dealias = r.read(int)
    r.skip()
    c.det_rand = r.read(int)
    c.rn1 = r.read(float)
    c.rn2 = r.read(float)
    c.rn3 = r.read(float)
    r.skip()
    c.nptot = r.read(int)
    c.particles_tracking_scheme = r.read(int)
    if c.particles_tracking_scheme not in (0, 1, 2):
        c.particles_tracking_scheme = 0
    if c.particles_tracking_scheme > 1:
        raise InputFileError("Cannot do this particle tracking")
    c.starttime_particles = r.read(float)
    c.particles_filter_size = r.read(float)
    if 0.0 < c.particles_filter_size < 3.0 * (2.0 * math.pi / c.nx):
        raise InputFileError("particles_filter_size is too small (less than 3*dx)")
    r.skip()
    c.les_model = r.read(int)
    r.skip()
    if c.les_model > 0 and c.dealias != 0:
        c.dealias = 0  # LES mode forces the 2/3 rule (m_parameters.f90:416-420)
    c.n_scalars = r.read(int)
    r.skip()
    if c.n_scalars > 0:
        r.line()  # header line of the scalar table
        for _ in range(c.n_scalars):
            t, sc, ire, pk, reac = r.read(int, float, float, float, float)
            c.scalar_type.append(t)
            c.sc.append(sc)
            c.ir_exp_sc.append(ire)
            c.peak_wavenum_sc.append(pk)
            c.reac_sc.append(reac)
    return c


def read_input_file(path: str, numprocs: int = 1) -> RunConfig:
    with open(path) as f:
        return parse_input(f.read(), numprocs=numprocs)
