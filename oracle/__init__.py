"""CPU oracle for the HIT3DP pseudospectral timestep -- TEST INFRASTRUCTURE ONLY.

This package wraps ``libhit3d_oracle.so`` (built from ``hit3d_oracle.c`` by the
Makefile beside it), an FP64 C restatement of the reference Fortran step.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
it, and only as the checker: the product library never calls it.

Parity status: unpinned against the reference's own build (no Fortran/MPI/FFTW
toolchain on these machines, no golden vectors in the reference).  Pinned against
the analytic checks restated from ``rhs_velocity.f90:430-553`` and
``rhs_scalars.f90:504-594``, against ``numpy.fft`` for the transform, and exactly for
the RANDu integer stream.

All arrays use the reference layout: a field is a Fortran-ordered
``(nx+2, ny, nz)`` float64 array; Fourier space is (kx re/im, kz, ky).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libhit3d_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle shared library with its Makefile."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "hit3d_oracle.c"))
    ):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                    dp, C.POINTER(C.c_int)]
        L.oracle_destroy.argtypes = [vp]
        for name in ("oracle_fields", "oracle_rhs_old", "oracle_wrk", "oracle_turb_visc"):
            getattr(L, name).restype = dp
            getattr(L, name).argtypes = [vp]
        L.oracle_kmax.restype = C.c_int
        L.oracle_kmax.argtypes = [vp]
        L.oracle_nforced.restype = C.c_int
        L.oracle_nforced.argtypes = [vp]
        L.oracle_courant.restype = C.c_double
        L.oracle_courant.argtypes = [vp]
        L.oracle_time.restype = C.c_double
        L.oracle_time.argtypes = [vp]
        L.oracle_set_time.argtypes = [vp, C.c_double]
        L.oracle_set_dt.argtypes = [vp, C.c_double]
        L.oracle_set_flags.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.oracle_get_flags.argtypes = [vp, C.POINTER(C.c_int)]
        L.oracle_step.argtypes = [vp, C.c_int]
        L.oracle_rhs.argtypes = [vp]
        L.oracle_pressure.argtypes = [vp]
        L.oracle_dealias_all.argtypes = [vp]
        L.oracle_fft3d.argtypes = [vp, C.c_int, dp]
        L.oracle_fft1d.argtypes = [C.c_int, dp, C.c_int]
        L.oracle_stats.argtypes = [vp, dp]
        L.oracle_les_stats.argtypes = [vp, dp]
        L.oracle_nwrk.argtypes = [vp]
        L.oracle_nwrk.restype = C.c_int
        L.oracle_set_les_constants.argtypes = [vp, C.c_double, C.c_double]
        L.oracle_set_reaction.argtypes = [vp, C.c_int, C.c_double]
        L.oracle_scalar_stats.argtypes = [vp, dp]
        L.oracle_energy_spectrum.argtypes = [vp, C.c_int, C.c_int, dp]
        L.oracle_forcing_energy.restype = C.c_double
        L.oracle_forcing_energy.argtypes = [vp]
        L.oracle_init_velocity.restype = C.c_int
        L.oracle_init_velocity.argtypes = [vp, C.c_double, C.c_int, C.c_double, C.c_double]
        L.oracle_init_scalar.argtypes = [vp, C.c_int, C.c_double, C.c_double]
        L.oracle_randu_stream.argtypes = [C.c_double, C.c_int64, dp]
        L.oracle_velocity_rescale.restype = C.c_int
        L.oracle_velocity_rescale.argtypes = [vp, C.c_int, C.c_double, C.c_double]
        L.oracle_particles_step.argtypes = [C.c_int, C.c_double, dp, C.c_int64, dp, dp, C.c_int]
        L.oracle_particles_lattice.restype = C.c_int64
        L.oracle_particles_lattice.argtypes = [C.c_int, C.c_int64, dp]
        L.oracle_filter_g.argtypes = [vp, C.c_int, C.c_double, dp]
        L.oracle_apply_filter.argtypes = [vp, dp, dp]
        L.oracle_read_restart.restype = C.c_int
        L.oracle_read_restart.argtypes = [vp, C.c_char_p, dp, dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(C.POINTER(C.c_double))


def randu_stream(seed: float, count: int) -> np.ndarray:
    """RANDu values 2..count+1 of the stream seeded with ``random(-seed)`` (RANDu.f)."""
    out = np.empty(count, dtype=np.float64)
    lib().oracle_randu_stream(float(seed), int(count), _dp(out))
    return out


def fft1d(x: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised complex FFT (sign -1 forward, +1 backward) of the oracle."""
    buf = np.ascontiguousarray(np.stack([x.real, x.imag], axis=-1).astype(np.float64))
    lib().oracle_fft1d(len(x), _dp(buf), int(sign))
    return buf[..., 0] + 1j * buf[..., 1]


def particles_lattice(n: int, nptot: int) -> np.ndarray:
    L = lib()
    m = L.oracle_particles_lattice(n, nptot, None)
    xyz = np.zeros((m, 3), dtype=np.float64)
    L.oracle_particles_lattice(n, nptot, _dp(xyz))
    return xyz


def particles_step(n: int, dt: float, uphys: np.ndarray, xyzp: np.ndarray, uvwp: np.ndarray,
                   scheme: int) -> None:
    """Advance particles one step in place (CINT scheme=1, trilinear scheme=0).

    ``uphys`` is a (3, nz, ny, nx+2) C-ordered view of three physical fields,
    ``xyzp``/``uvwp`` are (np, 3) C-ordered arrays in grid units."""
    assert uphys.flags.c_contiguous and xyzp.flags.c_contiguous and uvwp.flags.c_contiguous
    lib().oracle_particles_step(n, dt, _dp(uphys), xyzp.shape[0], _dp(xyzp), _dp(uvwp), scheme)


class Oracle:
    """One hydro task of the reference: fields, rhs_old and wrk on the host."""

    def __init__(self, n, *, nscal=0, dealias=0, flow_type=0, force_type=1, kfmax=2, nu=1.0 / 400,
                 dt=0.005, famp=0.5, les_model=0, c_smag=0.18, sc=(), scalar_type=()):
        L = lib()
        sc_arr = (C.c_double * 8)(*list(sc))
        st_arr = (C.c_int * 8)(*list(scalar_type))
        self._p = L.oracle_create(n, nscal, dealias, flow_type, force_type, kfmax, nu, dt, famp,
                                  les_model, c_smag, sc_arr, st_arr)
        if not self._p:
            raise MemoryError("oracle_create failed")
        self.n, self.nscal = n, nscal
        # LES fields: k_sgs, and (B T_B), (eps T_eps) with the lag model
        self.nles = {2: 1, 3: 3, 4: 1, 5: 3, 6: 1, 7: 3, 10: 2}.get(les_model, 0)
        self.nu = nu
        self.kmax = L.oracle_kmax(self._p)
        self.fsz = (n + 2) * n * n
        nf = 3 + nscal + self.nles
        self.fields = np.ctypeslib.as_array(L.oracle_fields(self._p), shape=(nf * self.fsz,)).reshape(
            nf, n, n, n + 2)
        self.rhs_old = np.ctypeslib.as_array(L.oracle_rhs_old(self._p), shape=(nf * self.fsz,)).reshape(
            nf, n, n, n + 2)
        nw = L.oracle_nwrk(self._p)
        self.wrk = np.ctypeslib.as_array(L.oracle_wrk(self._p), shape=(nw * self.fsz,)).reshape(
            nw, n, n, n + 2)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            lib().oracle_destroy(p)
            self._p = None

    # field views are (nfield, k, j, i) C-ordered == Fortran (i, j, k, nfield)
    def init_velocity(self, rn1, isp_type=1, peak_wavenum=4.0, ir_exp=2.0):
        rc = lib().oracle_init_velocity(self._p, float(rn1), int(isp_type), float(peak_wavenum), float(ir_exp))
        if rc != 0:
            raise ValueError(f"unsupported isp_type {isp_type}")

    def init_scalar(self, s, rn2, peak_wavenum=4.0):
        if lib().oracle_init_scalar(self._p, int(s), float(rn2), float(peak_wavenum)) != 0:
            raise ValueError("unsupported scalar type")

    def dealias_all(self):
        lib().oracle_dealias_all(self._p)

    def velocity_rescale(self, isp_type, peak_wavenum, ir_exp=2.0):
        if lib().oracle_velocity_rescale(self._p, int(isp_type), float(peak_wavenum), float(ir_exp)) != 0:
            raise ValueError(f"unsupported isp_type {isp_type}")

    def step(self, nsteps=1):
        lib().oracle_step(self._p, int(nsteps))

    def rhs(self):
        lib().oracle_rhs(self._p)

    def pressure(self):
        lib().oracle_pressure(self._p)

    def fft3d(self, flag, a: np.ndarray):
        assert a.shape == (self.n, self.n, self.n + 2) and a.flags.c_contiguous
        lib().oracle_fft3d(self._p, int(flag), _dp(a))

    def set_flags(self, fov, fos, int_scalars):
        lib().oracle_set_flags(self._p, int(fov), int(fos), int(int_scalars))

    def flags(self):
        f = (C.c_int * 3)()
        lib().oracle_get_flags(self._p, f)
        return tuple(f)

    def set_dt(self, dt):
        lib().oracle_set_dt(self._p, float(dt))

    @property
    def courant(self):
        return lib().oracle_courant(self._p)

    @property
    def time(self):
        return lib().oracle_time(self._p)

    def forcing_energy(self):
        return lib().oracle_forcing_energy(self._p)

    def nforced(self):
        return lib().oracle_nforced(self._p)

    def stats(self):
        """Return (e_spec[kmax], dict of derived statistics)."""
        out = np.zeros(self.kmax + 12)
        lib().oracle_stats(self._p, _dp(out))
        keys = ["energy", "eps_v", "eta", "etakmax", "uvar", "x_length", "lambda", "re_lambda",
                "re_lambda1", "tau_e", "enstrophy", "skewness"]
        return out[: self.kmax].copy(), dict(zip(keys, out[self.kmax:].tolist()))

    def set_reaction(self, s, rate):
        """reac_sc of scalar s (used by scalar type 311 with phase-shift dealiasing)."""
        lib().oracle_set_reaction(self._p, int(s), float(rate))

    def set_les_constants(self, c_t=1.0, c_mixed=0.0):
        """C_T of les_model 5 (c_t.in) and C_mixed of les_models 6 and 7 (c_mixed.in)."""
        lib().oracle_set_les_constants(self._p, float(c_t), float(c_mixed))

    def les_stats(self):
        """les.gp quantities of the last RHS evaluation (dynamic localization model)."""
        out = np.zeros(4)
        lib().oracle_les_stats(self._p, _dp(out))
        return dict(zip(("energy", "production", "B", "dissipation"), out.tolist()))

    def scalar_stats(self):
        out = np.zeros(self.nscal * (self.kmax + 5))
        lib().oracle_scalar_stats(self._p, _dp(out))
        res = []
        for s in range(self.nscal):
            d = out[s * (self.kmax + 5):(s + 1) * (self.kmax + 5)]
            res.append(dict(spectrum=d[: self.kmax].copy(), diss=d[self.kmax], mean=d[self.kmax + 1],
                            variance=d[self.kmax + 2], min=d[self.kmax + 3], max=d[self.kmax + 4]))
        return res

    def filter_g(self, kind, delta):
        g = np.zeros((self.n, self.n, self.n + 2))
        lib().oracle_filter_g(self._p, int(kind), float(delta), _dp(g))
        return g

    def read_restart(self, path):
        """restart_read_parallel (restart_io.f90:341-506) into this oracle's fields;
        returns (time, dt, nums_in_file, nles_in_file)."""
        t, d = C.c_double(0.0), C.c_double(0.0)
        nums, nles = C.c_int(0), C.c_int(0)
        rc = lib().oracle_read_restart(self._p, os.fsencode(path), C.byref(t), C.byref(d), C.byref(nums), C.byref(nles))
        if rc == -2:
            raise ValueError("Dimensions are different")
        if rc != 0:
            raise OSError(f"cannot read restart file {path}")
        return t.value, d.value, nums.value, nles.value

    def apply_filter(self, g, a):
        lib().oracle_apply_filter(self._p, _dp(g), _dp(a))
