"""ctypes binding of libhit3d_gpu.so (the C-ABI of include/hit3d_gpu.h).

This is the Python counterpart of the ISO_C_BINDING interfaces a Fortran host
would declare: every call maps 1:1 onto an ``extern "C"`` entry point, arrays are
passed as plain pointers in the reference's (nx+2, ny, nz, nfields) layout, and a
non-zero return code raises :class:`Hit3dError` (the reference stops through
``my_exit(-1)``, my_exit.f90:23-62).

There is no CPU fallback: if the shared library is missing this module raises on
import of :func:`lib`.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhit3d_gpu.so")
MAX_SCALARS = 8
LES_LEARNED = 20  # les_model of the learned closure (HIT3D_LES_LEARNED)
N_VARIANTS = 15  # launch-shape variants of the fused x pass (HIT3D_FUSED_VARIANTS)


def les_fields(les_model: int) -> int:
    """LES-related transported fields (m_les.f90:111-300): k_sgs for the models with
    an algebraic dissipation (2, 4, 6); k_sgs, (B T_B), (eps T_eps) with the lag
    model (3, 5, 7); (B T_B), (eps T_eps) for the one-equation mixed model (10)."""
    return {2: 1, 3: 3, 4: 1, 5: 3, 6: 1, 7: 3, 10: 2}.get(int(les_model), 0)


_lib = None


class Hit3dError(RuntimeError):
    pass


class _Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("dealias", C.c_int32), ("flow_type", C.c_int32), ("force_type", C.c_int32),
        ("kfmax", C.c_int32), ("n_scalars", C.c_int32), ("precision", C.c_int32), ("les_model", C.c_int32),
        ("scalar_type", C.c_int32 * MAX_SCALARS), ("device", C.c_int32), ("reserved", C.c_int32),
        ("nu", C.c_double), ("dt", C.c_double), ("famp", C.c_double), ("c_smag", C.c_double),
        ("sc", C.c_double * MAX_SCALARS), ("c_t", C.c_double), ("c_mixed", C.c_double),
        ("reac_sc", C.c_double * MAX_SCALARS),
    ]


@dataclass
class Params:
    """Run parameters (the values of <run_name>.in, m_parameters.f90:172-512)."""
    nx: int = 64
    dealias: int = 0
    flow_type: int = 0
    force_type: int = 1
    kfmax: int = 2
    n_scalars: int = 0
    precision: int = 0
    les_model: int = 0
    scalar_type: Sequence[int] = field(default_factory=list)
    device: int = 0
    nu: float = 1.0 / 400.0
    dt: float = 0.005
    famp: float = 0.5
    c_smag: float = 0.18
    sc: Sequence[float] = field(default_factory=list)
    c_t: float = 1.0        # lag-model C_T of les_model 5 (c_t.in)
    c_mixed: float = 0.0    # C_mixed of les_models 6, 7 (c_mixed.in)
    reac_sc: Sequence[float] = field(default_factory=list)  # reaction rates (scalar_type 311)

    @property
    def kmax(self) -> int:
        """Largest resolved shell (m_parameters.f90:123-131)."""
        dealias = 0 if self.les_model else self.dealias
        if dealias == 0:
            return self.nx // 3
        return int(np.floor(self.nx / 3.0 * np.sqrt(2.0)))

    def to_c(self) -> _Params:
        p = _Params()
        for k in ("nx", "dealias", "flow_type", "force_type", "kfmax", "n_scalars", "precision", "les_model",
                  "device"):
            setattr(p, k, int(getattr(self, k)))
        for k in ("nu", "dt", "famp", "c_smag", "c_t", "c_mixed"):
            setattr(p, k, float(getattr(self, k)))
        st = list(self.scalar_type) + [0] * MAX_SCALARS
        sc = list(self.sc) + [1.0] * MAX_SCALARS
        rc = list(self.reac_sc) + [0.0] * MAX_SCALARS
        for i in range(MAX_SCALARS):
            p.scalar_type[i] = int(st[i])
            p.sc[i] = float(sc[i])
            p.reac_sc[i] = float(rc[i])
        return p


# (name, restype, argtypes) of every entry point of include/hit3d_gpu.h
_vp, _dp, _i32, _i64, _d = C.c_void_p, C.POINTER(C.c_double), C.c_int32, C.c_int64, C.c_double
_fp = C.POINTER(C.c_float)
SIGNATURES = [
    ("hit3d_gpu_init", C.c_int, [C.POINTER(_Params), C.POINTER(C.c_void_p)]),
    ("hit3d_gpu_finalize", None, [_vp]),
    ("hit3d_gpu_last_error", C.c_char_p, []),
    ("hit3d_gpu_upload_fields", C.c_int, [_vp, _dp, _i64, _i32]),
    ("hit3d_gpu_download_fields", C.c_int, [_vp, _dp, _i64, _i32]),
    ("hit3d_gpu_upload_rhs_old", C.c_int, [_vp, _dp, _i64, _i32]),
    ("hit3d_gpu_download_rhs_old", C.c_int, [_vp, _dp, _i64, _i32]),
    ("hit3d_gpu_step", C.c_int, [_vp, _i32, C.POINTER(_i32), C.POINTER(_i32), _dp]),
    ("hit3d_gpu_step_host", C.c_int, [_vp, _i32, C.POINTER(_dp), C.POINTER(_dp), _i64, _i32, _i32, C.POINTER(_i32),
                                      C.POINTER(_i32), _i32]),
    ("hit3d_gpu_step_host_bytes", C.c_int64, [_vp, _i32, _i32]),
    ("hit3d_gpu_restart_bytes", C.c_int64, [_vp, _i32]),
    ("hit3d_gpu_restart_pack", C.c_int, [_vp, _i32, _d, _d, C.c_void_p]),
    ("hit3d_gpu_restart_unpack", C.c_int, [_vp, C.c_void_p, _i64, _dp, _dp, C.POINTER(_i32), C.POINTER(_i32)]),
    ("hit3d_gpu_stream", C.c_void_p, [_vp]),
    ("hit3d_gpu_launch_count", C.c_int64, [_vp]),
    ("hit3d_gpu_autotune", C.c_int, [_vp, C.POINTER(_i32), _dp]),
    ("hit3d_gpu_autotune_columns", C.c_int, [_vp, C.POINTER(_i32), _dp]),
    ("hit3d_gpu_set_column_tile", C.c_int, [_vp, _i32]),
    ("hit3d_gpu_set_variant", C.c_int, [_vp, _i32]),
    ("hit3d_gpu_set_pruning", C.c_int, [_vp, _i32]),
    ("hit3d_gpu_set_update_fusion", C.c_int, [_vp, _i32]),
    ("hit3d_gpu_check_finite", C.c_int, [_vp, C.POINTER(_i64)]),
    ("hit3d_gpu_les_stats", C.c_int, [_vp, _dp]),
    ("hit3d_gpu_pruned", C.c_int, [_vp]),
    ("hit3d_gpu_step_profile", C.c_int, [_vp, _i32, C.POINTER(_i32), C.POINTER(_i32), _dp]),
    ("hit3d_gpu_set_dt", C.c_int, [_vp, _d]),
    ("hit3d_gpu_set_scalars_active", C.c_int, [_vp, _i32]),
    ("hit3d_gpu_dealias_all", C.c_int, [_vp]),
    ("hit3d_gpu_init_velocity", C.c_int, [_vp, _d, _i32, _d, _d]),
    ("hit3d_gpu_stats", C.c_int, [_vp, _dp, _i32, _dp]),
    ("hit3d_gpu_scalar_stats", C.c_int, [_vp, _i32, _dp, _i32, _dp]),
    ("hit3d_gpu_particles_upload", C.c_int, [_vp, _dp, _dp, _i64, _i32]),
    ("hit3d_gpu_particles_download", C.c_int, [_vp, _dp, _dp]),
    ("hit3d_gpu_particles_filter", C.c_int, [_vp, _d]),
    ("hit3d_gpu_init_scalar", C.c_int, [_vp, _i32, _d, _d]),
    ("hit3d_gpu_xfft3d", C.c_int, [_vp, _i32, _dp, _dp, _i64]),
    ("hit3d_gpu_filter_field", C.c_int, [_vp, _i32, _d, _i32]),
    ("hit3d_gpu_xfft3d_static", C.c_int, [_i32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("hit3d_gpu_physical_velocity", C.c_int, [_vp, _dp, _i64]),
    ("hit3d_gpu_physical_fields", C.c_int, [_vp, _i32, _d, _dp, _i64]),
    ("hit3d_gpu_velocity_rescale", C.c_int, [_vp, _i32, _d, _d]),
    ("hit3d_gpu_sgs_fields", C.c_int, [_vp, _i32, _d, C.POINTER(C.c_float)]),
    ("hit3d_gpu_sgs_samples", C.c_int, [_vp, _i32, _d, _i32, C.POINTER(C.c_float)]),
    ("hit3d_batch_create", C.c_int, [C.POINTER(_Params), _i32, C.POINTER(C.c_void_p)]),
    ("hit3d_batch_context", C.c_int, [_vp, _i32, C.POINTER(C.c_void_p)]),
    ("hit3d_batch_step", C.c_int, [_vp, _i32, _i32]),
    ("hit3d_batch_graph_launches", C.c_int64, [_vp]),
    ("hit3d_batch_nclasses", C.c_int, [_vp]),
    ("hit3d_batch_autotune", C.c_int, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("hit3d_batch_destroy", None, [_vp]),
    ("hit3d_mlp_nparam", C.c_int, []),
    ("hit3d_mlp_create", C.c_int, [_i32, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("hit3d_mlp_destroy", C.c_int, [_vp]),
    ("hit3d_mlp_set_params", C.c_int, [_vp, _fp]),
    ("hit3d_mlp_get_params", C.c_int, [_vp, _fp]),
    ("hit3d_mlp_get_bf16", C.c_int, [_vp, C.POINTER(C.c_uint16)]),
    ("hit3d_mlp_set_data", C.c_int, [_vp, _fp, _fp, _i64, _d]),
    ("hit3d_mlp_norms", C.c_int, [_vp, _dp]),
    ("hit3d_mlp_loss_grad", C.c_int, [_vp, C.POINTER(_i32), _i64, _d, _fp, _fp]),
    ("hit3d_mlp_train", C.c_int, [_vp, _i32, _i64, _d, _d, C.c_uint64, _fp]),
    ("hit3d_mlp_predict", C.c_int, [_vp, _fp, _i64, _d, _i32, _i32, _fp]),
    ("hit3d_gpu_les_set_mlp", C.c_int, [_vp, C.POINTER(C.c_uint16), _i64, _d, _i32, _i32]),
]


def lib():
    """Load the in-tree library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Hit3dError(f"{LIB_PATH} is missing: build it with `python -m hit3d_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != 0:
        msg = lib().hit3d_gpu_last_error().decode(errors="replace")
        raise Hit3dError(f"{what}: code {rc}: {msg}")


def _ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


class Context:
    """One simulation resident on one GPU (a hydro task of the reference).

    Field arrays use the reference layout: a numpy array of shape
    (nfields, nz, ny, nx+2) in C order is exactly Fortran's fields(nx+2, ny, nz, nfields).
    """

    STAT_KEYS = ["energy", "eps_v", "eta", "etakmax", "uvar", "x_length", "lambda", "re_lambda",
                 "re_lambda1", "tau_e", "enstrophy", "skewness"]

    def __init__(self, params: Params, _handle: C.c_void_p | None = None):
        self.params = params
        self.n = params.nx
        # k_sgs of the dynamic localization model is state field 3 + n_scalars
        self.nfields = 3 + params.n_scalars + les_fields(params.les_model)
        self.kmax = params.kmax
        self._owned = _handle is None
        if _handle is None:
            h = C.c_void_p()
            cp = params.to_c()
            _check(lib().hit3d_gpu_init(C.byref(cp), C.byref(h)), "hit3d_gpu_init")
        else:
            h = _handle
        self._h = h
        self.fov = 1
        self.fos = 1
        self.courant = 0.0

    def close(self):
        if getattr(self, "_h", None):
            if self._owned:
                lib().hit3d_gpu_finalize(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    def field_shape(self, nf=None):
        return (self.nfields if nf is None else nf, self.n, self.n, self.n + 2)

    def upload_fields(self, fields: np.ndarray):
        nf = fields.shape[0]
        _check(lib().hit3d_gpu_upload_fields(self._h, _ptr(fields), self.n + 2, nf), "upload_fields")

    def download_fields(self, nf=None, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.field_shape(nf))
        _check(lib().hit3d_gpu_download_fields(self._h, _ptr(out), self.n + 2, out.shape[0]), "download_fields")
        return out

    def upload_rhs_old(self, r: np.ndarray):
        _check(lib().hit3d_gpu_upload_rhs_old(self._h, _ptr(r), self.n + 2, r.shape[0]), "upload_rhs_old")

    def download_rhs_old(self, nf=None) -> np.ndarray:
        out = np.empty(self.field_shape(nf))
        _check(lib().hit3d_gpu_download_rhs_old(self._h, _ptr(out), self.n + 2, out.shape[0]), "download_rhs_old")
        return out

    def step(self, nsteps: int = 1) -> float:
        fov, fos, cour = C.c_int32(self.fov), C.c_int32(self.fos), C.c_double(0.0)
        _check(lib().hit3d_gpu_step(self._h, int(nsteps), C.byref(fov), C.byref(fos), C.byref(cour)), "step")
        self.fov, self.fos, self.courant = fov.value, fos.value, cour.value
        return self.courant

    def step_host_bytes(self, nf: int, band_only: bool = False) -> int:
        """Bytes hit3d_gpu_step_host moves per input, each way."""
        return int(lib().hit3d_gpu_step_host_bytes(self._h, int(nf), int(bool(band_only))))

    def step_host(self, ins, outs, nsteps: int = 1, band_only: bool = False):
        """For each (in, out) pair of host arrays (field_shape()), upload `in`,
        advance nsteps and download into `out`, the next upload overlapping this
        step and download (hit3d_gpu_step_host).  Use pinned arrays for full rate.
        band_only: only the 2/3-rule band crosses PCIe (see the C header)."""
        n = len(ins)
        if n < 1 or len(outs) != n:
            raise ValueError("step_host: ins and outs must be non-empty and of equal length")
        nf = ins[0].shape[0]
        for a in list(ins) + list(outs):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != ins[0].shape:
                raise ValueError("step_host: C-contiguous float64 arrays of one shape")
        pin = (_dp * n)(*[_ptr(a) for a in ins])
        pout = (_dp * n)(*[_ptr(a) for a in outs])
        fov, fos = C.c_int32(self.fov), C.c_int32(self.fos)
        _check(lib().hit3d_gpu_step_host(self._h, n, pin, pout, self.n + 2, nf, int(nsteps), C.byref(fov),
                                         C.byref(fos), int(bool(band_only))), "step_host")
        self.fov, self.fos = fov.value, fos.value

    def restart_image(self, time: float, dt: float, nums: int | None = None) -> np.ndarray:
        """The restart file's bytes (header + Fourier body, restart_io.f90:240-334),
        packed on the device; nums passive scalars (default: all)."""
        nums = self.params.n_scalars if nums is None else int(nums)
        nb = int(lib().hit3d_gpu_restart_bytes(self._h, nums))
        if nb < 0:
            raise Hit3dError("restart_image: nums out of range")
        img = np.empty(nb, dtype=np.uint8)
        _check(lib().hit3d_gpu_restart_pack(self._h, nums, float(time), float(dt), img.ctypes.data_as(C.c_void_p)),
               "restart_pack")
        return img

    def restart_load(self, image) -> tuple:
        """Load a restart file's bytes (restart_io.f90:341-506); returns (time, dt,
        nums in the file, nles in the file).  Scalars the file lacks are zero."""
        img = np.ascontiguousarray(np.frombuffer(image, dtype=np.uint8) if not isinstance(image, np.ndarray) else image)
        t, d = C.c_double(0.0), C.c_double(0.0)
        nums, nles = C.c_int32(0), C.c_int32(0)
        _check(lib().hit3d_gpu_restart_unpack(self._h, img.ctypes.data_as(C.c_void_p), img.nbytes, C.byref(t),
                                              C.byref(d), C.byref(nums), C.byref(nles)), "restart_unpack")
        return t.value, d.value, nums.value, nles.value

    STAGES = ["z_inverse", "y_inverse", "x_fused", "y_forward", "z_forward", "update", "smagorinsky", "other"]

    def step_profile(self, nsteps: int = 1) -> dict:
        """Advance nsteps and return device milliseconds per stage (events between stages)."""
        fov, fos = C.c_int32(self.fov), C.c_int32(self.fos)
        ms = np.zeros(8)
        _check(lib().hit3d_gpu_step_profile(self._h, int(nsteps), C.byref(fov), C.byref(fos), _ptr(ms)),
               "step_profile")
        self.fov, self.fos = fov.value, fos.value
        return dict(zip(self.STAGES, ms.tolist()))

    def autotune(self):
        """Pick the fastest launch shape of the fused x pass, then the column tile of
        the strided passes (kept in self.column_tile, times in self.column_ms);
        returns (variant, ms per variant)."""
        v = C.c_int32(0)
        ms = np.full(N_VARIANTS, np.nan)
        _check(lib().hit3d_gpu_autotune(self._h, C.byref(v), _ptr(ms)), "autotune")
        self.column_tile, self.column_ms = self.autotune_columns()
        return v.value, [x for x in ms.tolist() if x == x]

    def autotune_columns(self):
        """Pick the column-tile shape of the strided passes; returns (tile, ms of the 4 shapes)."""
        t = C.c_int32(0)
        ms = np.zeros(4)
        _check(lib().hit3d_gpu_autotune_columns(self._h, C.byref(t), _ptr(ms)), "autotune_columns")
        return t.value, ms.tolist()

    def set_column_tile(self, t: int):
        _check(lib().hit3d_gpu_set_column_tile(self._h, int(t)), "set_column_tile")
        self.column_tile = int(t)

    def set_variant(self, v: int):
        _check(lib().hit3d_gpu_set_variant(self._h, int(v)), "set_variant")

    def nonfinite(self) -> int:
        """Number of non-finite components of the state and the AB2 history (on the device)."""
        v = C.c_int64(0)
        _check(lib().hit3d_gpu_check_finite(self._h, C.byref(v)), "check_finite")
        return int(v.value)

    def les_stats(self) -> dict:
        """les.gp quantities of the last step (dynamic localization model only)."""
        out = np.zeros(4)
        _check(lib().hit3d_gpu_les_stats(self._h, _ptr(out)), "les_stats")
        return dict(zip(("energy", "production", "B", "dissipation"), out.tolist()))

    def set_update_fusion(self, on: bool):
        """Fuse the velocity products' z pass with the update (the default) or not."""
        _check(lib().hit3d_gpu_set_update_fusion(self._h, int(bool(on))), "set_update_fusion")

    def set_pruning(self, on: bool):
        """Allow (default) or forbid 2/3-rule pruning of the step's transforms."""
        _check(lib().hit3d_gpu_set_pruning(self._h, int(bool(on))), "set_pruning")

    @property
    def pruned(self) -> bool:
        """Whether the next step runs pruned transforms (checks the state on the device)."""
        r = lib().hit3d_gpu_pruned(self._h)
        if r < 0:
            _check(r, "pruned")
        return bool(r)

    @property
    def launches(self) -> int:
        """Kernels launched by this context so far."""
        return int(lib().hit3d_gpu_launch_count(self._h))

    @property
    def stream(self) -> int:
        """cudaStream_t of this context (as an integer handle)."""
        return lib().hit3d_gpu_stream(self._h) or 0

    def set_dt(self, dt: float):
        _check(lib().hit3d_gpu_set_dt(self._h, float(dt)), "set_dt")
        self.params.dt = dt

    def set_scalars_active(self, on: bool):
        _check(lib().hit3d_gpu_set_scalars_active(self._h, int(bool(on))), "set_scalars_active")

    def dealias_all(self):
        _check(lib().hit3d_gpu_dealias_all(self._h), "dealias_all")

    def init_velocity(self, rn1: float, isp_type: int = 1, peak_wavenum: float = 4.0, ir_exp: float = 2.0):
        _check(lib().hit3d_gpu_init_velocity(self._h, float(rn1), int(isp_type), float(peak_wavenum),
                                             float(ir_exp)), "init_velocity")

    def stats(self):
        es = np.zeros(self.kmax)
        out = np.zeros(12)
        _check(lib().hit3d_gpu_stats(self._h, _ptr(es), self.kmax, _ptr(out)), "stats")
        return es, dict(zip(self.STAT_KEYS, out.tolist()))

    def scalar_stats(self, s: int):
        sp = np.zeros(self.kmax)
        out = np.zeros(5)
        _check(lib().hit3d_gpu_scalar_stats(self._h, int(s), _ptr(sp), self.kmax, _ptr(out)), "scalar_stats")
        return dict(spectrum=sp, diss=out[0], mean=out[1], variance=out[2], min=out[3], max=out[4])

    def particles_upload(self, xyzp: np.ndarray, uvwp: np.ndarray | None = None, scheme: int = 1):
        xyzp = np.ascontiguousarray(xyzp, dtype=np.float64)
        u = None if uvwp is None else np.ascontiguousarray(uvwp, dtype=np.float64)
        _check(lib().hit3d_gpu_particles_upload(self._h, _ptr(xyzp), None if u is None else _ptr(u),
                                                xyzp.shape[0], int(scheme)), "particles_upload")
        self._np = xyzp.shape[0]

    def init_scalar(self, s: int, rn2: float, peak_wavenum: float = 4.0):
        """init_scalar for passive scalar s (its scalar_type decides the form)."""
        _check(lib().hit3d_gpu_init_scalar(self._h, int(s), float(rn2), float(peak_wavenum)), "init_scalar")

    def particles_filter(self, delta: float):
        """Particles see the velocity filtered with a Gaussian of width delta (0: off)."""
        _check(lib().hit3d_gpu_particles_filter(self._h, float(delta)), "particles_filter")

    def particles_download(self):
        x = np.zeros((self._np, 3))
        u = np.zeros((self._np, 3))
        _check(lib().hit3d_gpu_particles_download(self._h, _ptr(x), _ptr(u)), "particles_download")
        return x, u

    def xfft3d(self, flag: int, a: np.ndarray) -> np.ndarray:
        """xFFT3d on one (nz, ny, nx+2) host array; returns a new array."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        out = np.zeros_like(a)
        _check(lib().hit3d_gpu_xfft3d(self._h, int(flag), _ptr(a), _ptr(out), self.n + 2), "xfft3d")
        return out

    def filter_field(self, kind: int, delta: float, field: int):
        _check(lib().hit3d_gpu_filter_field(self._h, int(kind), float(delta), int(field)), "filter_field")

    def physical_fields(self, nf: int, k2max: float = 0.0) -> np.ndarray:
        """Inverse transforms of the first nf state fields, optionally spherically truncated."""
        out = np.zeros((nf, self.n, self.n, self.n + 2))
        _check(lib().hit3d_gpu_physical_fields(self._h, int(nf), float(k2max), _ptr(out), self.n + 2),
               "physical_fields")
        return out

    def sgs_fields(self, kind: int = 4, delta: float | None = None) -> np.ndarray:
        """(18, nz, ny, nx) float32: filtered velocity, exact subgrid stress, filtered gradients."""
        if delta is None:
            delta = 4.0 * 2.0 * np.pi / self.n
        out = np.empty((18, self.n, self.n, self.n), dtype=np.float32)
        _check(lib().hit3d_gpu_sgs_fields(self._h, int(kind), float(delta),
                                          out.ctypes.data_as(C.POINTER(C.c_float))), "sgs_fields")
        return out

    def sgs_samples(self, kind: int, delta: float, stride: int) -> np.ndarray:
        """sgs_fields on every stride-th point per axis: (18, m, m, m), m = nx / stride."""
        m = self.n // stride
        out = np.empty((18, m, m, m), dtype=np.float32)
        _check(lib().hit3d_gpu_sgs_samples(self._h, int(kind), float(delta), int(stride),
                                           out.ctypes.data_as(C.POINTER(C.c_float))), "sgs_samples")
        return out

    def velocity_rescale(self, isp_type: int, peak_wavenum: float, ir_exp: float = 2.0):
        _check(lib().hit3d_gpu_velocity_rescale(self._h, int(isp_type), float(peak_wavenum), float(ir_exp)),
               "velocity_rescale")

    def physical_velocity(self) -> np.ndarray:
        out = np.zeros((3, self.n, self.n, self.n + 2))
        _check(lib().hit3d_gpu_physical_velocity(self._h, _ptr(out), self.n + 2), "physical_velocity")
        return out

    def les_set_mlp(self, bf16_weights: np.ndarray, delta: float, clip: bool = True, kernel: int = 1):
        """Use trained bf16 weights (uint16 bit patterns) as this context's subgrid model
        (les_model LES_LEARNED = 20); delta is the filter width the network was trained for; kernel 1
        runs the hidden layers on the tensor cores, 0 on the CUDA cores in fp32."""
        w = np.ascontiguousarray(bf16_weights, dtype=np.uint16)
        _check(lib().hit3d_gpu_les_set_mlp(self._h, w.ctypes.data_as(C.POINTER(C.c_uint16)), w.size, float(delta),
                                           int(bool(clip)), int(kernel)), "les_set_mlp")


def _f32(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


class Mlp:
    """The learned subgrid closure on one GPU: parameters, training data, the
    training step and inference (hit3d_mlp_* in the C-ABI)."""

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        _check(lib().hit3d_mlp_create(int(device), int(seed) & (2**64 - 1), C.byref(h)), "hit3d_mlp_create")
        self._h = h
        self.nparam = int(lib().hit3d_mlp_nparam())
        self.delta = None

    def close(self):
        if getattr(self, "_h", None):
            lib().hit3d_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        w = np.empty(self.nparam, dtype=np.float32)
        _check(lib().hit3d_mlp_get_params(self._h, w.ctypes.data_as(_fp)), "hit3d_mlp_get_params")
        return w

    @params.setter
    def params(self, w: np.ndarray):
        w = _f32(w)
        if w.size != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters")
        _check(lib().hit3d_mlp_set_params(self._h, w.ctypes.data_as(_fp)), "hit3d_mlp_set_params")

    def bf16(self) -> np.ndarray:
        w = np.empty(self.nparam, dtype=np.uint16)
        _check(lib().hit3d_mlp_get_bf16(self._h, w.ctypes.data_as(C.POINTER(C.c_uint16))), "hit3d_mlp_get_bf16")
        return w

    def set_data(self, A: np.ndarray, tau: np.ndarray, delta: float):
        """A: (9, P) gradients d u_i/d x_j at row 3i+j; tau: (6, P) stresses (11 12 13 22 23 33)."""
        A = _f32(A).reshape(9, -1)
        tau = _f32(tau).reshape(6, -1)
        if A.shape[1] != tau.shape[1]:
            raise ValueError("A and tau disagree on the number of points")
        _check(lib().hit3d_mlp_set_data(self._h, A.ctypes.data_as(_fp), tau.ctypes.data_as(_fp), A.shape[1],
                                        float(delta)), "hit3d_mlp_set_data")
        self.delta = float(delta)

    def norms(self):
        out = np.zeros(2)
        _check(lib().hit3d_mlp_norms(self._h, _ptr(out)), "hit3d_mlp_norms")
        return float(out[0]), float(out[1])

    def loss_grad(self, idx: np.ndarray, lam: float = 0.0):
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        loss = C.c_float()
        g = np.empty(self.nparam, dtype=np.float32)
        _check(lib().hit3d_mlp_loss_grad(self._h, idx.ctypes.data_as(C.POINTER(_i32)), idx.size, float(lam),
                                         C.byref(loss), g.ctypes.data_as(_fp)), "hit3d_mlp_loss_grad")
        return float(loss.value), g

    def train(self, nsteps: int, batch: int = 16384, lr: float = 1e-3, lam: float = 0.0, seed: int = 1) -> np.ndarray:
        losses = np.empty(max(int(nsteps), 1), dtype=np.float32)
        _check(lib().hit3d_mlp_train(self._h, int(nsteps), int(batch), float(lr), float(lam),
                                     int(seed) & (2**64 - 1), losses.ctypes.data_as(_fp)), "hit3d_mlp_train")
        return losses[:nsteps]

    def predict(self, A: np.ndarray, delta: float | None = None, clip: bool = False, kernel: int = 0) -> np.ndarray:
        A = _f32(A).reshape(9, -1)
        d = self.delta if delta is None else delta
        if d is None:
            raise ValueError("no filter width")
        out = np.empty((6, A.shape[1]), dtype=np.float32)
        _check(lib().hit3d_mlp_predict(self._h, A.ctypes.data_as(_fp), A.shape[1], float(d), int(bool(clip)),
                                       int(kernel), out.ctypes.data_as(_fp)), "hit3d_mlp_predict")
        return out
