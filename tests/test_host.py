"""Host-side pieces that need no GPU: the input-file reader, restart and real*4
file layouts, and their failure paths (my_exit(-1) conditions of the reference)."""
import os
import struct

import numpy as np
import pytest

from hit3d_b200.params import InputFileError, parse_input, read_input_file
from hit3d_b200.restart import RestartError, read_real4, read_restart, write_real4, write_restart

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_reads_sample_input():
    c = read_input_file(os.path.join(GOLDEN, "decay64_.in"))
    assert (c.nx, c.ny, c.nz_all) == (64, 64, 64)
    assert (c.itmin, c.itmax, c.iprint1, c.iprint2, c.iwrite4) == (0, 20, 10, 20, 20)
    assert c.trescale == 0.05 and c.nrescale == 2
    assert c.flow_type == 0 and c.re == 400.0 and c.nu == 1.0 / 400.0
    assert c.dt == 0.005 and not c.variable_dt
    assert (c.isp_type, c.ir_exp, c.peak_wavenum) == (1, 2, 4.0)
    assert c.rn1 == 67748937.0 and c.kmax == 21
    assert c.n_scalars == 2 and c.scalar_type == [0, 0] and c.sc == [0.7, 1.0]
    assert c.pe == [c.nu / 0.7, c.nu / 1.0]


def test_list_directed_reads_span_lines():
    """A scalar line with four values takes the fifth from the next line."""
    text = open(os.path.join(GOLDEN, "decay64_.in")).read()
    text = text.replace("0      0.7     4.0    2.    0.0\n0      1.0     4.0    4.    0.0",
                        "0      0.7     4.0    2.\n 0.25\n0      1.0     4.0    4.    0.0")
    c = parse_input(text)
    assert c.reac_sc == [0.25, 0.0] and c.sc == [0.7, 1.0]


def test_missing_nrescale_defaults_to_one():
    text = open(os.path.join(GOLDEN, "decay64_.in")).read().replace("0.05 2          TRESCALE", "0.05            TRESCALE")
    assert parse_input(text).nrescale == 1


def test_les_forces_two_thirds_rule_and_dealias_kmax():
    text = open(os.path.join(GOLDEN, "decay64_.in")).read()
    c = parse_input(text.replace("0		dealias", "1		dealias"))
    assert c.dealias == 1 and c.kmax == int(np.floor(64 / 3 * np.sqrt(2)))
    c = parse_input(text.replace("0		dealias", "1		dealias").replace("0               les_model", "1               les_model"))
    assert c.dealias == 0


def test_truncated_input_is_an_error():
    text = open(os.path.join(GOLDEN, "decay64_.in")).read()
    with pytest.raises(InputFileError):
        parse_input("\n".join(text.splitlines()[:20]))
    with pytest.raises(InputFileError):
        parse_input(text, numprocs=3)


def test_restart_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    f = rng.standard_normal((5, 8, 8, 10))
    p = str(tmp_path / "run_000001.64.000010")
    write_restart(p, f, 1.25, 0.005, nums=2)
    assert os.path.getsize(p) == 36 + 5 * 8 * 8 * 8 * 8
    with open(p, "rb") as fh:
        assert struct.unpack("<5i2d", fh.read(36)) == (8, 8, 8, 2, 0, 1.25, 0.005)
    g, t, dt, nums, nles = read_restart(p, 8, n_scalars=2)
    assert (t, dt, nums, nles) == (1.25, 0.005, 2, 0)
    assert np.array_equal(g[..., :8], f[..., :8]) and np.all(g[..., 8:] == 0)
    # the input file prevails: fewer scalars drop, more scalars come back as zeros
    g1, *_ = read_restart(p, 8, n_scalars=1)
    assert g1.shape[0] == 4 and np.array_equal(g1[3, ..., :8], f[3, ..., :8])
    g3, *_ = read_restart(p, 8, n_scalars=3)
    assert g3.shape[0] == 6 and np.all(g3[5] == 0)


def test_corrupt_restarts_are_rejected(tmp_path):
    f = np.zeros((3, 8, 8, 10))
    p = str(tmp_path / "r.64.000001")
    write_restart(p, f, 0.0, 0.01, nums=0)
    with pytest.raises(RestartError, match="Dimensions"):
        read_restart(p, 16, 0)
    with open(p, "r+b") as fh:
        fh.truncate(100)
    with pytest.raises(RestartError, match="size"):
        read_restart(p, 8, 0)
    with open(p, "wb") as fh:
        fh.write(b"\x00" * 10)
    with pytest.raises(RestartError, match="truncated"):
        read_restart(p, 8, 0)


def test_real4_layout(tmp_path):
    a = np.arange(4 * 4 * 6, dtype=np.float64).reshape(4, 4, 6)
    p = str(tmp_path / "u.000000")
    write_real4(p, a)
    assert os.path.getsize(p) == 12 + 4 * 4 * 4 * 4
    b = read_real4(p)
    assert np.array_equal(b, a[:, :, :4].astype(np.float32))


def test_spectral_truncate_maps_modes_between_grids():
    """A field made of modes |k_i| < n/2 has the same (rescaled) coefficients on an
    N^3 and an n^3 grid; the reference layout is [ky][kz][kx re/im]."""
    from hit3d_b200.les import spectral_truncate
    rng = np.random.default_rng(0)
    N, n = 16, 8
    modes = [(int(a), int(b), int(c), rng.standard_normal(), rng.standard_normal())
             for a, b, c in rng.integers(-3, 4, size=(12, 3))]

    def ref_layout(m):
        x = np.arange(m) * 2 * np.pi / m
        Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
        f = sum(a * np.cos(kx * X + ky * Y + kz * Z) + b * np.sin(kx * X + ky * Y + kz * Z)
                for kx, ky, kz, a, b in modes)
        F = np.fft.rfftn(f)                # [kz][ky][kx], unnormalised, e^{-i}
        F = F.transpose(1, 0, 2)           # [ky][kz][kx]
        out = np.zeros((1, m, m, m + 2))
        out[0, ..., 0::2], out[0, ..., 1::2] = F.real, F.imag
        return out

    got = spectral_truncate(ref_layout(N), n)
    want = ref_layout(n)
    want[..., n // 2 * 2:] = 0.0  # kx Nyquist column is not carried over
    assert np.abs(got - want).max() < 1e-9 * np.abs(want).max()


def test_sidecar_keys_and_defaults(tmp_path):
    from hit3d_b200.sidecar import GpuSettings, parse_sidecar, read_sidecar
    assert read_sidecar(str(tmp_path), "nosuchrun") == GpuSettings()
    s = parse_sidecar("""
        # settings beyond the .in file
        precision = 1
        Pruning = off       # keys are case-insensitive
        variant = 5
        device = 0
        c_smag = 0.16
        les_model = 20
        les_mlp = closure.npy
        les_mlp_delta = 0.39
        les_mlp_clip = off
        les_mlp_kernel = 0
        nonfinite_check = off
    """)
    assert (s.precision, s.pruning, s.variant, s.c_smag, s.les_model, s.les_mlp) == (1, False, 5, 0.16, 20, "closure.npy")
    assert (s.les_mlp_delta, s.les_mlp_clip, s.les_mlp_kernel, s.nonfinite_check) == (0.39, False, 0, False)
    assert parse_sidecar("variant = auto").variant is None


@pytest.mark.parametrize("text,msg", [
    ("precision = 2", "precision"),
    ("speed = 11", "unknown key"),
    ("variant = 15", "variant"),
    ("pruning = maybe", "on/off"),
    ("precision", "key = value"),
    ("precision = 1\nprecision = 0", "twice"),
    ("c_smag = -0.1", "positive"),
    ("les_model = 8", "not supported"),
    ("les_model = 20", "les_mlp"),
    ("device =", "no value"),
])
def test_sidecar_errors_name_the_line(text, msg):
    from hit3d_b200.sidecar import SidecarError, parse_sidecar
    with pytest.raises(SidecarError, match=msg):
        parse_sidecar(text, "run.gpu.in")


def test_particle_lattice_and_restart_file(tmp_path):
    """particles_init's lattice (m_particles.f90:195-226) and the pt.<ext> binary
    layout (m_particles.f90:620-640): int64 nptot, (int32 id, 3 x float64) per
    particle in physical units, float64 TIME."""
    from hit3d_b200 import particles as pt
    ip, phys = pt.lattice(30, 32)                 # nearer cube: 27
    assert len(ip) == 27 and ip[0] == 1 and ip[-1] == 27
    step = 2 * np.pi / 3
    assert np.allclose(phys[0], [0.5 * step] * 3) and np.allclose(phys[1], [1.5 * step, 0.5 * step, 0.5 * step])
    assert len(pt.lattice(35, 32)[0]) == 27 and len(pt.lattice(50, 32)[0]) == 64
    grid = pt.to_grid(phys, 32)
    assert np.allclose(grid, phys / (2 * np.pi / 32) + 1.0)
    assert np.allclose(pt.to_grid(np.array([[-0.5, 2 * np.pi + 0.25, 1.0]]), 32),
                       np.array([[2 * np.pi - 0.5, 0.25, 1.0]]) / (2 * np.pi / 32) + 1.0)
    path = str(tmp_path / "pt.000010")
    pt.write_pt(path, ip, grid, 32, 0.125)
    raw = open(path, "rb").read()
    assert len(raw) == 8 + 27 * 28 + 8 and struct.unpack_from("<q", raw)[0] == 27
    ip2, grid2, t = pt.read_pt(path, 32)
    assert np.array_equal(ip2, ip) and np.allclose(grid2, grid, rtol=0, atol=1e-12) and t == 0.125
    open(path, "r+b").truncate(100)
    with pytest.raises(pt.ParticleFileError, match="truncated"):
        pt.read_pt(path, 32)


def test_particle_trajectory_line_format(tmp_path):
    from hit3d_b200 import particles as pt
    pt.append_trajectories(str(tmp_path), 12, 0.06, np.array([7], dtype=np.int32),
                           np.array([[1.0, 2.0, 3.0]]), np.array([[0.5, -0.25, 1e-3]]), 32)
    line = open(tmp_path / "p.0007").read().rstrip("\n")
    assert line.startswith("000012    0")
    vals = [float(line[11 + 16 * k: 11 + 16 * (k + 1)]) for k in range(7)]
    dx = 2 * np.pi / 32
    assert np.allclose(vals, [0.06, 0.0, dx, 2 * dx, 0.5, -0.25, 1e-3], rtol=1e-7)


def test_restart_header_checks(tmp_path):
    from hit3d_b200.restart import read_restart_header
    f = np.zeros((4, 8, 8, 10))
    p = str(tmp_path / "r")
    write_restart(p, f, 2.5, 0.01, 1)
    assert read_restart_header(p, 8) == (8, 8, 8, 1, 0, 2.5, 0.01)
    with pytest.raises(RestartError, match="Dimensions"):
        read_restart_header(p, 16)
    with open(p, "ab") as fh:
        fh.write(b"\0" * 8)
    with pytest.raises(RestartError, match="size"):
        read_restart_header(p, 8)
    with open(p, "wb") as fh:
        fh.write(b"\0" * 12)
    with pytest.raises(RestartError, match="truncated"):
        read_restart_header(p, 8)
