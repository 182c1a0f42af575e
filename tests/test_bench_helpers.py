"""Host-side helpers of bench.py that need no GPU: the FP32-form E(k) error per
energy band of shells and the stage byte model."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_ek_error_bands():
    # peak shell 1.0; shells at 1e-1, 1e-3, 1e-5, 1e-7, 1e-9, 1e-11 of it
    e64 = np.array([1.0, 1e-1, 1e-3, 1e-5, 1e-7, 1e-9, 1e-11])
    rel = np.array([1e-9, 2e-9, 3e-8, 4e-7, 5e-6, 6e-5, 7e-4])
    e32 = e64 * (1.0 + rel)
    out = bench.ek_err_by_decade(e32, e64)
    assert list(out) == ["1e-2", "1e-4", "1e-6", "1e-8", "1e-10", "1e-12"]
    want = {"1e-2": 2e-9, "1e-4": 3e-8, "1e-6": 4e-7, "1e-8": 5e-6, "1e-10": 6e-5, "1e-12": 7e-4}
    for k, v in want.items():
        assert abs(out[k] - v) <= 1e-6 * v, (k, out[k], v)


def test_ek_error_bands_empty_band_is_none():
    e64 = np.array([1.0, 0.5])
    out = bench.ek_err_by_decade(e64.copy(), e64)
    assert out["1e-2"] == 0.0 and out["1e-4"] is None and out["1e-12"] is None


def test_stage_bytes_fp32_halves_the_work_fields():
    n = 512
    f64 = bench.stage_units(n, 0, True)
    f32 = bench.stage_units(n, 1, True)
    # the x pass and the y passes touch only work fields: half in the FP32 form
    for k in ("x_fused", "y_inverse", "y_forward", "z_forward"):
        assert abs(f32[k] - 0.5 * f64[k]) <= 1e-12 * f64[k]
    # the update reads and writes the FP64 state in both forms
    assert f32["update"] > 0.5 * f64["update"]
    assert abs(sum(f64.values()) - 27.9) < 0.1


def _rank_max(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r "took" 1.5 + r seconds for 60 steps; the job takes the slowest rank's time
        t = bench.max_over_ranks(dist, 1.5 + rank, device="cpu")
        q.put((rank, t, world * 60 / t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    """The replicas' timing of bench.py --gpus N (one all_reduce(MAX) of the
    timing scalar, value = N x steps / max time), with two gloo ranks on CPU."""
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_max, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]
    assert all(abs(o[2] - 2 * 60 / 2.5) < 1e-12 for o in out)
    assert bench.max_over_ranks(None, 3.25) == 3.25
