"""hit3d_gpu_xfft3d_static: the forward transform that allocates nothing.

Callers whose device memory is owned by their own pool allocator, or that must
not risk the synchronisation cudaMalloc can cause, pass device input and output
buffers and get the same result as hit3d_gpu_xfft3d, with the library's only
scratch held in a static __device__ array.  This file is collected last so that a
run stopping at its first failure has already run every other test; it must also
pass on its own in a fresh process, where its first call does the per-device
set-up.
"""
import ctypes as C

import numpy as np
import pytest

from _cases import relerr

pytestmark = pytest.mark.gpu


def _call_static(n, a_host):
    import torch
    from hit3d_b200 import gpu
    L = gpu.lib()
    d_in = torch.from_numpy(a_host).cuda()
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    rc = L.hit3d_gpu_xfft3d_static(n, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), None)
    assert rc == 0, L.hit3d_gpu_last_error().decode()
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


@pytest.mark.parametrize("n", [32, 48, 64, 128])
def test_static_matches_context_transform_twice(n):
    from hit3d_b200 import Context, Params
    rng = np.random.default_rng(1234 + n)
    g = Context(Params(nx=n))
    for call in range(2):  # two calls in a row: the shared scratch must not leak between them
        a = np.zeros((n, n, n + 2))
        a[:, :, :n] = rng.standard_normal((n, n, n))
        ref = g.xfft3d(1, a)
        out = _call_static(n, a)
        assert relerr(out, ref) < 1e-13, f"call {call}"
    g.close()


@pytest.mark.parametrize("n", [32, 128])
def test_static_in_place(n):
    """Input and output the same device buffer: the whole input reaches the
    scratch array before anything is written back."""
    import torch
    from hit3d_b200 import Context, Params, gpu
    rng = np.random.default_rng(77 + n)
    a = np.zeros((n, n, n + 2))
    a[:, :, :n] = rng.standard_normal((n, n, n))
    g = Context(Params(nx=n))
    ref = g.xfft3d(1, a)
    g.close()
    d = torch.from_numpy(a).cuda()
    torch.cuda.synchronize()
    L = gpu.lib()
    rc = L.hit3d_gpu_xfft3d_static(n, C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), None)
    assert rc == 0, L.hit3d_gpu_last_error().decode()
    torch.cuda.synchronize()
    assert relerr(d.cpu().numpy(), ref) < 1e-13


def test_static_rejects_sizes_beyond_the_limit():
    from hit3d_b200 import gpu
    L = gpu.lib()
    rc = L.hit3d_gpu_xfft3d_static(256, C.c_void_p(16), C.c_void_p(32), None)
    assert rc != 0
    assert b"N <= 128" in L.hit3d_gpu_last_error()
