"""CPU checks of the C-ABI boundary: the library loads, exports every entry point
declared in include/hit3d_gpu.h, the ctypes struct matches the C struct, and
calls that need no GPU fail cleanly with an error message."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hit3d_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hit3d_(?:gpu|batch|mlp)_\w+)\s*\(", text)))


def test_header_declares_every_binding():
    from hit3d_b200 import gpu
    bound = sorted(name for name, _, _ in gpu.SIGNATURES)
    assert bound == declared_functions()


def test_library_exports_every_declared_symbol():
    from hit3d_b200 import build
    build.build()
    L = C.CDLL(build.LIB)
    for name in declared_functions():
        assert hasattr(L, name), name


def test_params_struct_layout_matches_c(tmp_path):
    """Compile a C probe against the header and compare sizeof/offsetof."""
    from hit3d_b200.gpu import _Params
    src = tmp_path / "probe.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "hit3d_gpu.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu\\n\", sizeof(hit3d_params),"
        " offsetof(hit3d_params, scalar_type), offsetof(hit3d_params, device),"
        " offsetof(hit3d_params, nu), offsetof(hit3d_params, sc));"
        " printf(\"%zu %zu %zu\\n\", offsetof(hit3d_params, c_t), offsetof(hit3d_params, c_mixed),"
        " offsetof(hit3d_params, reac_sc)); return 0;}\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [C.sizeof(_Params), _Params.scalar_type.offset, _Params.device.offset, _Params.nu.offset,
           _Params.sc.offset, _Params.c_t.offset, _Params.c_mixed.offset, _Params.reac_sc.offset]
    assert [int(x) for x in out] == got


def test_null_arguments_return_errors():
    from hit3d_b200 import gpu
    L = gpu.lib()
    assert L.hit3d_gpu_init(None, None) != 0
    assert b"null" in L.hit3d_gpu_last_error()
    assert L.hit3d_gpu_step(None, 1, None, None, None) != 0
    assert L.hit3d_gpu_set_dt(None, 0.1) != 0


def test_unsupported_size_rejected_before_device_use():
    from hit3d_b200 import Hit3dError, Params, Context
    with pytest.raises(Hit3dError, match="grid size"):
        Context(Params(nx=100))


def test_reference_les_models_without_a_port_are_rejected():
    """The reference has no LES models 8 and 9 (m_les.f90:364-368 stops on them):
    an input asking for one fails at init."""
    from hit3d_b200 import Hit3dError, Params, Context
    for m in (8, 9, 11):
        with pytest.raises(Hit3dError, match="les_model"):
            Context(Params(nx=32, les_model=m))


def test_forcing_band_checks_before_device_use():
    """A forced run needs KFMAX >= 1, and any wider band passes the parameter
    checks (the reference reads any value, m_parameters.f90:308); without a
    GPU such a context then fails only at device use."""
    from hit3d_b200 import Hit3dError, Params, Context
    with pytest.raises(Hit3dError, match="kfmax"):
        Context(Params(nx=32, flow_type=1, force_type=1, kfmax=0))
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(Hit3dError) as e:
            Context(Params(nx=32, flow_type=1, force_type=1, kfmax=100))
        assert "kfmax" not in str(e.value)
