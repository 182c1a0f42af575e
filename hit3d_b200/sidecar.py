"""Settings that have no place in the reference's positional input file.

The reference reads everything from `<run_name>.in` (m_parameters.f90:172-512),
whose layout is positional: a new line would shift every later read.  The
settings of this implementation therefore live in a second file,
`<run_name>.gpu.in`, beside it, so that `.in` files stay byte-compatible
between the two codes.  Absent file: every key takes its default.

Format: one `key = value` per line; `#` starts a comment; blank lines are
ignored; keys are case-insensitive.  An unknown key or a bad value is an
error that names the line, as a bad `.in` line is in the reference.

  precision       0 | 1        FP64 transforms | FP32 transforms (FP64 state)
  pruning         on | off     skip work on the modes the 2/3 rule discards
  variant         auto | 0..12 launch shape of the fused row pass; auto tunes
  device          int          CUDA device ordinal
  c_smag          float        Smagorinsky constant (the reference fixes 0.18)
  les_model       int          overrides the `.in` LES model; 20 is the learned
                               closure (the 2/3 rule is then forced, as for
                               every LES model of the reference)
  les_mlp         path         bf16 weights of the learned closure: a .npy
                               array of uint16 bit patterns (relative paths are
                               taken from the run directory)
  les_mlp_delta   float        filter width the closure was trained for
                               (default 2 dx)
  les_mlp_clip    on | off     remove backscatter from the predicted stress
  les_mlp_kernel  0 | 1        hidden layers on the CUDA cores (fp32) or on
                               the tensor cores (bf16, fp32 accumulation)
  nonfinite_check on | off     device count of non-finite modes at every
                               statistics step (a run that diverged ends
                               with exit reason -2)
"""
from __future__ import annotations

import os
from dataclasses import dataclass, fields
from typing import Optional


class SidecarError(ValueError):
    """A line of `<run_name>.gpu.in` that cannot be used."""


@dataclass
class GpuSettings:
    precision: int = 0
    pruning: bool = True
    variant: Optional[int] = None      # None: the tuner picks
    device: int = 0
    c_smag: float = 0.18
    les_model: Optional[int] = None    # None: the `.in` file's model
    les_mlp: Optional[str] = None
    les_mlp_delta: Optional[float] = None
    les_mlp_clip: bool = True
    les_mlp_kernel: int = 1
    nonfinite_check: bool = True


def _flag(v: str) -> bool:
    s = v.lower()
    if s in ("on", "true", "yes", "1"):
        return True
    if s in ("off", "false", "no", "0"):
        return False
    raise ValueError(f"expected on/off, got {v!r}")


def _choice(*allowed):
    def conv(v: str) -> int:
        x = int(v)
        if x not in allowed:
            raise ValueError(f"expected one of {allowed}, got {x}")
        return x
    return conv


def _variant(v: str) -> Optional[int]:
    if v.lower() == "auto":
        return None
    from .gpu import N_VARIANTS
    return _choice(*range(N_VARIANTS))(v)


def _les_model(v: str) -> int:
    x = int(v)
    if x not in (0, 1, 2, 3, 4, 5, 6, 7, 10, 20):
        raise ValueError(f"les_model {x} is not supported (0-7, 10 or 20)")
    return x


def _positive(v: str) -> float:
    x = float(v)
    if not x > 0.0:
        raise ValueError(f"expected a positive number, got {v!r}")
    return x


_CONVERT = {
    "precision": _choice(0, 1),
    "pruning": _flag,
    "variant": _variant,
    "device": int,
    "c_smag": _positive,
    "les_model": _les_model,
    "les_mlp": str,
    "les_mlp_delta": _positive,
    "les_mlp_clip": _flag,
    "les_mlp_kernel": _choice(0, 1),
    "nonfinite_check": _flag,
}
assert set(_CONVERT) == {f.name for f in fields(GpuSettings)}


def parse_sidecar(text: str, name: str = "<sidecar>") -> GpuSettings:
    s = GpuSettings()
    seen = set()
    for no, raw in enumerate(text.splitlines(), 1):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if "=" not in line:
            raise SidecarError(f"{name}:{no}: expected 'key = value', got {raw.strip()!r}")
        key, val = (t.strip() for t in line.split("=", 1))
        key = key.lower()
        if key not in _CONVERT:
            raise SidecarError(f"{name}:{no}: unknown key {key!r}")
        if key in seen:
            raise SidecarError(f"{name}:{no}: {key!r} given twice")
        if not val:
            raise SidecarError(f"{name}:{no}: {key!r} has no value")
        try:
            setattr(s, key, _CONVERT[key](val))
        except ValueError as e:
            raise SidecarError(f"{name}:{no}: {key}: {e}") from e
        seen.add(key)
    if s.les_model == 20 and s.les_mlp is None:
        raise SidecarError(f"{name}: les_model 20 (learned closure) needs les_mlp weights")
    return s


def sidecar_path(workdir: str, run_name: str) -> str:
    return os.path.join(workdir, run_name + ".gpu.in")


def read_sidecar(workdir: str, run_name: str) -> GpuSettings:
    """The settings of `<run_name>.gpu.in` in workdir, or the defaults if it is absent."""
    p = sidecar_path(workdir, run_name)
    if not os.path.exists(p):
        return GpuSettings()
    with open(p) as fh:
        return parse_sidecar(fh.read(), p)
