"""input.yaml loading with the number rules the reference's YAML reader applies.

The reference loads its request file with YAML.jl (`src/iDFT/iDFT.jl:24`), whose
resolver reads exponent literals such as ``1e-6`` as floats.  PyYAML's default
resolver follows YAML 1.1 and keeps them as strings, so a resolver for the
YAML 1.2 float form is added here.
"""
from __future__ import annotations

import math
import re

import yaml


class _Loader(yaml.SafeLoader):
    pass


_FLOAT_RE = re.compile(
    r"""^(?:[-+]?(?:[0-9][0-9_]*)\.[0-9_]*(?:[eE][-+]?[0-9]+)?
        |[-+]?(?:[0-9][0-9_]*)(?:[eE][-+]?[0-9]+)
        |\.[0-9_]+(?:[eE][-+]?[0-9]+)?
        |[-+]?\.(?:inf|Inf|INF)
        |\.(?:nan|NaN|NAN))$""",
    re.X,
)

_Loader.add_implicit_resolver("tag:yaml.org,2002:float", _FLOAT_RE, list("-+0123456789."))


def load_text(text: str) -> dict:
    data = yaml.load(text, Loader=_Loader)
    if not isinstance(data, dict):
        raise ValueError("input.yaml must hold a mapping at the top level")
    return data


def load_file(path: str) -> dict:
    with open(path, "r", encoding="utf-8") as fh:
        return load_text(fh.read())


def as_float(v) -> float:
    """Float64(v) for numbers, parse(Float64, string(v)) otherwise
    (`src/iDFT/setup/setup_steps/process_numerical.jl:17-28`)."""
    if isinstance(v, bool):
        return float(v)
    if isinstance(v, (int, float)):
        return float(v)
    return float(str(v))


def numerics_int(num: dict, key: str, default: int, clamp: bool) -> int:
    """Int(x) of `src/NonlinearSolvers/fixed_point/AndersonMixing.jl:74-79`: a
    finite integral value, or an error.  max_iters beyond the int32 field is
    clamped (a count that large is never reached); anderm must fit."""
    v = float(num.get(key, default))
    lo, hi = -2 ** 31, 2 ** 31 - 1
    if not math.isfinite(v) or v != math.floor(v) or (not clamp and not lo <= v <= hi):
        raise ValueError(f"numerical.{key} must be an integer")
    return int(min(max(v, lo), hi))
