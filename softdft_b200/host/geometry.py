"""Cartesian slit geometry: grid size, walls and wall charges.

Restates `src/geometry/setup/coordinate_system/Cartesian/create_cartesian.jl:42-68`
(grid rule ``NP = cld(L, dz) + 1``), `process_cartesian.jl:14-45` (mirrored,
offset 0) and the hard/charged wall parsers in `external_fields/hard_walls.jl:26-49`
and `external_fields/charged_walls.jl:36-87`.  Only the 1D slit is supported by
the device solve; 2D/3D grids raise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction
from typing import List, Optional

from .yamlio import as_float


def cld(x: float, y: float) -> int:
    """Julia's ``cld`` on Float64 operands: the ceiling of the exact quotient of
    the two binary64 values."""
    q = Fraction(x) / Fraction(y)
    return math.ceil(q)


def julia_round(x: float) -> int:
    """``round(Int, x)``: round half to even, as Julia does."""
    return int(round(x))


@dataclass
class CartesianGrid:
    dimensions: float            # slit width H (the z extent)
    bin_width: float             # dz
    NP: int
    mirrored: bool = True
    offset: int = 0
    total_charge: float = 0.0
    hard_walls: Optional[List[float]] = None        # [lo, hi] wall positions
    charged_walls: Optional[List[float]] = None     # [lo, hi] positions
    wall_charges: List[float] = field(default_factory=lambda: [0.0, 0.0])

    @property
    def NP_star(self) -> int:
        return (self.NP + 2 * self.offset) * (2 if self.mirrored else 1)


def _listed(v) -> list:
    """The entries a Julia `for x in v` loop visits: a list's items, or a
    scalar itself."""
    if isinstance(v, (list, tuple)):
        return list(v)
    if isinstance(v, dict):
        raise ValueError("expected a list")
    return [v]


def geometry_system(dataset: dict) -> CartesianGrid:
    geom = dataset.get("geometry")
    if geom is None:
        raise ValueError("Missing required section: 'geometry'.")
    cs = geom.get("coordinate_system")
    if cs is None:
        raise ValueError("Missing required key: 'coordinate_system' under 'geometry'.")
    if str(cs) != "Cartesian":
        raise ValueError(f"Unknown coordinate system: {cs}. Supported: Cartesian.")
    if "dimensions" not in geom or "bin_width" not in geom:
        raise ValueError("Please specify both `dimensions` and `bin_width` under `geometry`.")
    dims = [as_float(x) for x in geom["dimensions"]]
    bins = [as_float(x) for x in geom["bin_width"]]
    if len(dims) != len(bins):
        raise ValueError("Mismatch in number of `dimensions` and `bin_width` entries.")
    if len(dims) != 1:
        raise NotImplementedError("only the 1D Cartesian slit is supported by the device solve")
    H, dz = dims[0], bins[0]
    NP = cld(H, dz) + 1
    g = CartesianGrid(dimensions=H, bin_width=dz, NP=NP)
    ext = geom.get("external_field") or {}
    for name, desc in ext.items():
        if name == "hard_walls":
            d = desc.get("dims") if isinstance(desc, dict) else None
            if d is None:
                raise ValueError("Missing 'dims' key in external_field[:hard_walls].")
            for dim in _listed(d):
                if int(dim) != 1:
                    raise ValueError(f"Invalid dimension index: {dim}")
                g.hard_walls = [0.0, H]
        elif name == "charged_walls":
            d = desc.get("dims")
            if d is None:
                raise ValueError("Please specify the dimensions using 'dims: [i, j, ...]'.")
            ch = desc.get("charge")
            if ch is None:
                raise ValueError("Please specify wall charges under 'charge'.")
            d = _listed(d)
            if len(ch) > 0 and not isinstance(ch[0], (list, tuple)):
                ch = [ch]
            if len(ch) != len(d):
                raise ValueError("Mismatch: number of charge entries does not match dims.")
            for i, dim in enumerate(d):
                if int(dim) != 1:
                    raise ValueError(f"Invalid dimension index in dims: {d}")
                qL, qR = as_float(ch[i][0]), as_float(ch[i][1])
                g.charged_walls = [0.0, H]
                g.wall_charges = [qL, qR]
                g.total_charge += qL + qR
        else:
            raise NotImplementedError(f"external field '{name}' is not supported by the device solve")
    return g
