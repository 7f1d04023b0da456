"""Result files of a solve, in the reference's text formats.

Restates the analysis writers of `src/iDFT/evaluation/analysis/`:
`print_array.jl` (write_scalar_value, write_field_array, write_segment_array,
write_state_fraction_profiles), `degree_of_dissociation.jl`
(write_total_state_fractions), `output_arrays.jl`, `contact_value_theorem.jl`
with the hard- and charged-wall contributions
(`coordinate_system/Cartesian/external_fields/hard_walls.jl:49-78`,
`charged_walls.jl:60-79`), `brush_height.jl` and `analysis.jl`
(call_analysis).  The routines (`routines/adjust_pH.jl:246-311`) parse these
files back, so names, headers, column order and number formatting follow the
reference: numbers print as Julia prints a Float64 (the shortest digits that
round-trip; scientific form `d.ddde-N` below 1e-4 and from 1e6 on, otherwise
plain decimal with at least one fractional digit), grid indices are 1-based.

The array writers take host arrays in the reference's layout (grid index
first); `output_arrays` and `call_analysis` fetch them from a solved request.
"""
from __future__ import annotations

import math
import os
from decimal import Decimal
from typing import Optional, Sequence

import numpy as np

from .host.geometry import julia_round


def jl(x) -> str:
    """A number as Julia's `print` writes it (Float64: shortest round-trip digits)."""
    if isinstance(x, (int, np.integer)) and not isinstance(x, (bool, np.bool_)):
        return str(int(x))
    if isinstance(x, str):
        return x
    v = float(x)
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "Inf" if v > 0 else "-Inf"
    if v == 0.0:
        return "-0.0" if math.copysign(1.0, v) < 0 else "0.0"
    sign = "-" if v < 0 else ""
    t = Decimal(repr(abs(v))).as_tuple()
    digits = "".join(str(d) for d in t.digits).rstrip("0") or "0"
    # value = 0.d1d2... * 10^(E+1), i.e. d1.d2... * 10^E
    E = len(t.digits) + t.exponent - 1
    if E < -4 or E >= 6:
        mant = digits[0] + "." + (digits[1:] or "0")
        return f"{sign}{mant}e{E}"
    if E >= 0:
        ip = digits[: E + 1].ljust(E + 1, "0")
        fp = digits[E + 1:] or "0"
        return f"{sign}{ip}.{fp}"
    return f"{sign}0.{'0' * (-E - 1)}{digits}"


def write_scalar_value(value: float, filename: str, label: Optional[str] = None) -> None:
    """print_array.jl:1-9."""
    with open(filename, "w") as fh:
        fh.write((jl(value) if label is None else f"{label}: {jl(value)}") + "\n")


def write_field_array(arr, filename: str, names: Optional[Sequence[str]] = None) -> None:
    """print_array.jl:11-38 for a 1D grid: one row per grid point, index then values."""
    a = np.asarray(arr, dtype=np.float64)
    if a.ndim == 1:
        a = a[:, None]
    with open(filename, "w") as fh:
        if names is not None:
            fh.write("Index_1  " + " ".join(names) + "\n")
        for K in range(a.shape[0]):
            fh.write(f"{K + 1}  " + " ".join(jl(v) for v in a[K]) + "\n")


def _state_columns(family, monomers):
    return [f"seg{g + 1}_{monomers[st]}" for g, fam in enumerate(family) for st in fam]


def write_segment_array(rho_segments, molsys, directory: str = ".") -> None:
    """print_array.jl:40-89: rho_segments_<species>.txt for species with more than one segment."""
    for u, (rho, cfg) in enumerate(zip(rho_segments, molsys.configurations)):
        fam = cfg.state_family
        if len(fam) <= 1:
            continue
        path = os.path.join(directory, "rho_segments_" + molsys.species[u] + ".txt")
        with open(path, "w") as fh:
            fh.write("Index_1  " + " ".join(_state_columns(fam, molsys.monomers)) + "\n")
            for K in range(rho.shape[0]):
                vals = [rho[K, i, g] for g, f in enumerate(fam) for i in range(len(f))]
                fh.write(f"{K + 1}  " + " ".join(jl(v) for v in vals) + "\n")


def write_state_fraction_profiles(rho_segments, molsys, directory: str = ".", prefix: str = "state_fraction_") -> None:
    """print_array.jl:92-152: per grid point and segment, each state's share."""
    for u, (rho, cfg) in enumerate(zip(rho_segments, molsys.configurations)):
        fam = cfg.state_family
        if not any(len(f) > 1 for f in fam):
            continue
        path = os.path.join(directory, prefix + molsys.species[u] + ".txt")
        with open(path, "w") as fh:
            fh.write("Index_1  " + " ".join(_state_columns(fam, molsys.monomers)) + "\n")
            for K in range(rho.shape[0]):
                vals = []
                for g, f in enumerate(fam):
                    loc = [rho[K, i, g] for i in range(len(f))]
                    den = 0.0
                    for v in loc:
                        den += v
                    vals += [v / den for v in loc] if den > 0 else [0.0] * len(loc)
                fh.write(f"{K + 1}  " + " ".join(jl(v) for v in vals) + "\n")


def write_total_state_fractions(rho_segments, molsys, directory: str = ".",
                                prefix: str = "total_state_fractions_") -> None:
    """degree_of_dissociation.jl:1-78: per dissociating segment the state
    fractions of the summed profile (no trapezoid weights), then their average."""
    for u, (rho, cfg) in enumerate(zip(rho_segments, molsys.configurations)):
        fam = cfg.state_family
        if not any(len(f) > 1 for f in fam):
            continue
        S = max(len(f) for f in fam)
        sums = [0.0] * S
        cnt = [0] * S
        path = os.path.join(directory, prefix + molsys.species[u] + ".txt")
        with open(path, "w") as fh:
            fh.write("segment " + " ".join(f"state{n + 1}" for n in range(S)) + "\n")
            for g, f in enumerate(fam):
                ns = len(f)
                if ns == 1:
                    continue
                loc = []
                for i in range(ns):
                    t = 0.0
                    for v in rho[:, i, g]:
                        t += float(v)
                    loc.append(t)
                tot = 0.0
                for v in loc:
                    tot += v
                normed = [v / tot for v in loc] if tot > 0 else [0.0] * ns
                for j in range(ns):
                    sums[j] += normed[j]
                    cnt[j] += 1
                padded = [jl(v) for v in normed] + [""] * (S - ns)
                fh.write(f"{g + 1} " + " ".join(padded) + "\n")
            fh.write("\n# Average state fractions across all dissociating segments:\n")
            avg = [jl(sums[j] / cnt[j]) if cnt[j] > 0 else "" for j in range(S)]
            fh.write("avg " + " ".join(avg) + "\n")


def trapez_weights(geometry, diameters) -> np.ndarray:
    """(NP, NB) trapezoid weights of hard walls (hard_walls.jl:6-46): 1/2 at the
    contact grid point of each bead type, 1 elsewhere."""
    P, dz = geometry.NP, geometry.bin_width
    tr = np.ones((P, len(diameters)))
    if geometry.hard_walls:
        lo_w, hi_w = geometry.hard_walls
        for j, d in enumerate(diameters):
            lo = julia_round((lo_w + d / 2.0) / dz) + 1
            hi = julia_round((hi_w - d / 2.0) / dz) + 1
            for idx in (lo, hi):
                if 1 <= idx <= P:
                    tr[idx - 1, j] = 0.5
    return tr


def contact_value_theorem_arrays(rho_beads, molsys, geometry) -> np.ndarray:
    """contact_value_theorem.jl:5-20 for the 1D slit: [lo wall, hi wall] sums of
    the hard-wall contact densities (hard_walls.jl:49-78) and the charged-wall
    terms -2 pi lB q^2 (charged_walls.jl:60-79)."""
    contr = np.zeros(2)
    dz, P = geometry.bin_width, geometry.NP
    if geometry.hard_walls:
        lo_w, hi_w = geometry.hard_walls
        hw = np.zeros(2)
        for j, d in enumerate(molsys.diameters):
            lo = julia_round((lo_w + d / 2.0) / dz) + 1
            hi = julia_round((hi_w - d / 2.0) / dz) + 1
            if 1 <= lo <= P:
                hw[0] += rho_beads[lo - 1, j]
            if 1 <= hi <= P:
                hw[1] += rho_beads[hi - 1, j]
        contr += hw
    if geometry.charged_walls:
        lB = molsys.bjerrum_length
        q = geometry.wall_charges
        contr += np.array([-2.0 * math.pi * lB * q[0] ** 2, -2.0 * math.pi * lB * q[1] ** 2])
    return contr


def write_cvt(contr, filename: str) -> None:
    with open(filename, "w") as fh:
        fh.write("# Contact Value Theorem results\n")
        fh.write(f"dim1  {jl(contr[0])}  {jl(contr[1])}\n")


def brush_height_values(rho_segments, molsys, geometry, fixed_coord) -> dict:
    """brush_height.jl:1-64: 2 <z> per species with a fixed segment; fixed
    segments weigh rho/dz, free ones rho * trapez."""
    P, dz = geometry.NP, geometry.bin_width
    z = np.arange(P) * dz
    tr = trapez_weights(geometry, molsys.diameters)
    out = {}
    for u, cfg in enumerate(molsys.configurations):
        fixed = np.asarray(fixed_coord[u]) >= 0
        if not fixed.any():
            continue
        rho = rho_segments[u]
        num = den = 0.0
        for g, fam in enumerate(cfg.state_family):
            for i, st in enumerate(fam):
                w = rho[:, i, g] / dz if fixed[g] else rho[:, i, g] * tr[:, st]
                for K in range(P):
                    num += w[K] * z[K]
                    den += w[K]
        out[molsys.species[u]] = 2.0 * num / den if den > 0 else 0.0
    return out


def write_brush_height(values: dict, filename: str) -> None:
    if not values:
        return
    with open(filename, "w") as fh:
        fh.write("# Brush heights per species (computed as 2 * <z>)\n")
        fh.write("# Format: species brush_height\n")
        for name, h in values.items():
            fh.write(f"{name} {jl(h)}\n")


# ---- from a solved request ----------------------------------------------------

def output_arrays(dft, directory: str = ".") -> None:
    """output_arrays.jl:1-9."""
    from .api import densities
    ms = dft.bulk_system.molsys
    segs, beads, _ = densities(dft)
    _, _, psi, _ = dft.state
    write_field_array(psi, os.path.join(directory, "MEP.txt"), names=["MEP"])
    write_field_array(beads, os.path.join(directory, "rho_beads_K.txt"), names=list(ms.monomers))
    write_segment_array(segs, ms, directory)
    write_state_fraction_profiles(segs, ms, directory)
    write_total_state_fractions(segs, ms, directory)


def contact_value_theorem(dft, directory: str = ".") -> np.ndarray:
    from .api import densities
    _, beads, _ = densities(dft)
    contr = contact_value_theorem_arrays(beads, dft.bulk_system.molsys, dft.geometry)
    write_cvt(contr, os.path.join(directory, "cvt.txt"))
    return contr


def brush_height(dft, directory: str = ".") -> dict:
    from .api import densities
    segs, _, _ = densities(dft)
    vals = brush_height_values(segs, dft.bulk_system.molsys, dft.geometry, dft.descriptor.fixed_coord)
    write_brush_height(vals, os.path.join(directory, "brush_height.txt"))
    return vals


def call_analysis(dft, directory: str = ".") -> None:
    """analysis.jl:9-15: cvt.txt, grand_potential.txt, brush_height.txt and the arrays."""
    from .api import grand_potential
    os.makedirs(directory, exist_ok=True)
    contact_value_theorem(dft, directory)
    write_scalar_value(grand_potential(dft), os.path.join(directory, "grand_potential.txt"))
    brush_height(dft, directory)
    output_arrays(dft, directory)
