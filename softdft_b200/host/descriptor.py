"""ctypes mirror of include/softdft.h and the builder that fills it.

``build_descriptor`` is the host half of the reference's `setup_iDFT`
(`src/iDFT/setup/setup_iDFT.jl:9-30`): it resolves the fixed (grafted) segments
(`setup/setup_steps/process_fixed.jl:2-46`,
`coordinate_system/Cartesian/fixed_species/determine_fixed.jl:1-29`), the
functional set (`setup/setup_steps/process_functionals.jl:70-89`) and the initial
guess (`setup/setup_steps/process_guess.jl:5-54`: bulk mu_ex and ln g everywhere,
Psi = PsiC = 0).  Grid fields (Ext, trapez), k-space weights and the surface
charge spectrum are built from these numbers by the library itself.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List

import numpy as np

from .geometry import CartesianGrid, julia_round
from .ilst import BulkState
from .molsys import MolecularSystem
from .yamlio import numerics_int

ABI_VERSION = 2
FUNC_BITS = {"mfmt": 0x1, "TPT1mfmt": 0x2, "msa": 0x4, "TPT1msa": 0x8}
PREC_FP64 = 0
PREC_MIXED = 1


class SpeciesDesc(C.Structure):
    _fields_ = [
        ("n_seg", C.c_int32),
        ("max_states", C.c_int32),
        ("parent", C.POINTER(C.c_int32)),
        ("n_states", C.POINTER(C.c_int32)),
        ("states", C.POINTER(C.c_int32)),
        ("fixed_coord", C.POINTER(C.c_int32)),
        ("fixed_density", C.c_double),
        ("max_distance", C.POINTER(C.c_double)),
        ("mu_species", C.c_double),
    ]


class SystemDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("np", C.c_int32),
        ("bin_width", C.c_double),
        ("length", C.c_double),
        ("hard_walls", C.c_int32),
        ("charged_walls", C.c_int32),
        ("wall_charge", C.c_double * 2),
        ("bjerrum_length", C.c_double),
        ("nb", C.c_int32),
        ("diameter", C.POINTER(C.c_double)),
        ("valence", C.POINTER(C.c_double)),
        ("delta_muH", C.POINTER(C.c_double)),
        ("mb", C.c_int32),
        ("bond_types", C.POINTER(C.c_int32)),
        ("n_species", C.c_int32),
        ("species", C.POINTER(SpeciesDesc)),
        ("functionals", C.c_uint32),
        ("mu_ex_bulk", C.POINTER(C.c_double)),
        ("lng_bulk", C.POINTER(C.c_double)),
    ]


class Numerics(C.Structure):
    _fields_ = [
        ("max_iters", C.c_int32),
        ("anderm", C.c_int32),
        ("damping", C.c_double),
        ("mixing_max", C.c_double),
        ("switch_tole", C.c_double),
        ("tole", C.c_double),
        ("mixed_switch", C.c_double),
    ]


class SolverState(C.Structure):
    """sdft_solver_state: the Anderson driver's state between iterations."""
    _fields_ = [
        ("anderm", C.c_int32),
        ("iter", C.c_int32),
        ("use_picard", C.c_int32),
        ("reserved", C.c_int32),
        ("err", C.c_double),
        ("lambdas", C.c_double * 15),
    ]


def numerics_from_dict(num: dict) -> Numerics:
    """Defaults of `src/NonlinearSolvers/fixed_point/AndersonMixing.jl:74-79`."""
    return Numerics(
        max_iters=numerics_int(num, "max_iters", 100000, True),
        anderm=numerics_int(num, "anderm", 5, False),
        damping=float(num.get("damping", 0.5)),
        mixing_max=float(num.get("mixing_max", 1.0)),
        switch_tole=float(num.get("switch_tole", 1e-3)),
        tole=float(num.get("tole", 1e-6)),
        mixed_switch=float(num.get("mixed_switch", 0.0)),
    )


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(arr, ctype):
    return arr.ctypes.data_as(C.POINTER(ctype))


@dataclass
class Descriptor:
    """Owns the numpy buffers a SystemDesc points into."""

    desc: SystemDesc
    keep: List[object] = field(default_factory=list)
    np_: int = 0
    nb: int = 0
    mb: int = 0
    n_species: int = 0
    n_seg: List[int] = field(default_factory=list)
    max_states: List[int] = field(default_factory=list)
    fixed_coord: List[np.ndarray] = field(default_factory=list)
    mu_species: List[float] = field(default_factory=list)

    @property
    def n_unknowns(self) -> int:
        return self.np_ * (self.nb + 2 * self.mb + 1) + 1

    def initial_state(self):
        """process_guess: x0 = (bulk mu_ex, bulk ln g, 0, 0) on every grid point."""
        d = self.desc
        mu = np.repeat(np.ctypeslib.as_array(d.mu_ex_bulk, (self.nb,))[None, :], self.np_, axis=0)
        lng = np.repeat(np.ctypeslib.as_array(d.lng_bulk, (self.mb,))[None, None, :], 2, axis=1) if self.mb else np.zeros((1, 2, 0))
        lng = np.repeat(lng, self.np_, axis=0) if self.mb else np.zeros((self.np_, 2, 0))
        return (np.asfortranarray(mu), np.asfortranarray(lng), np.zeros(self.np_), np.zeros(1))


def fixed_segments(dataset: dict, ms: MolecularSystem, geom: CartesianGrid):
    """Per species: (density, [coordinate or -1 per segment])."""
    out = []
    sdata = dataset["species"]
    idx_LW = julia_round(0.0 / geom.bin_width) + 1
    idx_RW = julia_round(geom.dimensions / geom.bin_width) + 1
    for u, cfg in enumerate(ms.configurations):
        n = len(cfg.sequence)
        coords = np.full(n, -1, dtype=np.int32)
        dens = 0.0
        entry = sdata[u]
        if "fixed" in entry:
            fx = entry["fixed"]
            if ms.input_densities[u] > 0.0:
                raise ValueError(f"Species {u+1} defines a fixed segment but also has nonzero input density "
                                 f"({ms.input_densities[u]}). Simultaneous bulk and brush densities are not supported.")
            if "density" not in fx:
                raise ValueError(f"Species {u+1} contains 'fixed' but does not specify a density.")
            dens = float(fx["density"])
            if "segment" not in fx or "position" not in fx:
                raise ValueError(f"Species {u+1} contains 'fixed' but is missing 'segment' or 'position'.")
            segs, pos = list(fx["segment"]), list(fx["position"])
            if len(segs) != len(pos):
                raise ValueError(f"Mismatch in number of fixed segments and specified positions for species {u+1}.")
            for L, tag in zip(segs, pos):
                L = int(L)
                j = cfg.sequence[L - 1]
                dzr = julia_round(ms.diameters[j] / geom.bin_width / 2.0)
                if tag == "left":
                    c1 = idx_LW + dzr
                elif tag == "right":
                    c1 = idx_RW - dzr
                else:
                    raise ValueError(f"Invalid grafting position tag for species {u+1}, segment {L}: '{tag}'")
                coords[L - 1] = c1 - 1
            # the reference reads a fixed segment's grid point as
            # coordinates[1][seg]: only segment 1 can be fixed in 1D
            if np.any(coords[1:] >= 0):
                raise ValueError(f"Species {u+1}: only the first segment can be fixed in a 1D slit")
        out.append((dens, coords))
    return out


def build_descriptor(dataset: dict, ms: MolecularSystem, bulk: BulkState, geom: CartesianGrid) -> Descriptor:
    keep: List[object] = []
    nb = len(ms.monomers)
    mb = len(ms.bond_types)
    funcs = 0
    for m in ms.fe_model:
        if m in FUNC_BITS:
            funcs |= FUNC_BITS[m]
        elif m in ("ideal", "coul"):
            continue
        else:
            raise NotImplementedError(f"functional '{m}' is not supported by the device solve")
    fixed = fixed_segments(dataset, ms, geom)
    sp_arr = (SpeciesDesc * len(ms.configurations))()
    d = Descriptor(desc=SystemDesc(), keep=keep, np_=geom.NP, nb=nb, mb=mb, n_species=len(ms.configurations))
    for u, cfg in enumerate(ms.configurations):
        if cfg.model != "freely_jointed":
            raise NotImplementedError("monomerbead species are not supported by the device solve")
        n = len(cfg.sequence)
        S = max(len(f) for f in cfg.state_family)
        parent = _i32([(p[0] if p else -1) for p in cfg.topology.parents])
        for g, p in enumerate(cfg.topology.parents):
            if len(p) > 1:
                raise NotImplementedError("segments with more than one parent are not supported")
        nst = _i32([len(f) for f in cfg.state_family])
        st = np.full((n, S), -1, dtype=np.int32)
        for g, f in enumerate(cfg.state_family):
            st[g, :len(f)] = f
        st = _i32(st.reshape(-1))
        dens, coords = fixed[u]
        coords = _i32(coords)
        if np.any(coords >= 0):
            md = _f64(np.asarray(cfg.max_distance, dtype=np.float64).reshape(-1))
        else:
            md = None
        keep += [parent, nst, st, coords] + ([md] if md is not None else [])
        mu_u = float(bulk.mu_species[u])
        sp_arr[u] = SpeciesDesc(n, S, _ptr(parent, C.c_int32), _ptr(nst, C.c_int32), _ptr(st, C.c_int32),
                                _ptr(coords, C.c_int32), dens,
                                _ptr(md, C.c_double) if md is not None else C.POINTER(C.c_double)(),
                                mu_u)
        d.n_seg.append(n)
        d.max_states.append(S)
        d.fixed_coord.append(coords)
        d.mu_species.append(mu_u)
    keep.append(sp_arr)
    diam, val, dmu = _f64(ms.diameters), _f64(ms.valences), _f64(ms.delta_muH)
    bonds = _i32(np.asarray(ms.bond_types, dtype=np.int32).reshape(-1)) if mb else _i32(np.zeros(2))
    mu_ex, lng = _f64(bulk.mu_ex), _f64(bulk.lng if mb else np.zeros(1))
    keep += [diam, val, dmu, bonds, mu_ex, lng]
    wc = (C.c_double * 2)(*geom.wall_charges)
    d.desc = SystemDesc(
        abi_version=ABI_VERSION, np=geom.NP, bin_width=geom.bin_width, length=geom.dimensions,
        hard_walls=1 if geom.hard_walls is not None else 0,
        charged_walls=1 if geom.charged_walls is not None else 0,
        wall_charge=wc, bjerrum_length=ms.bjerrum_length, nb=nb,
        diameter=_ptr(diam, C.c_double), valence=_ptr(val, C.c_double), delta_muH=_ptr(dmu, C.c_double),
        mb=mb, bond_types=_ptr(bonds, C.c_int32), n_species=len(ms.configurations), species=sp_arr,
        functionals=funcs, mu_ex_bulk=_ptr(mu_ex, C.c_double), lng_bulk=_ptr(lng, C.c_double),
    )
    return d
