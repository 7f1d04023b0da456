"""Host-side mirror of the reference's iDFT entry points, driving the device solve.

    iDFT(input_file)                  src/iDFT/iDFT.jl:23-39
    iLST(dataset)                     src/iLST/iLST.jl:35-52
    geometry_system(dataset)          src/geometry/geometry.jl:28-35
    setup_iDFT(dataset, bulk, geom)   src/iDFT/setup/setup_iDFT.jl:9-30
    eval_inhomogeneous(dft)           src/iDFT/evaluation/eval_inhomogeneous.jl:4-11
    solver_dft(dft)                   src/iDFT/evaluation/objective/solver_dft.jl:5-25
    objective_dft(dft)                src/iDFT/evaluation/objective/objective_dft.jl:6-30
    grand_potential(dft)              src/iDFT/evaluation/analysis/grand_potential.jl:4-28
    get_num_species(dft)              src/iDFT/evaluation/analysis/num_species.jl:1-38
    state_fractions(dft)              src/iDFT/evaluation/analysis/degree_of_dissociation.jl:1-78

Arrays use the reference's shapes and column-major order: mu_ex_K (NP, NB),
lng_K (NP, 2, MB), Psi (NP,), PsiC (1,), rho_segments[u] (NP, S_u, N_u).
Everything after setup runs in libsoftdft on the GPU; there is no CPU path.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import native
from .host import descriptor as desc_mod
from .host import geometry as geom_mod
from .host import ilst as ilst_mod
from .host import molsys as molsys_mod
from .host import yamlio


@dataclass
class IsingLST:
    """`src/iLST/structures/IsingLST.jl:15-19`."""

    molsys: molsys_mod.MolecularSystem
    bulk: ilst_mod.BulkState
    numerics: dict


@dataclass
class IsingDFT:
    """`src/iDFT/structures/IsingDFT.jl:67-74`: setup plus the device handle."""

    bulk_system: IsingLST
    geometry: geom_mod.CartesianGrid
    descriptor: desc_mod.Descriptor
    numerics: dict
    dataset: dict
    precision: int = desc_mod.PREC_FP64
    device: Optional[native.DeviceSystem] = None
    iterations: int = 0
    residual: float = float("nan")
    status: int = 0
    history: List[float] = field(default_factory=list)

    def handle(self) -> native.DeviceSystem:
        if self.device is None:
            self.device = native.DeviceSystem(self.descriptor, self.precision)
        return self.device

    # shapes of the reference arrays
    @property
    def NP(self) -> int:
        return self.descriptor.np_

    def split(self, x: np.ndarray):
        d = self.descriptor
        P, NB, MB = d.np_, d.nb, d.mb
        mu = x[: P * NB].reshape((P, NB), order="F")
        lng = x[P * NB: P * (NB + 2 * MB)].reshape((P, 2, MB), order="F")
        psi = x[P * (NB + 2 * MB): P * (NB + 2 * MB + 1)].copy()
        psic = x[-1:].copy()
        return mu, lng, psi, psic

    def join(self, mu_ex_K, lng_K, Psi, PsiC) -> np.ndarray:
        return np.concatenate([np.asarray(mu_ex_K).reshape(-1, order="F"), np.asarray(lng_K).reshape(-1, order="F"),
                               np.asarray(Psi).reshape(-1), np.asarray(PsiC).reshape(-1)])

    @property
    def state(self):
        """(mu_ex_K, lng_K, Psi, PsiC) on the device."""
        return self.split(self.handle().get_x())

    @state.setter
    def state(self, value):
        self.handle().set_x(self.join(*value))


def iLST(dataset: dict) -> IsingLST:
    ms = molsys_mod.molecular_system(dataset)
    num = dict(dataset.get("numerical") or {})
    bulk = ilst_mod.solve_bulk(ms, num)
    return IsingLST(ms, bulk, num)


def geometry_system(dataset: dict) -> geom_mod.CartesianGrid:
    return geom_mod.geometry_system(dataset)


def setup_iDFT(dataset: dict, bulk_system: IsingLST, geometry: geom_mod.CartesianGrid,
               precision: int = desc_mod.PREC_FP64) -> IsingDFT:
    d = desc_mod.build_descriptor(dataset, bulk_system.molsys, bulk_system.bulk, geometry)
    num = {str(k): yamlio.as_float(v) for k, v in (dataset.get("numerical") or {}).items()}
    return IsingDFT(bulk_system, geometry, d, num, dataset, precision)


def setup_request(dataset: dict, precision: int = desc_mod.PREC_FP64) -> IsingDFT:
    """iLST + geometry + setup_iDFT for one parsed input.yaml."""
    return setup_iDFT(dataset, iLST(dataset), geometry_system(dataset), precision)


def objective_dft(dft: IsingDFT):
    """One G(x) evaluation; returns new (mu_ex_K, lng_K, Psi, PsiC)."""
    return dft.split(dft.handle().objective())


def solver_dft(dft: IsingDFT) -> int:
    """Anderson-mixing solve of the current state in place; returns iterations.
    Reaching max_iters is not an error (AndersonMixing.jl:98-168)."""
    num = desc_mod.numerics_from_dict(dft.numerics)
    it, err, rc = dft.handle().solve(num)
    dft.iterations, dft.residual, dft.status = it, err, rc
    return it


def eval_inhomogeneous(dft: IsingDFT, directory: Optional[str] = ".") -> IsingDFT:
    """solver_dft, then the analysis files of call_analysis written into
    `directory` (eval_inhomogeneous.jl:4-11); directory=None only solves."""
    solver_dft(dft)
    if directory is not None:
        from .output import call_analysis
        call_analysis(dft, directory)
    return dft


def iDFT(input_file: str, precision: int = desc_mod.PREC_FP64, directory: Optional[str] = ".") -> IsingDFT:
    dataset = yamlio.load_file(input_file)
    dft = setup_request(dataset, precision)
    return eval_inhomogeneous(dft, directory)


def shape_densities(d, segs, beads, bonds):
    """Flat density arrays in the ABI's column-major order -> rho_segments (list
    of (NP, S_u, N_u)), rho_beads_K (NP, NB), rho_bonds_K (NP, 2, MB)."""
    segs = [s.reshape((d.np_, d.max_states[u], d.n_seg[u]), order="F") for u, s in enumerate(segs)]
    return segs, beads.reshape((d.np_, d.nb), order="F"), bonds.reshape((d.np_, 2, d.mb), order="F")


def densities(dft: IsingDFT):
    """rho_segments (list of (NP, S_u, N_u)), rho_beads_K (NP, NB), rho_bonds_K (NP, 2, MB)."""
    return shape_densities(dft.descriptor, *dft.handle().densities())


def grand_potential(dft: IsingDFT) -> float:
    return dft.handle().grand_potential()


def get_num_species(dft: IsingDFT) -> np.ndarray:
    return dft.handle().num_species()


def state_fractions(dft: IsingDFT):
    """Per species with multi-state segments: per-segment state fractions and
    their average over dissociating segments (write_total_state_fractions)."""
    return state_fractions_of(dft, densities(dft)[0])


def state_fractions_of(dft: IsingDFT, segs):
    """state_fractions for given segment densities (list of (NP, S_u, N_u)):
    the degree of dissociation of degree_of_dissociation.jl:1-78, a plain sum
    over the grid per (segment, state) normalised over the segment's states."""
    out = {}
    for u, cfg in enumerate(dft.bulk_system.molsys.configurations):
        fam = cfg.state_family
        if not any(len(f) > 1 for f in fam):
            continue
        S = max(len(f) for f in fam)
        rows = []
        sums = np.zeros(S)
        cnt = np.zeros(S)
        for g, f in enumerate(fam):
            if len(f) == 1:
                continue
            vals = segs[u][:, : len(f), g].sum(axis=0)
            tot = vals.sum()
            normed = vals / tot if tot > 0 else np.zeros(len(f))
            rows.append((g, normed))
            sums[: len(f)] += normed
            cnt[: len(f)] += 1
        avg = np.where(cnt > 0, sums / np.maximum(cnt, 1), np.nan)
        out[dft.bulk_system.molsys.species[u]] = {"segments": rows, "avg": avg}
    return out
