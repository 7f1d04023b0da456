"""Synthetic input.yaml requests for the benchmark workloads.

No public dataset exists for this solve; each workload is a seeded synthetic
request (or request stream) with the shapes of the benchmark configurations:

* ``plain_slit``      -- weak-polyacid chain (N=20, pKa 4.5, pH 7), 1:1 salt 0.1 M,
                         hard-sphere solvent, total packing fraction 0.3, hard walls,
                         NP = 1024 at dz = 0.02 (H = 1023*dz so that NP = cld(H,dz)+1
                         = 1024 exactly), Anderson m=5, damping 0.1, tole 1e-8.
* ``diblock_slit``    -- diblock weak polyelectrolyte (100 acid pKa 4.0 + 100 base
                         pKa 9.5), 2:1 salt 10 mM, solvent, packing 0.35, walls
                         charged -0.1 e/sigma^2, NP = 16384 at dz = 0.01, m=10.
* ``batch_uneven``    -- seeded draws: NP log-uniform, N uniform, pH, salt, packing.
* ``serving_stream``  -- seeded Poisson arrivals of single-slit requests.
* ``brush_branch``    -- grafted weak-polyacid brushes on both walls for the
                         wall-separation continuation.

Chain monomer volume fraction is 0.05 wherever a workload does not fix it; the
solvent density fills the packing fraction.

Mixing controls: a charged chain responds to the slit-scale potential as a whole
(charge ~ -N), so the Picard map's gain on the lowest potential mode is ~1e3 and
the reference's linear mixing needs a coefficient below ~1e-3 (its own example
inputs use mixing_max 0.001).  The workloads keep damping 0.1 and anderm 5 and
set mixing_max 0.002 with switch_tole 10, i.e. Anderson from iteration m on.  Every generator returns plain
dicts in the reference's input.yaml schema (`input.yaml:1-74`).
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

PI = math.pi
NA = 6.0221415e23
L_SC = 0.5e-9


def molar_to_density(c: float) -> float:
    return c * NA * L_SC ** 3 * 1000.0


def slit_length(np_: int, dz: float) -> float:
    """Largest-representable H close to (np_-1)*dz for which the reference's
    grid rule NP = cld(H, dz) + 1 gives exactly ``np_`` points."""
    from .host.geometry import cld
    H = (np_ - 1) * dz
    while cld(H, dz) + 1 > np_:
        H = math.nextafter(H, 0.0)
    while cld(H, dz) + 1 < np_:
        H = math.nextafter(H, math.inf)
    return H


def _monomers(extra: dict | None = None) -> dict:
    mons = {
        "A": {"diameter": 1.0, "valence": 0.0},
        "B": {"diameter": 1.0, "valence": -1.0},
        "S": {"diameter": 1.0, "valence": 0.0},
        "Y": {"diameter": 1.0, "valence": 1.0},
        "Z": {"diameter": 1.0, "valence": -1.0},
        "c": {"diameter": 1.0, "valence": 1.0},
        "a": {"diameter": 1.0, "valence": -1.0},
    }
    if extra:
        mons.update(extra)
    return mons


def weak_acid_slit(np_: int, dz: float, n_chain: int, pKa: float, pH: float, salt_M: float,
                   eta: float, phi_chain: float = 0.05, anderm: int = 5, damping: float = 0.1,
                   tole: float = 1e-8, wall_charge: float | None = None, cation_valence: float = 1.0,
                   max_iters: int = 100000, mixing_max: float = 0.002, switch_tole: float = 10.0) -> dict:
    """One slit request with a weak-polyacid homopolymer of ``n_chain`` segments."""
    H = slit_length(np_, dz)
    rho_chain = phi_chain / (PI / 6.0)
    rho_salt = molar_to_density(salt_M)
    rho_anion = rho_salt * cation_valence
    eta_ions = PI / 6.0 * (rho_salt + rho_anion)
    rho_solvent = max((eta - phi_chain - eta_ions) / (PI / 6.0), 0.0)
    ext = {"hard_walls": {"dims": [1]}}
    if wall_charge is not None:
        ext["charged_walls"] = {"dims": [1], "charge": [wall_charge, wall_charge]}
    return {
        "procedure": "iDFT",
        "geometry": {"coordinate_system": "Cartesian", "dimensions": [H], "bin_width": [dz], "external_field": ext},
        "species": [
            {"sequence": "A" * n_chain, "density": rho_chain},
            {"sequence": "S", "density": rho_solvent},
            {"sequence": "c", "density": rho_salt, "adjustable": True},
            {"sequence": "a", "density": rho_anion, "adjustable": True},
            {"sequence": "Y", "pSpecies": pH},
            {"sequence": "Z"},
        ],
        "reactions": [
            {"species": ["A", "Y", "B"], "coeffs": [-1, 1, 1], "pK": pKa},
            {"species": ["Y", "Z"], "coeffs": [1, 1], "pK": 14.0},
        ],
        "monomers": _monomers({"c": {"diameter": 1.0, "valence": cation_valence}}),
        "numerical": {"anderm": anderm, "damping": damping, "tole": tole, "max_iters": max_iters,
                      "mixing_max": mixing_max, "switch_tole": switch_tole},
        "model": ["ideal", "TPT1mfmt", "TPT1msa"],
    }


def plain_slit() -> dict:
    return weak_acid_slit(1024, 0.02, 20, 4.5, 7.0, 0.1, 0.3)


def diblock_slit(np_: int = 16384) -> dict:
    """Diblock weak polyelectrolyte: 100 acid (A -> B + Y, pK 4.0) and 100 base
    (C + Y -> D, pK 9.5) segments, 2:1 salt at 10 mM, charged walls."""
    dz = 0.01
    H = slit_length(np_, dz)
    rho_chain = 0.05 / (PI / 6.0)
    rho_salt = molar_to_density(0.010)
    rho_anion = 2.0 * rho_salt
    eta = 0.35
    rho_solvent = (eta - 0.05 - PI / 6.0 * (rho_salt + rho_anion)) / (PI / 6.0)
    return {
        "procedure": "iDFT",
        "geometry": {"coordinate_system": "Cartesian", "dimensions": [H], "bin_width": [dz],
                     "external_field": {"hard_walls": {"dims": [1]},
                                        "charged_walls": {"dims": [1], "charge": [-0.1, -0.1]}}},
        "species": [
            {"sequence": "A" * 100 + "C" * 100, "density": rho_chain},
            {"sequence": "S", "density": rho_solvent},
            {"sequence": "c", "density": rho_salt, "adjustable": True},
            {"sequence": "a", "density": rho_anion, "adjustable": True},
            {"sequence": "Y", "pSpecies": 7.0},
            {"sequence": "Z"},
        ],
        "reactions": [
            {"species": ["A", "Y", "B"], "coeffs": [-1, 1, 1], "pK": 4.0},
            {"species": ["C", "Y", "D"], "coeffs": [-1, -1, 1], "pK": -9.5},
            {"species": ["Y", "Z"], "coeffs": [1, 1], "pK": 14.0},
        ],
        "monomers": _monomers({"C": {"diameter": 1.0, "valence": 0.0}, "D": {"diameter": 1.0, "valence": 1.0},
                               "c": {"diameter": 1.0, "valence": 2.0}}),
        "numerical": {"anderm": 10, "damping": 0.1, "tole": 1e-8},
        "model": ["ideal", "TPT1mfmt", "TPT1msa"],
    }


def _smooth7(n: int) -> bool:
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def batch_uneven(n: int = 512, seed: int = 3, np_lo: int = 2048, np_hi: int = 16384,
                 n_lo: int = 10, n_hi: int = 300, pow2: bool = False) -> List[dict]:
    """Seeded uneven batch.  NP is drawn log-uniform and moved up to the next
    7-smooth size (prime factors 2, 3, 5, 7 only), or rounded to a power of two
    with ``pow2``."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        draw = math.exp(rng.uniform(math.log(np_lo), math.log(np_hi)))
        if pow2:
            np_ = int(2 ** round(math.log2(draw)))
        else:
            np_ = int(round(draw))
            while not _smooth7(np_):
                np_ += 1
        nch = int(rng.integers(n_lo, n_hi + 1))
        pH = float(rng.uniform(2.0, 12.0))
        salt = float(math.exp(rng.uniform(math.log(1e-3), math.log(1.0))))
        eta = float(rng.uniform(0.1, 0.4))
        out.append(weak_acid_slit(np_, 0.02, nch, 4.5, pH, salt, eta))
    return out


def grafted_brush(np_: int, dz: float, n_chain: int, sigma_g: float, pKa: float, pH: float, salt_M: float,
                  eta: float = 0.3, anderm: int = 5, damping: float = 0.1, tole: float = 1e-8,
                  mixing_max: float = 0.05, switch_tole: float = 10.0) -> dict:
    """Weak-polyacid brushes grafted by segment 1 on both walls."""
    H = slit_length(np_, dz)
    rho_salt = molar_to_density(salt_M)
    rho_solvent = (eta - PI / 6.0 * 2 * rho_salt) / (PI / 6.0)
    return {
        "procedure": "iDFT",
        "geometry": {"coordinate_system": "Cartesian", "dimensions": [H], "bin_width": [dz],
                     "external_field": {"hard_walls": {"dims": [1]}}},
        "species": [
            {"sequence": "A" * n_chain, "density": 0.0,
             "fixed": {"density": sigma_g, "segment": [1], "position": ["left"]}},
            {"sequence": "A" * n_chain, "density": 0.0,
             "fixed": {"density": sigma_g, "segment": [1], "position": ["right"]}},
            {"sequence": "S", "density": rho_solvent},
            {"sequence": "c", "density": rho_salt, "adjustable": True},
            {"sequence": "a", "density": rho_salt, "adjustable": True},
            {"sequence": "Y", "pSpecies": pH},
            {"sequence": "Z"},
        ],
        "reactions": [
            {"species": ["A", "Y", "B"], "coeffs": [-1, 1, 1], "pK": pKa},
            {"species": ["Y", "Z"], "coeffs": [1, 1], "pK": 14.0},
        ],
        "monomers": _monomers(),
        "numerical": {"anderm": anderm, "damping": damping, "tole": tole, "mixing_max": mixing_max,
                      "switch_tole": switch_tole},
        "model": ["ideal", "TPT1mfmt", "TPT1msa"],
    }
