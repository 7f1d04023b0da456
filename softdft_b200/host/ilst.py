"""Bulk Ising liquid-state theory (iLST): the homogeneous state that seeds every
inhomogeneous solve.

Host-side restatement of `src/iLST/` (`iLST.jl:35-52`): initial densities
(`setup/setup_steps/initialize_densities.jl:31-121`), the residual
(`evaluation/objective/residual_bulkstate.jl:26-35`), the AndersonResidual driver
(`src/NonlinearSolvers/residual/AndersonResidual.jl:27-138`) and the bulk
pressure (`evaluation/analysis/eval_pressure.jl:10-25`).  This is O(species^2)
scalar work per request and stays on the host.

Documented departures: an ``anderm`` key in the numerical section is converted to
an integer here; the reference passes the Float64 straight to ``zeros`` and fails.
``coul`` in the model list is accepted as the (zero) bulk Coulomb term of
`src/iLST/free_energy/coulomb/coulomb.jl`, which the reference's registry never
includes.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

from .lsqr import lsqr_inplace
from .molsys import LOG10, MolecularSystem, concentration_to_density
from .yamlio import numerics_int

PI = math.pi
SUPPORTED_MODELS = ("ideal", "mfmt", "TPT1mfmt", "msa", "TPT1msa", "coul")


# --------------------------------------------------------------------------
# pointwise bulk formulas (iLST free_energy/*)
# --------------------------------------------------------------------------
def free_energy_mfmt(n0, n1, n2, n3):
    """Bulk White-Bear FMT (`free_energy/excluded_volume/mfmt.jl:143-156`)."""
    om = 1.0 - n3
    lt = math.log(om)
    inv_denom = 1.0 / (36.0 * PI * n3 * n3 * om * om)
    return -n0 * lt + (n1 * n2) / om + n2 ** 3 * (n3 + om * om * lt) * inv_denom


def mfmt_deriv_bulk(n0, n1, n2, n3):
    """`free_energy/excluded_volume/mfmt.jl:275-299` (rows 1-4, vectors zero)."""
    om = 1.0 - n3
    l1 = math.log(om)
    i1 = 1.0 / om
    i3 = 1.0 / n3
    i36 = 1.0 / (36.0 * PI)
    d1 = -l1
    d2 = n2 * i1
    d3 = n1 * i1 + (n2 ** 2) * 3.0 * i36 * i3 * (l1 * i3 + i1 ** 2)
    d4 = (n0 * i1 + (n1 * n2) * i1 ** 2
          - (l1 * i3 ** 3 * 2.0 * i36 + i3 ** 2 * i1 * i36 + (1.0 - 3.0 * n3) * i3 ** 2 * i36 * i1 ** 3) * (n2 ** 3))
    return d1, d2, d3, d4


def gamma_msa(rho, sig, Z, lB):
    """MSA screening parameter by the damped fixed point of
    `free_energy/electrostaticcorrelations/msa.jl:181-230`."""
    tol = 1e-10
    s = float(np.sum(rho * Z * Z))
    kappa = math.sqrt(4.0 * PI * lB * s)
    if kappa < tol:
        return kappa / 2.0, 0.0, 2.0 / PI
    sig_eff = float(np.sum(rho * sig)) / float(np.sum(rho))
    x = sig_eff * math.sqrt(4.0 * PI * lB * s)
    G = (math.sqrt(1.0 + 2.0 * x) - 1.0) / (2.0 * sig_eff)
    term2 = 2.0 / PI * (1.0 - PI / 6.0 * float(np.sum(rho * sig ** 3)))
    it = 0
    while True:
        H = float(np.sum(rho * sig ** 3 / (1.0 + G * sig))) + term2
        eta = float(np.sum(rho * Z * sig / (1.0 + G * sig))) / H
        G1 = math.sqrt(PI * lB * float(np.sum(rho * (Z - eta * sig * sig) ** 2 / (1.0 + G * sig) ** 2)))
        Gn = 0.9 * G + 0.1 * G1
        it += 1
        if abs(G1 - G) < tol or it >= 1000:
            G = Gn
            break
        G = Gn
    if it == 1000 and math.isnan(abs(G1 - G)):
        raise FloatingPointError("Gamma is NaN")
    return G, eta, H


def msa_deriv(rho, sig, Z, lB):
    """`free_energy/electrostaticcorrelations/msa.jl:147-155`."""
    G, eta, _ = gamma_msa(rho, sig, Z, lB)
    u_star = -PI / 6 * float(np.sum(rho * sig * sig * ((Z - eta * sig * sig) / (1.0 + G * sig) + Z)))
    return -lB * (G * Z ** 2 / (1.0 + G * sig)
                  + eta * sig * ((2.0 * Z - eta * sig ** 2) / (1.0 + G * sig) + eta * sig ** 2 / 3.0)
                  + Z * u_star)


def free_energy_msa(rho, sig, Z, lB):
    """`free_energy/electrostaticcorrelations/msa.jl:115-118`."""
    G, eta, _ = gamma_msa(rho, sig, Z, lB)
    return G ** 3 / (3.0 * PI) - lB * float(np.sum(rho * Z * (Z * G + eta * sig) / (1.0 + G * sig)))


def tpt1msa_deriv(bonds2, bond_types, rho, sig, Z, lB):
    """`free_energy/electrostaticcorrelations/TPT1msa.jl:200-282`: MSA derivative
    plus the TPT1 chain term; ``bonds2`` is (2, MB)."""
    mb = len(bond_types)
    lng = np.zeros(mb)
    dphi = msa_deriv(rho, sig, Z, lB)
    G, eta, H = gamma_msa(rho, sig, Z, lB)
    if G == 0.0:
        for u, (i, j) in enumerate(bond_types):
            lng[u] = -lB / ((sig[i] + sig[j]) / 2.0) * Z[i] * Z[j]
        return dphi, lng
    for u, (i, j) in enumerate(bond_types):
        sij = (sig[i] + sig[j]) / 2.0
        Xi = (Z[i] - eta * sig[i] ** 2) / (1.0 + G * sig[i])
        Xj = (Z[j] - eta * sig[j] ** 2) / (1.0 + G * sig[j])
        lng[u] = -lB / sij * Xi * Xj
    opg = 1.0 + G * sig
    dfG = -2.0 * PI * lB * float(np.sum(rho * sig * (Z - eta * sig * sig) ** 2 / opg ** 3))
    dfe = -2.0 * PI * lB * float(np.sum(rho * sig * sig * (Z - eta * sig * sig) / opg ** 2))
    deG = -1.0 / H * float(np.sum(rho * Z * sig * sig / opg ** 2))
    deH = -eta / H
    dHG = -float(np.sum(rho * sig ** 4 / opg ** 2))
    detaG = deG + deH * dHG
    denom = 1.0 / (2.0 * G - dfe * detaG - dfG)
    dphi = dphi.copy()
    for w in range(len(rho)):
        inv = 1.0 / (1.0 + G * sig[w])
        Xw = (Z[w] - eta * sig[w] ** 2) * inv
        dfr = PI * lB * Xw ** 2
        der = sig[w] / H * Z[w] * inv
        dHr = sig[w] ** 3 * (inv - 1.0 / 3.0)
        dGr = (dfr + dfe * (der + dfe * deH * dHr)) * denom
        detar = detaG * dGr
        for u, (i, j) in enumerate(bond_types):
            sij = (sig[i] + sig[j]) / 2.0
            ii = 1.0 / (1.0 + G * sig[i])
            Xi = (Z[i] - eta * sig[i] ** 2) * ii
            dXi = -(sig[i] ** 2 * ii * detar + sig[i] * Xi * ii * dGr)
            ij = 1.0 / (1.0 + G * sig[j])
            Xj = (Z[j] - eta * sig[j] ** 2) * ij
            dXj = -(sig[j] ** 2 * ij * detar + sig[j] * Xj * ij * dGr)
            dphi[w] += (bonds2[0, u] + bonds2[1, u]) / 2.0 * lB / sij * (dXi * Xj + Xi * dXj)
    return dphi, lng


def tpt1mfmt_deriv_bulk(bonds2, bond_types, rho, sig):
    """`free_energy/excluded_volume/TPT1mfmt.jl:399-444`; returns the per-bead
    chemical potential increment and the per-bond ln y_HS."""
    n0 = float(np.sum(rho))
    n1 = float(np.sum(rho * sig / 2))
    n2 = float(np.sum(rho * PI * sig ** 2))
    n3 = float(np.sum(rho * PI * sig ** 3 / 6))
    d1, d2, d3, d4 = mfmt_deriv_bulk(n0, n1, n2, n3)
    i1 = 1.0 / (1.0 - n3)
    term2 = n2 / 4.0 * i1 ** 2
    term3 = n2 ** 2 / 72.0 * i1 ** 3
    lng = np.zeros(len(bond_types))
    for u, (i, j) in enumerate(bond_types):
        sij = (sig[i] + sig[j]) / 2
        tau = sig[i] * sig[j] / sij
        y = i1 + term2 * tau + term3 * tau ** 2
        dl2 = (tau / 4.0 * i1 ** 2 + n2 * tau ** 2 * i1 ** 3 / 36.0) / y
        dl3 = (i1 ** 2 + n2 / 2.0 * i1 ** 3 * tau + n2 ** 2 / 24.0 * i1 ** 4 * tau ** 2) / y
        d3 -= 0.5 * (bonds2[0, u] + bonds2[1, u]) * dl2
        d4 -= 0.5 * (bonds2[0, u] + bonds2[1, u]) * dl3
        lng[u] = math.log(y)
    mu = d1 + d2 * sig / 2 + d3 * PI * sig ** 2 + d4 * PI * sig ** 3 / 6
    return mu, lng


def free_energy_tpt1mfmt_bulk(bonds2, bond_types, rho, sig):
    """`free_energy/excluded_volume/TPT1mfmt.jl:238-262`."""
    n0 = float(np.sum(rho))
    n1 = float(np.sum(rho * sig / 2))
    n2 = float(np.sum(rho * PI * sig ** 2))
    n3 = float(np.sum(rho * PI * sig ** 3 / 6))
    f = free_energy_mfmt(n0, n1, n2, n3)
    i1 = 1.0 / (1.0 - n3)
    term2 = n2 / 4.0 * i1 ** 2
    term3 = n2 ** 2 / 72.0 * i1 ** 3
    for u, (i, j) in enumerate(bond_types):
        sij = (sig[i] + sig[j]) / 2
        tau = sig[i] * sig[j] / sij
        y = i1 + term2 * tau + term3 * tau ** 2
        f -= 0.5 * (bonds2[0, u] + bonds2[1, u]) * math.log(y)
    return f


def free_energy_tpt1msa_bulk(bonds2, bond_types, rho, sig, Z, lB):
    """`free_energy/electrostaticcorrelations/TPT1msa.jl:138-155`."""
    f = free_energy_msa(rho, sig, Z, lB)
    G, eta, _ = gamma_msa(rho, sig, Z, lB)
    for u, (i, j) in enumerate(bond_types):
        sij = (sig[i] + sig[j]) / 2.0
        Xi = (Z[i] - eta * sig[i] ** 2) / (1.0 + G * sig[i])
        Xj = (Z[j] - eta * sig[j] ** 2) / (1.0 + G * sig[j])
        f -= 0.5 * (bonds2[0, u] + bonds2[1, u]) * (-lB / sij * Xi * Xj)
    return f


# --------------------------------------------------------------------------
# bulk state
# --------------------------------------------------------------------------
@dataclass
class BulkState:
    """`structures/BulkState.jl:27-58` (pair densities are not kept: nothing on the
    solve path reads them)."""

    rho_species: np.ndarray
    rho_segments: List[np.ndarray]     # [u] -> (max_states, n_seg)
    rho_beads: np.ndarray
    rho_bonds: np.ndarray              # (2, MB)
    mu_species: np.ndarray
    mu_ex: np.ndarray
    lng: np.ndarray
    Xi: np.ndarray
    pressure: float = 0.0
    iterations: int = 0
    residual: float = 0.0
    numerics: dict = field(default_factory=dict)


def _bond_index(bond_types, a, b):
    return bond_types.index((min(a, b), max(a, b)))


def initialize_densities(ms: MolecularSystem) -> BulkState:
    """`setup/setup_steps/initialize_densities.jl:31-121` (ideal state weights).
    Also overwrites ``ms.species_charge`` with the ideal state-averaged charge per
    chain, as the reference does."""
    ns = len(ms.species)
    nb = len(ms.monomers)
    mb = len(ms.bond_types)
    rho_species = np.zeros(ns)
    rho_segments = []
    rho_beads = np.zeros(nb)
    rho_bonds = np.zeros((2, mb))
    dm = ms.delta_muH
    z = ms.valences
    for u in range(ns):
        ms.species_charge[u] = 0.0
    for u, cfg in enumerate(ms.configurations):
        nseg = len(cfg.sequence)
        mx = max(len(f) for f in cfg.state_family)
        seg = np.zeros((mx, nseg))
        if not math.isnan(ms.input_pSpecies[u]):
            dens = concentration_to_density(10.0 ** (-ms.input_pSpecies[u]), ms.constants)
        else:
            dens = ms.input_densities[u]
        pd = dens / nseg
        rho_species[u] = pd
        for si in range(nseg):
            sti = cfg.state_family[si]
            Qi = sum(math.exp(-dm[s]) for s in sti)
            for ii, s_i in enumerate(sti):
                wi = math.exp(-dm[s_i]) / Qi
                seg[ii, si] += pd * wi
                rho_beads[s_i] += pd * wi
                ms.species_charge[u] += wi * z[s_i]
                if cfg.topology.parents[si]:
                    for sj in range(nseg):
                        if cfg.topology.parents[si][0] != sj:
                            continue
                        stj = cfg.state_family[sj]
                        Qj = sum(math.exp(-dm[s]) for s in stj)
                        for s_j in stj:
                            wj = math.exp(-dm[s_j]) / Qj
                            rho_bonds[:, _bond_index(ms.bond_types, s_i, s_j)] += pd * wi * wj
        rho_segments.append(seg)
    return BulkState(rho_species, rho_segments, rho_beads, rho_bonds,
                     np.zeros(ns), np.zeros(nb), np.zeros(mb), np.zeros(ns))


def _fj_propagators(ms: MolecularSystem, bulk: BulkState, u: int):
    """Bulk freely-jointed child/parent propagators and the partition function
    (`src/iLST/species_model/freely_jointed/child_propagators.jl:22-62`,
    `parent_propagators.jl:27-73`, `partition_function.jl:21-53`)."""
    cfg = ms.configurations[u]
    fam = cfg.state_family
    topo = cfg.topology
    n = len(cfg.sequence)
    ms_ = max(max(len(f) for f in fam), 1)
    mc = max(max(len(c) for c in topo.children), 1)
    dm, mu, lng = ms.delta_muH, bulk.mu_ex, bulk.lng
    gC = np.zeros((ms_, mc, ms_, n))
    for level in reversed(topo.levels):
        for p in level:
            for ii, s_i in enumerate(fam[p]):
                gC[0, 0, ii, p] = 1.0
                for ic, c in enumerate(topo.children[p]):
                    for ij, s_j in enumerate(fam[c]):
                        b = _bond_index(ms.bond_types, s_i, s_j)
                        val = math.exp(-dm[s_j] - mu[s_j] + lng[b])
                        for igc, _ in enumerate(topo.children[c]):
                            val *= float(np.sum(gC[:, igc, ij, c]))
                        gC[ij, ic, ii, p] = val
    gP = np.zeros((ms_, ms_, n))
    for level in topo.levels:
        for c in level:
            for ij, s_j in enumerate(fam[c]):
                gP[0, ij, c] = 1.0
                for p in topo.parents[c]:
                    for ii, s_i in enumerate(fam[p]):
                        b = _bond_index(ms.bond_types, s_i, s_j)
                        val = math.exp(-dm[s_i] - mu[s_i] + lng[b])
                        val *= float(np.sum(gP[:, ii, p]))
                        for ioc, oc in enumerate(topo.children[p]):
                            if oc != c:
                                val *= float(np.sum(gC[:, ioc, ii, p]))
                        gP[ii, ij, c] = val
    Xi = 0.0
    for ii, s_i in enumerate(fam[0]):
        t = math.exp(-(mu[s_i] + dm[s_i])) * float(np.sum(gP[:, ii, 0]))
        for ic, _ in enumerate(topo.children[0]):
            t *= float(np.sum(gC[:, ic, ii, 0]))
        Xi += t
    return gC, gP, Xi


def _lse(vals):
    """log(sum(exp(v))) over finite-or--inf entries."""
    v = np.asarray(vals, dtype=np.float64)
    m = np.max(v) if v.size else -np.inf
    if not np.isfinite(m):
        return m
    return float(m + np.log(np.sum(np.exp(v - m))))


def _fj_log_propagators(ms: MolecularSystem, bulk: BulkState, u: int):
    """The propagators of `_fj_propagators` as natural logarithms, for chains
    whose products leave the double range (the reference's unscaled products
    underflow past ~100 segments at mu_ex ~ 6 and then yield NaN).  Zero
    entries are -inf."""
    cfg = ms.configurations[u]
    fam = cfg.state_family
    topo = cfg.topology
    n = len(cfg.sequence)
    ms_ = max(max(len(f) for f in fam), 1)
    mc = max(max(len(c) for c in topo.children), 1)
    dm, mu, lng = ms.delta_muH, bulk.mu_ex, bulk.lng
    lC = np.full((ms_, mc, ms_, n), -np.inf)
    for level in reversed(topo.levels):
        for p in level:
            for ii, s_i in enumerate(fam[p]):
                lC[0, 0, ii, p] = 0.0
                for ic, c in enumerate(topo.children[p]):
                    for ij, s_j in enumerate(fam[c]):
                        b = _bond_index(ms.bond_types, s_i, s_j)
                        val = -dm[s_j] - mu[s_j] + lng[b]
                        for igc, _ in enumerate(topo.children[c]):
                            val += _lse(lC[:, igc, ij, c])
                        lC[ij, ic, ii, p] = val
    lP = np.full((ms_, ms_, n), -np.inf)
    for level in topo.levels:
        for c in level:
            for ij, s_j in enumerate(fam[c]):
                lP[0, ij, c] = 0.0
                for p in topo.parents[c]:
                    for ii, s_i in enumerate(fam[p]):
                        b = _bond_index(ms.bond_types, s_i, s_j)
                        val = -dm[s_i] - mu[s_i] + lng[b] + _lse(lP[:, ii, p])
                        for ioc, oc in enumerate(topo.children[p]):
                            if oc != c:
                                val += _lse(lC[:, ioc, ii, p])
                        lP[ii, ij, c] = val
    terms = []
    for ii, s_i in enumerate(fam[0]):
        t = -(mu[s_i] + dm[s_i]) + _lse(lP[:, ii, 0])
        for ic, _ in enumerate(topo.children[0]):
            t += _lse(lC[:, ic, ii, 0])
        terms.append(t)
    return lC, lP, _lse(terms)


def _fj_accumulate_log(ms: MolecularSystem, bulk: BulkState, u: int, seg: np.ndarray) -> None:
    """`accumulate_densities!` of the bulk freely-jointed chain evaluated with
    log-domain propagators."""
    cfg = ms.configurations[u]
    fam = cfg.state_family
    topo = cfg.topology
    lC, lP, lXi = _fj_log_propagators(ms, bulk, u)
    bulk.Xi[u] = math.exp(lXi) if lXi < 700 else math.inf
    for si in range(len(cfg.sequence)):
        for ii, s_i in enumerate(fam[si]):
            lam = bulk.mu_ex[s_i] + ms.delta_muH[s_i]
            lpref = math.log(bulk.rho_species[u]) - lam + _lse(lP[:, ii, si]) - lXi
            if topo.children[si]:
                child = topo.children[si][0]
                terms = []
                for ij, _ in enumerate(fam[child]):
                    t = lC[ij, 0, ii, si]
                    for ioc, oc in enumerate(topo.children[si]):
                        if oc != child:
                            t += _lse(lC[:, ioc, ii, si])
                    terms.append(t)
                lcc = _lse(terms)
            else:
                lcc = 0.0
            lval = lpref + lcc
            val = math.exp(lval)
            seg[ii, si] = val
            bulk.rho_beads[s_i] += val
            for ic, c in enumerate(topo.children[si]):
                lQ = _lse(lC[:, ic, ii, si])
                for ij, s_j in enumerate(fam[c]):
                    f = math.exp(lval + lC[ij, ic, ii, si] - lQ)
                    bulk.rho_bonds[:, _bond_index(ms.bond_types, s_i, s_j)] += f


def _fj_log_xi(ms, bulk, u) -> float:
    """ln Xi of a freely-jointed species: direct products when finite, else
    log-domain propagators."""
    with np.errstate(all="ignore"):
        _, _, Xi = _fj_propagators(ms, bulk, u)
    if np.isfinite(Xi) and Xi > 0:
        return math.log(Xi)
    return _fj_log_propagators(ms, bulk, u)[2]


def _monomerbead_xi(ms, bulk, u):
    """`src/iLST/species_model/monomerbead/partition_function.jl:17-38`."""
    cfg = ms.configurations[u]
    return sum(math.exp(-bulk.mu_ex[s] - ms.delta_muH[s]) for s in cfg.state_family[0])


def eval_bulk_density(ms: MolecularSystem, bulk: BulkState) -> None:
    """`evaluation/objective/functions/eval_bulk_density.jl:9-22` with the
    per-model accumulation of `species_model/*/accumulate_densities.jl`.
    Uses the current ``mu_ex``/``lng`` (those of the previous residual call)."""
    bulk.rho_beads[:] = 0.0
    bulk.rho_bonds[:] = 0.0
    dm = ms.delta_muH
    for u, cfg in enumerate(ms.configurations):
        seg = bulk.rho_segments[u]
        seg[:] = 0.0
        fam = cfg.state_family
        topo = cfg.topology
        if cfg.model == "monomerbead":
            Xi = _monomerbead_xi(ms, bulk, u)
            bulk.Xi[u] = Xi
            for si in range(len(cfg.sequence)):
                for ii, s_i in enumerate(fam[si]):
                    val = bulk.rho_species[u] / Xi * math.exp(-bulk.mu_ex[s_i] - dm[s_i])
                    bulk.rho_beads[s_i] += val
                    seg[ii, si] += val
            continue
        with np.errstate(all="ignore"):
            gC, gP, Xi = _fj_propagators(ms, bulk, u)
        if not (np.isfinite(Xi) and Xi > 0 and np.all(np.isfinite(gC)) and np.all(np.isfinite(gP))
                and bulk.rho_species[u] > 0):
            if bulk.rho_species[u] > 0:
                _fj_accumulate_log(ms, bulk, u, seg)
            else:
                bulk.Xi[u] = Xi
            continue
        bulk.Xi[u] = Xi
        for si in range(len(cfg.sequence)):
            for ii, s_i in enumerate(fam[si]):
                lam = bulk.mu_ex[s_i] + dm[s_i]
                pref = bulk.rho_species[u] * math.exp(-lam) * float(np.sum(gP[:, ii, si])) / Xi
                if topo.children[si]:
                    child = topo.children[si][0]
                    cc = 0.0
                    for ij, _ in enumerate(fam[child]):
                        t = gC[ij, 0, ii, si]
                        for ioc, oc in enumerate(topo.children[si]):
                            if oc != child:
                                t *= float(np.sum(gC[:, ioc, ii, si]))
                        cc += t
                else:
                    cc = 1.0
                val = pref * cc
                seg[ii, si] = val
                bulk.rho_beads[s_i] += val
                for ic, c in enumerate(topo.children[si]):
                    Qc = float(np.sum(gC[:, ic, ii, si]))
                    for ij, s_j in enumerate(fam[c]):
                        f = val * gC[ij, ic, ii, si] / Qc
                        b = _bond_index(ms.bond_types, s_i, s_j)
                        bulk.rho_bonds[:, b] += f


def bulk_chemical_potential(ms: MolecularSystem, bulk: BulkState) -> None:
    """`evaluation/analysis/bulk_chemical_potential.jl:9-25`."""
    bulk.mu_species[:] = 0.0
    bulk.mu_ex[:] = 0.0
    bulk.lng[:] = 0.0
    sig = np.asarray(ms.diameters)
    Z = np.asarray(ms.valences)
    lB = ms.bjerrum_length
    rho = bulk.rho_beads
    for model in ms.fe_model:
        if model == "ideal":
            bulk.mu_species += np.where(bulk.rho_species > 1e-100,
                                        np.log(np.maximum(bulk.rho_species, 1e-300)), -1e20)
        elif model == "mfmt":
            n0 = float(np.sum(rho)); n1 = float(np.sum(rho * sig / 2))
            n2 = float(np.sum(rho * sig * sig * PI)); n3 = float(np.sum(rho * sig ** 3 * PI / 6))
            d1, d2, d3, d4 = mfmt_deriv_bulk(n0, n1, n2, n3)
            bulk.mu_ex += d1 + d2 * sig / 2 + d3 * PI * sig ** 2 + d4 * PI * sig ** 3 / 6
        elif model == "TPT1mfmt":
            mu, lng = tpt1mfmt_deriv_bulk(bulk.rho_bonds, ms.bond_types, rho, sig)
            bulk.mu_ex += mu
            bulk.lng += lng
        elif model == "msa":
            bulk.mu_ex += msa_deriv(rho, sig, Z, lB)
        elif model == "TPT1msa":
            dphi, lng = tpt1msa_deriv(bulk.rho_bonds, ms.bond_types, rho, sig, Z, lB)
            bulk.mu_ex += dphi
            bulk.lng += lng
        elif model == "coul":
            pass  # Psi = 0 in the bulk: mu_ex += 0 * Z
        else:
            raise NotImplementedError(f"model '{model}' is not supported")
    for u, cfg in enumerate(ms.configurations):
        if cfg.model == "monomerbead":
            Xi = _monomerbead_xi(ms, bulk, u)
            bulk.Xi[u] = Xi
            bulk.mu_species[u] -= math.log(Xi)
        else:
            lxi = _fj_log_xi(ms, bulk, u)
            bulk.Xi[u] = math.exp(lxi) if lxi < 700 else math.inf
            bulk.mu_species[u] -= lxi


def _species_in_reactions(ms: MolecularSystem) -> set:
    out = set()
    for rxn in ms.reactions:
        if all(c == 0 for c in rxn.coeffs):
            continue
        out.update(rxn.species)
    return out


def balance_charge(ms: MolecularSystem, bulk: BulkState, Q: float, adjustable: List[bool]) -> None:
    """`evaluation/objective/functions/balance_charge.jl:21-79` (strategy :equal)."""
    sc = ms.species_charge
    if Q == 0.0:
        for i in range(len(adjustable)):
            adjustable[i] = ms.compensator[i] and np.sign(sc[i]) == 1.0
        return
    sQ = float(np.sign(Q))
    for i in range(len(adjustable)):
        adjustable[i] = ms.compensator[i] and np.sign(sc[i]) == -sQ
    if not any(adjustable):
        raise RuntimeError(f"No compensating species available to absorb net charge {Q}")
    tw = float(sum(1.0 for a in adjustable if a))
    for i in range(len(adjustable)):
        if adjustable[i]:
            d = -Q * (1.0 / tw) / sc[i]
            bulk.rho_species[i] = ms.input_densities[i] + max(d, 0.0)
        elif ms.compensator[i]:
            bulk.rho_species[i] = ms.input_densities[i]


# --------------------------------------------------------------------------
# native evaluation (sdft_bulk_eval of libsoftdft.so)
# --------------------------------------------------------------------------
_MODEL_BITS = {"ideal": 1, "mfmt": 2, "TPT1mfmt": 4, "msa": 8, "TPT1msa": 16, "coul": 0}


class _BulkSpecies(ctypes.Structure):
    _fields_ = [("n_seg", ctypes.c_int32), ("max_states", ctypes.c_int32), ("max_children", ctypes.c_int32),
                ("n_levels", ctypes.c_int32), ("monomerbead", ctypes.c_int32),
                ("n_states", ctypes.c_void_p), ("states", ctypes.c_void_p), ("parent", ctypes.c_void_p),
                ("n_children", ctypes.c_void_p), ("children", ctypes.c_void_p), ("level_ptr", ctypes.c_void_p),
                ("level_segs", ctypes.c_void_p)]


class _BulkSystem(ctypes.Structure):
    _fields_ = [("nb", ctypes.c_int32), ("mb", ctypes.c_int32), ("ns", ctypes.c_int32), ("models", ctypes.c_uint32),
                ("diameter", ctypes.c_void_p), ("valence", ctypes.c_void_p), ("delta_muH", ctypes.c_void_p),
                ("bond_types", ctypes.c_void_p), ("species", ctypes.c_void_p), ("bjerrum_length", ctypes.c_double)]


def _native_bulk(ms: MolecularSystem):
    """ctypes descriptor of the molecular system for sdft_bulk_eval (cached on ms)."""
    cached = getattr(ms, "_bulk_native", None)
    if cached is not None:
        return cached
    from .. import native
    lib = native.lib()
    keep = []

    def arr(a, dt):
        v = np.ascontiguousarray(np.asarray(a, dtype=dt))
        keep.append(v)
        return v.ctypes.data

    models = 0
    for m in ms.fe_model:
        if m not in _MODEL_BITS:
            raise NotImplementedError(f"model '{m}' is not supported")
        models |= _MODEL_BITS[m]
    sp = (_BulkSpecies * len(ms.configurations))()
    seg_sizes = []
    for u, cfg in enumerate(ms.configurations):
        fam, topo = cfg.state_family, cfg.topology
        n = len(cfg.sequence)
        S = max(max(len(f) for f in fam), 1)
        C = max(max((len(c) for c in topo.children), default=0), 1)
        states = np.full((n, S), -1, dtype=np.int32)
        for g, f in enumerate(fam):
            states[g, :len(f)] = f
        children = np.full((n, C), -1, dtype=np.int32)
        for g, ch in enumerate(topo.children):
            children[g, :len(ch)] = ch
        parent = [p[0] if p else -1 for p in topo.parents]
        level_ptr = np.cumsum([0] + [len(l) for l in topo.levels])
        level_segs = [g for l in topo.levels for g in l]
        sp[u] = _BulkSpecies(n, S, C, len(topo.levels), 1 if cfg.model == "monomerbead" else 0,
                             arr([len(f) for f in fam], np.int32), arr(states, np.int32), arr(parent, np.int32),
                             arr([len(c) for c in topo.children], np.int32), arr(children, np.int32),
                             arr(level_ptr, np.int32), arr(level_segs, np.int32))
        seg_sizes.append((S, n))
    keep.append(sp)
    sysd = _BulkSystem(len(ms.monomers), len(ms.bond_types), len(ms.configurations), models,
                       arr(ms.diameters, np.float64), arr(ms.valences, np.float64), arr(ms.delta_muH, np.float64),
                       arr([x for b in ms.bond_types for x in b], np.int32), ctypes.addressof(sp),
                       float(ms.bjerrum_length))
    f = lib.sdft_bulk_eval
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 11
    cached = (lib, sysd, keep, seg_sizes)
    ms._bulk_native = cached
    return cached


def eval_bulk_state_native(ms: MolecularSystem, bulk: BulkState) -> None:
    """eval_bulk_density followed by bulk_chemical_potential in one native call."""
    lib, sysd, _, seg_sizes = _native_bulk(ms)
    nb, mb, ns = len(ms.monomers), len(ms.bond_types), len(ms.configurations)
    segs = np.zeros(sum(S * n for S, n in seg_sizes))
    rb = np.zeros(nb)
    rbo = np.zeros(2 * mb + 1)
    mus = np.zeros(ns)
    mu = np.zeros(nb)
    lng = np.zeros(mb + 1)
    xi = np.zeros(ns)
    rs = np.ascontiguousarray(bulk.rho_species, dtype=np.float64)
    mu_in = np.ascontiguousarray(bulk.mu_ex, dtype=np.float64)
    lng_in = np.ascontiguousarray(np.concatenate([bulk.lng, [0.0]]), dtype=np.float64)
    p = lambda a: a.ctypes.data
    rc = lib.sdft_bulk_eval(ctypes.byref(sysd), p(rs), p(mu_in), p(lng_in), p(segs), p(rb), p(rbo), p(mus), p(mu),
                            p(lng), p(xi))
    if rc != 0:
        raise RuntimeError(f"sdft_bulk_eval failed ({rc})")
    off = 0
    for u, (S, n) in enumerate(seg_sizes):
        bulk.rho_segments[u][:, :] = segs[off: off + S * n].reshape(n, S).T
        off += S * n
    bulk.rho_beads[:] = rb
    bulk.rho_bonds[:, :] = rbo[: 2 * mb].reshape(2, mb)
    bulk.mu_species[:] = mus
    bulk.mu_ex[:] = mu
    bulk.lng[:] = lng[:mb]
    bulk.Xi[:] = xi


# False keeps the bulk evaluation in numpy (no shared library loaded), e.g. for
# a CPU-only process that times the oracle
USE_NATIVE_BULK = True


def _use_native() -> bool:
    if not USE_NATIVE_BULK:
        return False
    from .. import native
    return native.library_present()


def residual_bulkstate(ms: MolecularSystem, bulk: BulkState, sol, adjustable, native_eval: bool = True) -> np.ndarray:
    """`evaluation/objective/residual_bulkstate.jl:26-35` +
    `functions/update_bulk_structures.jl:10-44` + `functions/eval_residuals.jl:26-60`."""
    log_rxn, log_ph, Q = sol
    balance_charge(ms, bulk, Q[0], adjustable)
    inr = _species_in_reactions(ms)
    ir = ip = 0
    for i, s in enumerate(ms.species):
        if not math.isnan(ms.input_pSpecies[i]):
            bulk.rho_species[i] = math.exp(log_ph[ip]); ip += 1
        elif s in inr:
            bulk.rho_species[i] = math.exp(log_rxn[ir]); ir += 1
    if native_eval and _use_native():
        eval_bulk_state_native(ms, bulk)
    else:
        eval_bulk_density(ms, bulk)
        bulk_chemical_potential(ms, bulk)
    res = []
    unit = concentration_to_density(1.0, ms.constants)
    for i in range(len(ms.species)):
        if not math.isnan(ms.input_pSpecies[i]):
            res.append(bulk.mu_species[i] + ms.input_pSpecies[i] * LOG10 - math.log(unit))
    for rxn in ms.reactions:
        if all(c == 0 for c in rxn.coeffs):
            continue
        musum = sum(cf * bulk.mu_species[ms.species.index(s)] for s, cf in zip(rxn.species, rxn.coeffs))
        res.append(musum - rxn.pK)
    res.append(-float(np.sum(np.asarray(ms.species_charge) * bulk.rho_species)))
    return np.asarray(res, dtype=np.float64)


def eval_bulk_pressure(ms: MolecularSystem, bulk: BulkState) -> float:
    """`evaluation/analysis/eval_pressure.jl:10-25` with `excess_free_energy.jl:10-19`."""
    sig = np.asarray(ms.diameters)
    Z = np.asarray(ms.valences)
    rho = bulk.rho_beads
    fex = 0.0
    for model in ms.fe_model:
        if model == "mfmt":
            n0 = float(np.sum(rho)); n1 = float(np.sum(rho * sig / 2))
            n2 = float(np.sum(rho * sig * sig * PI)); n3 = float(np.sum(rho * sig ** 3 * PI / 6))
            fex += free_energy_mfmt(n0, n1, n2, n3)
        elif model == "TPT1mfmt":
            fex += free_energy_tpt1mfmt_bulk(bulk.rho_bonds, ms.bond_types, rho, sig)
        elif model == "msa":
            fex += free_energy_msa(rho, sig, Z, ms.bjerrum_length)
        elif model == "TPT1msa":
            fex += free_energy_tpt1msa_bulk(bulk.rho_bonds, ms.bond_types, rho, sig, Z, ms.bjerrum_length)
    return (float(np.sum(bulk.rho_species)) - fex + float(np.sum(rho * bulk.mu_ex))
            - float(np.sum(bulk.rho_bonds[0] * bulk.lng)) / 2.0
            - float(np.sum(bulk.rho_bonds[1] * bulk.lng)) / 2.0)


class BulkDiverged(RuntimeError):
    pass


def solve_bulk(ms: MolecularSystem, numerical: dict, cap: int = 3000) -> BulkState:
    """`evaluation/objective/solver_bulkstate.jl:31-62` driving AndersonResidual
    (`src/NonlinearSolvers/residual/AndersonResidual.jl:27-138`).

    The restated driver runs first.  Its secant-projected Picard branch diverges
    when the bulk excess chemical potential is large (dense solvent, packing
    fraction >= 0.3): the projection coefficient reaches 1e4 within three
    iterations and the reference then carries -Inf/NaN until max_iters.  When
    that happens (non-finite residual, or no convergence within ``cap``
    iterations) the same residual is solved by ``_solve_bulk_robust``; both
    stop on the same max-norm residual, so they return the same bulk state to
    within the tolerance."""
    for m in ms.fe_model:
        if m not in SUPPORTED_MODELS:
            raise NotImplementedError(f"Unknown or unsupported model(s): {m}")
    charge0 = list(ms.species_charge)
    num = _bulk_numerics(numerical)
    # zeros(n, anderm) of the history (AndersonResidual.jl) needs anderm >= 1
    if numerics_int(num, "anderm", 5, False) < 1:
        raise ValueError("numerical.anderm must be at least 1")
    numerics_int(num, "max_iters", 100000, True)
    try:
        return _solve_bulk_reference(ms, numerical, cap)
    except (BulkDiverged, ValueError, OverflowError, FloatingPointError, ZeroDivisionError):
        ms.species_charge[:] = charge0
        return _solve_bulk_robust(ms, numerical)


def _bulk_numerics(numerical: dict) -> dict:
    num = {"mixing_max": 0.1, "tole": 1e-10, "damping": 0.1}
    num.update({k: float(v) for k, v in numerical.items()})
    return num


def _initial_solution(ms: MolecularSystem, bulk: BulkState):
    """assign_solution_variables (`solver_bulkstate.jl:65-103`)."""
    inr = _species_in_reactions(ms)
    log_rxn, log_ph = [], []
    for i, s in enumerate(ms.species):
        if not math.isnan(ms.input_pSpecies[i]):
            log_ph.append(math.log(bulk.rho_species[i]))
        elif s in inr:
            log_rxn.append(math.log(bulk.rho_species[i]))
    sizes = (len(log_rxn), len(log_ph), 1)

    def unflat(x):
        a, b = sizes[0], sizes[0] + sizes[1]
        return (list(x[:a]), list(x[a:b]), [x[b]])

    return np.asarray(log_rxn + log_ph + [0.0], dtype=np.float64), unflat


def _solve_bulk_robust(ms: MolecularSystem, numerical: dict) -> BulkState:
    """Undamped Picard x <- x - F(x) accelerated by Anderson mixing (type II,
    depth 5) on the reference's bulk residual.  dF/dx is close to the identity
    here: the pSpecies residuals are log-density offsets and the neutrality
    residual moves one-for-one with the compensator charge."""
    num = _bulk_numerics(numerical)
    tole = min(num.get("tole", 1e-6), 1e-10)
    bulk = initialize_densities(ms)
    adjustable = list(ms.adjustable)
    Xk, unflat = _initial_solution(ms, bulk)
    m = 5
    hx, hf = [], []
    err = math.inf
    for it in range(1, 2001):
        Fk = residual_bulkstate(ms, bulk, unflat(Xk), adjustable)
        if not np.all(np.isfinite(Fk)):
            raise RuntimeError("bulk solve: non-finite residual")
        err = float(np.max(np.abs(Fk)))
        if err < tole:
            break
        G = Xk - Fk
        hx.append(Xk.copy()); hf.append(Fk.copy())
        if len(hx) > m:
            hx.pop(0); hf.pop(0)
        if len(hx) >= 2:
            dF = np.stack([hf[i + 1] - hf[i] for i in range(len(hf) - 1)], axis=1)
            dX = np.stack([hx[i + 1] - hx[i] for i in range(len(hx) - 1)], axis=1)
            gam, *_ = np.linalg.lstsq(dF, Fk, rcond=None)
            Xk = G - (dX - dF) @ gam
        else:
            Xk = G
    else:
        raise RuntimeError(f"bulk solve did not converge (residual {err})")
    bulk.iterations = it
    bulk.residual = err
    bulk.pressure = eval_bulk_pressure(ms, bulk)
    bulk.numerics = num
    bulk.numerics["bulk_solver"] = "picard-anderson"
    return bulk


def _solve_bulk_reference(ms: MolecularSystem, numerical: dict, cap: int) -> BulkState:
    bulk = initialize_densities(ms)
    num = _bulk_numerics(numerical)
    max_iters = numerics_int(num, "max_iters", 100000, True)
    damping = num.get("damping", 0.1)
    mix_max = num.get("mixing_max", 0.1)
    switch_mix = num.get("switch_mix", 1e-4)
    tole = num.get("tole", 1e-6)
    m = numerics_int(num, "anderm", 5, False)
    adjustable = list(ms.adjustable)
    Xk, unflat = _initial_solution(ms, bulk)
    n = Xk.size
    X = np.zeros((n, m)); F = np.zeros((n, m))
    Fk = residual_bulkstate(ms, bulk, unflat(Xk), adjustable)
    X[:, 0] = Xk; F[:, 0] = Fk
    lambdas = np.zeros(m - 1)
    it = 0
    err = 1.0
    while it < max_iters:
        it += 1
        if it > cap:
            raise BulkDiverged(f"no convergence within {cap} iterations")
        Fk = residual_bulkstate(ms, bulk, unflat(Xk), adjustable)
        if not np.all(np.isfinite(Fk)):
            raise BulkDiverged("non-finite bulk residual")
        err = max(float(np.max(np.abs(Fk))), 1e-20)
        amix = min(mix_max, damping / err)
        col = it % m
        X[:, col] = Xk; F[:, col] = Fk
        if it < m or err > switch_mix:
            prev = (it - 1) % m
            dX = Xk - X[:, prev]
            dF = Fk - F[:, prev]
            numer = float(Fk @ dF); denom = float(dF @ dF)
            lam = 0.0 if denom == 0.0 else numer / denom
            Xk = Xk - lam * dX - amix * (Fk - lam * dF)
        else:
            cols = [j for j in range(m) if j != col]
            tX = X[:, cols] - Xk[:, None]
            tF = F[:, cols] - Fk[:, None]
            lsqr_inplace(lambdas, tF, -Fk)
            Xk = Xk + tX @ lambdas + amix * (Fk + tF @ lambdas)
        if err < tole:
            break
    # the solution tuple is left at the last mixed iterate, as in the reference
    bulk.iterations = it
    bulk.residual = err
    bulk.pressure = eval_bulk_pressure(ms, bulk)
    bulk.numerics = num
    return bulk
