"""Molecular system: input.yaml -> species, state families, dmuH, topology, bonds.

Host-side restatement of the reference's `src/molecular_system/` setup
(`setup/setup_molsys.jl:48-75`).  Every function names the reference function it
follows; behaviour (including the quirks listed in each docstring) is kept so that
the descriptor handed to the device solve carries the same numbers the
reference's Julia setup would produce.

Indices are 0-based here; the reference is 1-based.  Bead ("monomer") types are
the sorted monomer names (`species/chemistry/used_monomers.jl:42-48`).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

from .yamlio import as_float

LOG10 = math.log(10.0)


# --------------------------------------------------------------------------
# constants and system properties
# --------------------------------------------------------------------------
@dataclass
class Constants:
    """`structures/ConstantsStruct.jl:18-24` (SI values)."""

    epsilon0: float = 8.854187817e-12
    e0: float = 1.60217653e-19
    k_B: float = 1.3806505e-23
    NA: float = 6.0221415e23
    l_sc: float = 0.5e-9


def process_constants(dataset: dict) -> Constants:
    """`setup/core/constants/process_constants.jl:10-16`: l_sc in nm, default 0.5 nm."""
    ru = dataset.get("reduced_units")
    if isinstance(ru, dict) and "l_sc" in ru:
        return Constants(l_sc=as_float(ru["l_sc"]) * 1e-9)
    return Constants()


def concentration_to_density(conc: float, c: Constants) -> float:
    """mol/L -> 1/l_sc^3 (`setup/core/conversions/conversions.jl:19-22`)."""
    vol_liters = c.l_sc ** 3 * 1000.0
    return conc * c.NA * vol_liters


def density_to_concentration(rho: float, c: Constants) -> float:
    """1/l_sc^3 -> mol/L (`setup/core/conversions/conversions.jl:8-12`)."""
    vol_liters = c.l_sc ** 3 * 1000.0
    return rho / vol_liters / c.NA


def _constraint_value(dataset: dict, key: str, default: float) -> float:
    """Temperature and dielectric constant are read from the ``constraints``
    section, not ``system`` (`setup/core/system/get_temperature.jl:14-21`,
    `get_dielectric_constant.jl:15-22`); the value must be a float."""
    cons = dataset.get("constraints")
    if isinstance(cons, dict) and key in cons:
        v = cons[key]
        if not isinstance(v, float):
            raise ValueError(f"{key} must be a Float64 value.")
        return v
    return default


def process_system(dataset: dict, c: Constants) -> Dict[str, float]:
    """`setup/core/system/process_system.jl:15-26` with the Bjerrum length of
    `get_Bjerrumlength.jl:12-14` in units of l_sc."""
    T = _constraint_value(dataset, "temperature", 298.15)
    er = _constraint_value(dataset, "dielectric_constant", 78.4)
    bj = c.e0 ** 2 / (4 * math.pi * c.epsilon0 * er * c.k_B * T) / c.l_sc
    return {"temperature": T, "dielectric_constant": er, "bjerrum_length": bj}


# --------------------------------------------------------------------------
# topology
# --------------------------------------------------------------------------
@dataclass
class Topology:
    """`structures/TopologyStruct.jl:23-30` (0-based)."""

    monomers: str
    children: List[List[int]]
    parents: List[List[int]]
    levels: List[List[int]]
    sequ_bonds: List[Tuple[int, int]]


def parse_topology(sequence: str) -> Topology:
    """Recursive descent over letters, ``(group)`` and ``(group)k`` repeats
    (`setup/configurations/parse_topology.jl:16-127`).  A letter's parent is the
    letter before it at the enclosing nesting level; a group repeats ``k`` times
    from the same parent and level.  The reference's children array grows one
    spurious trailing empty entry for single letters; only the first ``n``
    entries are kept here."""
    monomers: List[str] = []
    children: List[List[int]] = []
    parents: List[List[int]] = []
    levels: List[List[int]] = []
    sequ_bonds: List[Tuple[int, int]] = []
    state = {"current": 0, "last_linear": 0}

    def matching(seq: str) -> int:
        bal = 1
        for j in range(1, len(seq)):
            if seq[j] == "(":
                bal += 1
            elif seq[j] == ")":
                bal -= 1
            if bal == 0:
                return j
        raise ValueError(f"Unmatched parenthesis in: {seq}")

    def recurse(sub: str, level: int, parent: int) -> None:
        ch = sub[0]
        if ch.isalpha():
            state["current"] += 1
            cur = state["current"]
            monomers.append(ch)
            if level > len(levels):
                levels.append([])
            levels[level - 1].append(cur)
            if parent == 0:
                children.append([])
                parents.append([])
            else:
                if parent > len(children):
                    children.append([cur])
                else:
                    children[parent - 1].append(cur)
                if cur > len(parents):
                    parents.append([parent])
                else:
                    parents[cur - 1].append(parent)
            if state["last_linear"] != 0:
                sequ_bonds.append((state["last_linear"], cur))
            state["last_linear"] = cur
            if len(sub) > 1:
                recurse(sub[1:], level + 1, cur)
            else:
                children.append([])
        elif ch == "(":
            end = matching(sub)
            group = sub[1:end]
            remaining = sub[end + 1:]
            mult = 1
            if remaining and remaining[0].isdigit():
                i = 0
                while i < len(remaining) and remaining[i].isdigit():
                    i += 1
                mult = int(remaining[:i])
                remaining = remaining[i:]
            for _ in range(mult):
                recurse(group, level, parent)
            if remaining:
                recurse(remaining, level, parent)
        else:
            raise ValueError(f"Not a recognized character: {ch}")

    recurse(sequence, 1, 0)
    n = len(monomers)
    to0 = lambda lst: [x - 1 for x in lst]
    return Topology(
        monomers="".join(monomers),
        children=[to0(c) for c in children[:n]] + [[] for _ in range(max(0, n - len(children)))],
        parents=[to0(p) for p in parents[:n]],
        levels=[to0(l) for l in levels],
        sequ_bonds=[(a - 1, b - 1) for a, b in sequ_bonds],
    )


# --------------------------------------------------------------------------
# chemistry
# --------------------------------------------------------------------------
@dataclass
class Reaction:
    """`structures/ReactionStruct.jl:24-28`; ``coeffs`` are zeroed once a reaction
    is resolved into dmuH (bookkeeping reaction)."""

    species: List[str]
    coeffs: List[int]
    pK: float


@dataclass
class SpeciesEntry:
    """`species/chemistry/parse_species.jl:29-36`."""

    name: str
    density: float
    concentration: float
    pSpecies: float
    adjustable: bool
    role: str


def parse_reactions(dataset: dict) -> List[Reaction]:
    """`species/chemistry/parse_reactions.jl:30-73`: coefficients must be +-1."""
    raw = dataset.get("reactions")
    if raw is None:
        return []
    if not isinstance(raw, list):
        raise ValueError("Expected 'reactions' to be a list of reaction entries")
    out = []
    for rxn in raw:
        species = [str(s) for s in rxn["species"]]
        coeffs_raw = rxn["coeffs"]
        if len(species) != len(coeffs_raw):
            raise ValueError(f"Mismatch between number of species and coefficients in reaction: {rxn}")
        coeffs = []
        for c in coeffs_raw:
            c = as_float(c)
            ci = int(round(c))
            if abs(c - ci) > 1e-8:
                raise ValueError(f"Non-integer stoichiometric coefficient {c} in reaction: {rxn}")
            if ci not in (1, -1):
                raise ValueError(f"Unsupported coefficient {ci} in reaction: {rxn}")
            coeffs.append(ci)
        out.append(Reaction(species, coeffs, as_float(rxn["pK"])))
    return out


def parse_species(dataset: dict) -> List[SpeciesEntry]:
    """`species/chemistry/parse_species.jl:38-82` including its exclusivity rules."""
    if "species" not in dataset:
        raise ValueError("Input file is missing the required 'species' section.")
    out = []
    for entry in dataset["species"]:
        if "sequence" not in entry:
            raise ValueError("Each species must define a 'sequence' field.")
        name = str(entry["sequence"])
        has_d, has_c, has_p = "density" in entry, "concentration" in entry, "pSpecies" in entry
        adjustable = bool(entry.get("adjustable", False))
        role = str(entry.get("role", "monomer"))
        if (has_d or has_c) and has_p:
            raise ValueError(f"Species '{name}' is overspecified: both 'density/concentration' and 'pSpecies' are defined.")
        if has_d and has_c:
            raise ValueError(f"Species '{name}' is overspecified: both 'density' and 'concentration'.")
        if has_p and adjustable:
            raise ValueError(f"Species '{name}' has 'pSpecies' and is also marked as 'adjustable'.")
        out.append(SpeciesEntry(
            name,
            as_float(entry.get("density", 0.0)),
            as_float(entry.get("concentration", 0.0)),
            as_float(entry["pSpecies"]) if has_p else math.nan,
            adjustable,
            role,
        ))
    return out


def build_used_monomers(species_data: list, reactions: List[Reaction]) -> Dict[str, int]:
    """Letters of every sequence plus every reaction species, sorted by name
    (`species/chemistry/used_monomers.jl:29-48`)."""
    names = set()
    for entry in species_data:
        for ch in str(entry["sequence"]):
            if ch.isalpha():
                names.add(ch)
    for rxn in reactions:
        names.update(rxn.species)
    return {n: i for i, n in enumerate(sorted(names))}


def _neutralization_participants(reactions: List[Reaction]) -> set:
    """`state_families.jl:213-231`."""
    out = set()
    for rxn in reactions:
        reac = [s for s, c in zip(rxn.species, rxn.coeffs) if c == -1]
        prod = [s for s, c in zip(rxn.species, rxn.coeffs) if c == +1]
        if not reac or not prod:
            out.update(prod if not reac else reac)
    return out


def build_state_families(entries: List[SpeciesEntry], reactions: List[Reaction]) -> Dict[str, List[str]]:
    """Connected components of the monomer graph induced by reactions
    (`species/chemistry/state_families.jl:1-90,140-166`)."""
    neutral = _neutralization_participants(reactions)
    for e in entries:
        if e.name in neutral:
            e.role = "neutralizer"
    roles = {e.name: e.role for e in entries}
    polymer_monomers = set()
    for e in entries:
        if len(e.name) > 1:
            polymer_monomers.update(ch for ch in e.name if ch.isalpha())
    neighbors: Dict[str, set] = {}
    pending = []
    for rxn in reactions:
        reac = [s for s, c in zip(rxn.species, rxn.coeffs) if c == -1]
        prod = [s for s, c in zip(rxn.species, rxn.coeffs) if c == +1]
        if not reac or not prod:
            for s in (prod if not reac else reac):
                if s in polymer_monomers:
                    raise ValueError(f"Monomer '{s}' appears in a neutralization reaction, but it is part of a polymer sequence.")
            continue
        r, p = len(reac), len(prod)
        if not ((r == 1 and p in (1, 2)) or (r == 2 and p == 1)):
            raise ValueError(f"Unsupported reaction form: {rxn.species} with coeffs {rxn.coeffs}")
        if r == 2 and p == 1 and all(roles.get(x, "monomer") == "monomer" for x in reac):
            raise ValueError(f"Reaction {rxn.species} has two reactants and one product, but both reactants are :monomer.")
        if r == 1 and p == 2 and all(roles.get(x, "monomer") == "monomer" for x in prod):
            raise ValueError(f"Reaction {rxn.species} has one reactant and two products, but both products are :monomer.")
        lhs = [s for s in reac if roles.get(s, "monomer") not in ("partner", "neutralizer")]
        rhs = [s for s in prod if roles.get(s, "monomer") not in ("partner", "neutralizer")]
        tot = len(lhs) + len(rhs)
        if tot > 2:
            raise ValueError(f"Reaction {rxn.species} connects more than two candidate monomers.")
        if tot == 2:
            # both candidates on one side cannot pair lhs[0] with rhs[0]; the
            # reference indexes lhs[1], rhs[1] and would throw a BoundsError
            if not lhs or not rhs:
                raise ValueError(f"Reaction {rxn.species}: candidate monomers on one side only.")
            a, b = lhs[0], rhs[0]
            neighbors.setdefault(a, set()).add(b)
            neighbors.setdefault(b, set()).add(a)
        elif tot == 1:
            pending.append((reac, prod))
    # resolve_pending_edges! (`state_families.jl:93-125`)
    for reac, prod in pending:
        cands = [s for s in list(dict.fromkeys(reac + prod)) if roles.get(s) == "monomer"]
        if len(cands) != 2:
            continue
        a, b = cands
        fa, fb = _component(neighbors, a), _component(neighbors, b)
        neighbors.setdefault(a, set())
        neighbors.setdefault(b, set())
        if a in fb or b in fa:
            continue
        neighbors[a].add(b)
        neighbors[b].add(a)
    all_monomers = set()
    for e in entries:
        all_monomers.update(ch for ch in e.name if ch.isalpha())
    visited = set()
    families: Dict[str, List[str]] = {}
    for mon in sorted(all_monomers):
        if mon in visited:
            continue
        group = []
        stack = [mon]
        while stack:
            node = stack.pop()
            if node not in visited:
                visited.add(node)
                group.append(node)
                stack.extend(neighbors.get(node, ()))
        group = sorted(group)
        for m in group:
            families[m] = group
    return families


def _component(neighbors: Dict[str, set], start: str) -> set:
    seen, stack = set(), [start]
    while stack:
        n = stack.pop()
        if n in seen:
            continue
        seen.add(n)
        stack.extend(neighbors.get(n, ()))
    return seen


# --------------------------------------------------------------------------
# configurations
# --------------------------------------------------------------------------
@dataclass
class Configuration:
    """`structures/ConfigurationStruct.jl:41-47` plus the freely-jointed
    max-distance matrix (`species_model/freely_jointed.jl:9-16`)."""

    model: str                  # "freely_jointed" or "monomerbead"
    sequence: List[int]         # bead type per segment
    states: List[int]           # number of states per segment
    topology: Topology
    state_family: List[List[int]]
    max_distance: Optional[List[List[float]]] = None


def process_configurations(dataset: dict, used: Dict[str, int], families: Dict[str, List[str]]) -> List[Configuration]:
    """`setup/configurations/process_configs.jl:25-83`."""
    out = []
    for sp in dataset["species"]:
        topo = parse_topology(str(sp["sequence"]))
        n = len(topo.monomers)
        model = str(sp.get("model", "freely_jointed"))
        if model not in ("freely_jointed", "monomerbead"):
            raise ValueError(f"Unknown chain model {model}.")
        seq, states, fam = [], [], []
        for ch in topo.monomers:
            if ch not in used:
                raise ValueError(f"Monomer {ch} not found in used_monomers.")
            seq.append(used[ch])
            if ch in families:
                idxs = [used[x] for x in families[ch]]
                states.append(len(idxs))
                fam.append(idxs)
            else:
                states.append(1)
                fam.append([used[ch]])
        out.append(Configuration(model, seq, states, topo, fam))
    return out


def process_bonds(configs: List[Configuration]) -> List[Tuple[int, int]]:
    """Sorted unique (min, max) state pairs over every parent-child bond
    (`setup/configurations/process_bonds.jl:8-29`)."""
    bonds = set()
    for cfg in configs:
        for level in cfg.topology.levels:
            for child in level:
                for j in cfg.state_family[child]:
                    for parent in cfg.topology.parents[child]:
                        for j1 in cfg.state_family[parent]:
                            bonds.add((min(j, j1), max(j, j1)))
    return sorted(bonds)


def max_distance_matrix(cfg: Configuration, diameters: List[float]) -> List[List[float]]:
    """Bidirectional BFS path lengths with bond length (d_i + d_j)/2
    (`species_model/freely_jointed.jl:45-113`)."""
    n = len(cfg.sequence)
    topo = cfg.topology
    mat = [[0.0] * n for _ in range(n)]
    for start in range(n):
        dist = [0.0] * n
        queue = [(start, 0.0)]
        visited = {start}
        while queue:
            cur, d = queue.pop(0)
            for nb in list(topo.children[cur]) + list(topo.parents[cur]):
                if nb not in visited and nb < n:
                    dij = (diameters[cfg.sequence[cur]] + diameters[cfg.sequence[nb]]) / 2.0
                    nd = d + dij
                    dist[nb] = max(dist[nb], nd)
                    queue.append((nb, nd))
                    visited.add(nb)
        mat[start] = dist
    for i in range(n):
        mat[i][i] = 0.0
    return mat


# --------------------------------------------------------------------------
# molecular system
# --------------------------------------------------------------------------
@dataclass
class MolecularSystem:
    """`structures/MolecularSystem.jl:33-37` flattened into plain fields."""

    constants: Constants
    system: Dict[str, float]
    fe_model: List[str]
    species: List[str]                       # sequence strings (species names)
    monomers: List[str]                      # sorted bead-type names
    used: Dict[str, int]
    state_families: Dict[str, List[str]]
    reactions: List[Reaction]
    configurations: List[Configuration]
    bond_types: List[Tuple[int, int]]
    diameters: List[float]
    valences: List[float]
    delta_muH: List[float]
    input_densities: List[float]
    input_pSpecies: List[float]
    adjustable: List[bool]
    compensator: List[bool]
    species_charge: List[float]
    monomer_props: Dict[str, List[float]] = field(default_factory=dict)

    @property
    def bjerrum_length(self) -> float:
        return self.system["bjerrum_length"]


def process_monomers(used: Dict[str, int], dataset: dict) -> Dict[str, List[float]]:
    """Scalar monomer properties pluralised ("diameter" -> "diameters"), zero where a
    monomer does not set them (`species/properties/process_monomers.jl:35-70`)."""
    data = dataset.get("monomers") or {}
    nb = len(used)
    props: Dict[str, List[float]] = {}
    for name, idx in sorted(used.items(), key=lambda kv: kv[1]):
        if name not in data:
            raise ValueError(f"Species {name} listed in used_monomers not found in dataset[\"monomers\"]")
        if not isinstance(data[name], dict):
            raise ValueError(f"the properties of monomer {name} must be a mapping")
        for key, value in data[name].items():
            if isinstance(value, dict):
                continue  # nested properties are unused on the solve path
            pk = str(key) + "s"
            props.setdefault(pk, [0.0] * nb)[idx] = as_float(value)
    return props


def assign_delta_muH(ms_props: Dict[str, List[float]], used: Dict[str, int], families: Dict[str, List[str]],
                     reactions: List[Reaction], names: List[str], densities: List[float],
                     pSpecies: List[float], c: Constants) -> List[float]:
    """Ideal protonation work per bead type relative to the alphabetically first
    member of its state family (`species/properties/assign_delta_muH.jl:50-248`).

    Mutates ``pSpecies`` (a neutralisation partner inherits pK_w - pSpecies) and
    zeroes the coefficients of every reaction it resolves, exactly as the
    reference does."""
    name_to_index = {n: i for i, n in enumerate(names)}
    delta = [0.0] * len(used)
    # step 1: neutralisation partners
    for rxn in reactions:
        reac = [s for s, cf in zip(rxn.species, rxn.coeffs) if cf == -1]
        prod = [s for s, cf in zip(rxn.species, rxn.coeffs) if cf == +1]
        if not reac or not prod:
            mon1, mon2 = prod if not reac else reac
            dmu_total = -LOG10 * rxn.pK
            i1, i2 = name_to_index[mon1], name_to_index[mon2]
            p1, p2 = pSpecies[i1], pSpecies[i2]
            if not math.isnan(p1):
                d1 = -LOG10 * p1
                pSpecies[i2] = (dmu_total - d1) / -LOG10
            elif not math.isnan(p2):
                d2 = -LOG10 * p2
                pSpecies[i1] = (dmu_total - d2) / -LOG10
    # step 2: dmu graph
    graph: Dict[str, List[Tuple[str, float]]] = {}
    valences = ms_props.get("valences")
    for rxn in reactions:
        species, coeffs = rxn.species, rxn.coeffs
        reac = [s for s, cf in zip(species, coeffs) if cf == -1]
        prod = [s for s, cf in zip(species, coeffs) if cf == +1]
        if valences is not None:
            dq = 0.0
            for sp, cf in zip(species, coeffs):
                if sp in used:
                    dq += cf * valences[used[sp]]
            if abs(dq) > 1e-6:
                raise ValueError(f"Reaction {species} violates charge neutrality: dq = {dq}")
        sr = [s for s in reac if s in families]
        spd = [s for s in prod if s in families]
        found = False
        mon1 = mon2 = ""
        fam1: List[str] = []
        for r in sr:
            for p in spd:
                mon1, mon2 = r, p
                fam1 = families[mon1]
                if families[mon1] == families[mon2]:
                    found = True
                    break
            if found:
                break
        if not found:
            continue
        base = sorted(fam1)[0]
        fwd = mon1 == base
        frm, to = (mon1, mon2) if fwd else (mon2, mon1)
        dmu = LOG10 * rxn.pK
        for sp, cf in zip(species, coeffs):
            if sp == mon1 or sp == mon2:
                continue
            idx = name_to_index.get(sp)
            if idx is None:
                raise ValueError(f"Context species {sp} is not defined in species list.")
            ps = pSpecies[idx]
            if not math.isnan(ps):
                dmu -= LOG10 * ps * cf
            else:
                rho = densities[idx]
                if rho > 0:
                    conc = density_to_concentration(rho, c)
                    dmu += cf * -math.log(conc)
                else:
                    dmu = 0.0
        graph.setdefault(frm, []).append((to, dmu))
        graph.setdefault(to, []).append((frm, dmu))
        rxn.coeffs = [0] * len(rxn.coeffs)
    # step 3: accumulate from each family's base along the graph
    for fam in families.values():
        base = sorted(fam)[0]
        work = {base: 0.0}
        visited = set()

        def dfs(mon, acc):
            visited.add(mon)
            for nb, dmu in graph.get(mon, []):
                if nb not in visited:
                    work[nb] = acc + dmu
                    dfs(nb, acc + dmu)

        dfs(base, 0.0)
        for mon, val in work.items():
            delta[used[mon]] = val
        delta[used[base]] = 0.0
    # step 4: neutralisation reactions with a defined pSpecies become bookkeeping
    for rxn in reactions:
        reac = [s for s, cf in zip(rxn.species, rxn.coeffs) if cf == -1]
        prod = [s for s, cf in zip(rxn.species, rxn.coeffs) if cf == +1]
        if (not reac or not prod) and all(cf != 0 for cf in rxn.coeffs):
            mon1, mon2 = prod if not reac else reac
            p1, p2 = pSpecies[name_to_index[mon1]], pSpecies[name_to_index[mon2]]
            if not math.isnan(p1) or not math.isnan(p2):
                rxn.coeffs = [0] * len(rxn.coeffs)
    return delta


def parse_free_energy(models_raw) -> List[str]:
    """`setup/core/parse_free_energy.jl:24-31`."""
    if isinstance(models_raw, str):
        return [models_raw]
    return [str(m) for m in models_raw]


def molecular_system(dataset: dict) -> MolecularSystem:
    """`setup/setup_molsys.jl:48-75`."""
    c = process_constants(dataset)
    system = process_system(dataset, c)
    fe_model = parse_free_energy(dataset["model"])
    reactions = parse_reactions(dataset)
    species_data = dataset["species"]
    entries = parse_species(dataset)
    used = build_used_monomers(species_data, reactions)
    families = build_state_families(entries, reactions)
    names = [str(s["sequence"]) for s in species_data]
    densities = []
    for s in species_data:
        if "concentration" in s:
            densities.append(concentration_to_density(as_float(s["concentration"]), c))
        else:
            densities.append(as_float(s.get("density", 0.0)))
    pS = [as_float(s["pSpecies"]) if "pSpecies" in s else math.nan for s in species_data]
    adjustable = [bool(s.get("adjustable", False)) for s in species_data]
    compensator = list(adjustable)
    configs = process_configurations(dataset, used, families)
    bonds = process_bonds(configs)
    props = process_monomers(used, dataset)
    delta = assign_delta_muH(props, used, families, reactions, names, densities, pS, c)
    nb = len(used)
    valences = props.get("valences", [0.0] * nb)
    diameters = props.get("diameters")
    # assign_species_charge! (`species/properties/assign_species_charge.jl:1-20`)
    charge = [sum(valences[m] for m in cfg.sequence) for cfg in configs] if "valences" in props else [0.0] * len(configs)
    # bonding_constraint (`configurations/species_model/process_bonding.jl:12-16`)
    for cfg in configs:
        if cfg.model == "freely_jointed":
            if diameters is None:
                raise ValueError("Missing 'diameters' in properties.monomers. This is required for freely_jointed species_model.")
            cfg.max_distance = max_distance_matrix(cfg, diameters)
    return MolecularSystem(
        constants=c, system=system, fe_model=fe_model, species=names, monomers=sorted(used, key=used.get),
        used=used, state_families=families, reactions=reactions, configurations=configs, bond_types=bonds,
        diameters=list(diameters) if diameters is not None else [0.0] * nb, valences=list(valences),
        delta_muH=delta, input_densities=densities, input_pSpecies=pS, adjustable=adjustable,
        compensator=compensator, species_charge=charge, monomer_props=props,
    )
