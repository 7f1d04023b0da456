"""Host-side setup mirror: input.yaml -> molecular system, bulk state, grid."""
import math

import numpy as np
import pytest

from softdft_b200 import workloads
from softdft_b200.host import geometry, ilst, molsys, yamlio
from softdft_b200.host.descriptor import build_descriptor, numerics_from_dict

YAML = """
procedure: iDFT
geometry:
  coordinate_system: Cartesian
  dimensions: [10.0]
  bin_width: [0.05]
  external_field:
    hard_walls:
      dims: [1]
    charged_walls:
      dims: [1]
      charge: [-0.05, -0.05]
species:
  - sequence: "AAAAA"
    concentration: 0.05
  - sequence: "c"
    concentration: 0.02
    adjustable: true
  - sequence: "a"
    concentration: 0.02
    adjustable: true
  - sequence: "Y"
    pSpecies: 6.0
  - sequence: "Z"
reactions:
  - species: ["A", "Y", "B"]
    coeffs: [-1, +1, +1]
    pK: 4.0
  - species: ["Y", "Z"]
    coeffs: [+1, +1]
    pK: 14.0
monomers:
  A: {diameter: 1.0, valence: 0.0}
  B: {diameter: 1.0, valence: -1.0}
  c: {diameter: 1.0, valence: 1.0}
  a: {diameter: 1.0, valence: -1.0}
  Y: {diameter: 1.0, valence: 1.0}
  Z: {diameter: 1.0, valence: -1.0}
numerical:
  damping: 0.01
  mixing_max: 0.001
  tole: 1e-6
model: [ideal, TPT1mfmt, TPT1msa]
"""


def test_yaml_exponent_floats():
    d = yamlio.load_text("a: 1e-6\nb: 2E+3\nc: text")
    assert d["a"] == 1e-6 and d["b"] == 2000.0 and d["c"] == "text"


def test_molecular_system_state_families_and_dmuH():
    ds = yamlio.load_text(YAML)
    ms = molsys.molecular_system(ds)
    assert ms.monomers == ["A", "B", "Y", "Z", "a", "c"]
    assert ms.state_families["A"] == ["A", "B"] and ms.state_families["c"] == ["c"]
    # A -> B + Y with pK 4 at pSpecies 6: dmuH_B = ln10 (pK - pH)
    assert ms.delta_muH[ms.used["B"]] == pytest.approx(math.log(10) * (4.0 - 6.0), rel=1e-14)
    assert ms.delta_muH[ms.used["A"]] == 0.0
    # the water reaction fixes pZ = 14 - pY and becomes bookkeeping
    assert ms.input_pSpecies[4] == pytest.approx(8.0, rel=1e-14)
    assert all(c == 0 for r in ms.reactions for c in r.coeffs)
    assert ms.bond_types == [(0, 0), (0, 1), (1, 1)]
    # Bjerrum length at the default 298.15 K / 78.4 (the `system:` keys are not read)
    assert ms.bjerrum_length == pytest.approx(1.4297414291151598, rel=1e-12)


def test_topology_parser_branches_and_repeats():
    t = molsys.parse_topology("A(BC)2D")
    assert t.monomers == "ABCBCD"
    assert t.parents == [[], [0], [1], [0], [3], [0]]
    assert t.children[0] == [1, 3, 5]
    assert t.levels == [[0], [1, 3, 5], [2, 4]]
    lin = molsys.parse_topology("AAAA")
    assert lin.parents == [[], [0], [1], [2]] and lin.levels == [[0], [1], [2], [3]]


def test_grid_rule_cld():
    assert geometry.cld(20.0, 0.02) == 1000
    assert geometry.cld(workloads.slit_length(1024, 0.02), 0.02) + 1 == 1024
    assert geometry.cld(workloads.slit_length(16384, 0.01), 0.01) + 1 == 16384


def test_bulk_solution_residual_and_neutrality():
    ds = yamlio.load_text(YAML)
    ms = molsys.molecular_system(ds)
    bulk = ilst.solve_bulk(ms, ds["numerical"])
    assert bulk.residual < 1e-6
    # electroneutrality with the ideal per-chain charge the reference uses
    q = float(np.sum(np.asarray(ms.species_charge) * bulk.rho_species))
    assert abs(q) < 1e-6
    # pSpecies constraint: mu_Y = ln(unit * 10^-pY)
    unit = molsys.concentration_to_density(1.0, ms.constants)
    assert bulk.mu_species[3] == pytest.approx(math.log(unit) - 6.0 * math.log(10), abs=1e-5)
    assert bulk.pressure > 0


def test_bulk_dense_solvent_converges():
    ds = workloads.plain_slit()
    ms = molsys.molecular_system(ds)
    bulk = ilst.solve_bulk(ms, ds["numerical"])
    assert bulk.residual < 1e-8
    assert 6.0 < bulk.mu_ex[0] < 7.0


def test_descriptor_layout():
    ds = workloads.weak_acid_slit(128, 0.05, 6, 4.5, 7.0, 0.1, 0.3)
    ms = molsys.molecular_system(ds)
    bulk = ilst.solve_bulk(ms, ds["numerical"])
    g = geometry.geometry_system(ds)
    d = build_descriptor(ds, ms, bulk, g)
    assert d.np_ == 128 and d.nb == 7 and d.mb == 3
    assert d.n_unknowns == 128 * (7 + 6 + 1) + 1
    assert d.desc.functionals == 0x2 | 0x8
    num = numerics_from_dict(ds["numerical"])
    assert num.anderm == 5 and num.tole == 1e-8


def test_grafted_coordinates():
    ds = workloads.grafted_brush(256, 0.05, 10, 0.05, 4.5, 7.0, 0.01)
    ms = molsys.molecular_system(ds)
    bulk = ilst.solve_bulk(ms, ds["numerical"])
    g = geometry.geometry_system(ds)
    d = build_descriptor(ds, ms, bulk, g)
    # left: round(0/dz)+1 + round(sigma/2/dz) (1-based) -> 0-based 10; right: NP-1-10
    assert d.fixed_coord[0][0] == 10 and d.fixed_coord[1][0] == 255 - 10
    assert all(c < 0 for c in d.fixed_coord[0][1:])
