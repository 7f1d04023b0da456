"""The library's host input pipeline (sdft_input_from_yaml: YAML subset,
molecular system, bulk solve, slit, descriptor) against the Python host
(softdft_b200/host) on the same input.yaml text.

Setup quantities (grid, walls, bead properties, dmuH, bonds, topologies, state
families, fixed segments, max-distance matrices, Bjerrum length, numerics) must
agree exactly.  The bulk-state chemical potentials come out of the same residual
(sdft_bulk_eval) and the same iteration, but the Python driver's dot products
and norms run through numpy/BLAS in another summation order, so the two
iterations stop at neighbouring iterates; they are compared at 1e-9 relative
(the bulk solves stop at a residual of 1e-10 or tole).
"""
import copy

import numpy as np
import pytest
import yaml

from softdft_b200 import native, workloads
from softdft_b200.api import setup_request
from softdft_b200.host import yamlio
from softdft_b200.host.descriptor import numerics_from_dict

from test_host_setup import YAML

pytestmark = pytest.mark.skipif(not native.library_present(), reason="libsoftdft.so not built")


def _arr(p, n):
    return np.ctypeslib.as_array(p, (n,)).copy() if n else np.zeros(0)


def _compare(text):
    ds = yamlio.load_text(text)
    dft = setup_request(copy.deepcopy(ds))
    py = dft.descriptor.desc
    inp = native.Input(text)
    cc = inp.descriptor().desc
    for k in ("np", "bin_width", "length", "hard_walls", "charged_walls", "bjerrum_length", "nb", "mb", "n_species",
              "functionals"):
        assert getattr(py, k) == getattr(cc, k), k
    assert list(py.wall_charge) == list(cc.wall_charge)
    for k in ("diameter", "valence", "delta_muH"):
        np.testing.assert_array_equal(_arr(getattr(cc, k), cc.nb), _arr(getattr(py, k), py.nb), err_msg=k)
    np.testing.assert_array_equal(_arr(cc.bond_types, 2 * cc.mb), _arr(py.bond_types, 2 * py.mb))
    np.testing.assert_allclose(_arr(cc.mu_ex_bulk, cc.nb), _arr(py.mu_ex_bulk, py.nb), rtol=1e-9, atol=1e-10)
    np.testing.assert_allclose(_arr(cc.lng_bulk, cc.mb), _arr(py.lng_bulk, py.mb), rtol=1e-9, atol=1e-10)
    for u in range(py.n_species):
        a, b = py.species[u], cc.species[u]
        n, S = a.n_seg, a.max_states
        assert (b.n_seg, b.max_states) == (n, S)
        for k, m in (("parent", n), ("n_states", n), ("states", n * S), ("fixed_coord", n)):
            np.testing.assert_array_equal(_arr(getattr(b, k), m), _arr(getattr(a, k), m), err_msg=f"{u}.{k}")
        assert b.fixed_density == a.fixed_density
        assert bool(b.max_distance) == bool(a.max_distance)
        if bool(a.max_distance):
            np.testing.assert_array_equal(_arr(b.max_distance, n * n), _arr(a.max_distance, n * n))
        assert b.mu_species == pytest.approx(a.mu_species, rel=1e-9, abs=1e-10)
    num_py = numerics_from_dict({str(k): yamlio.as_float(v) for k, v in (ds.get("numerical") or {}).items()})
    num_c = inp.numerics()
    for f, _ in num_py._fields_:
        assert getattr(num_c, f) == getattr(num_py, f), f
    it, res = inp.bulk_stats()
    assert it >= 1 and res < 1e-6
    inp.close()


def _dump(ds):
    return yaml.safe_dump(ds, sort_keys=False)


def _branched(seq):
    ds = workloads.weak_acid_slit(128, 0.05, 6, 4.5, 7.0, 0.1, 0.3)
    ds["species"][0]["sequence"] = seq
    return ds


CASES = {
    "ions_tpt1": YAML,
    "ions_plain_fmt_msa": YAML.replace("[ideal, TPT1mfmt, TPT1msa]", "[ideal, mfmt, msa]"),
    "weak_acid_20": _dump(workloads.plain_slit()),
    "diblock_200": _dump(workloads.diblock_slit(2048)),
    "brush_50": _dump(workloads.grafted_brush(2048, 0.02, 50, 0.05, 4.5, 7.0, 0.1)),
    "odd_grid_charged": _dump(workloads.weak_acid_slit(1001, 0.02, 20, 4.5, 6.0, 0.05, 0.25, wall_charge=-0.05)),
    "dense_300": _dump(workloads.weak_acid_slit(4096, 0.02, 300, 4.5, 3.0, 0.001, 0.4)),
    # a repeated species name: name lookups take its last entry, as the
    # reference's Dict does (assign_delta_muH.jl:67)
    "repeated_species": YAML.replace('  - sequence: "Y"\n    pSpecies: 6.0', '  - sequence: "Y"\n  - sequence: "Y"\n    pSpecies: 6.0'),
    "branched": _dump(_branched("AA(AA)AA")),
    "branched_repeat": _dump(_branched("A(AB)2A")),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_descriptor_matches_python_host(name):
    _compare(CASES[name])


def test_yaml_forms():
    """Comments, flow mappings, a block sequence at its key's indentation,
    quoted scalars, exponent floats and constraints give the same request."""
    text = """# a request written by hand
procedure: iDFT          # only iDFT is read
geometry: {coordinate_system: Cartesian, dimensions: [10.0], bin_width: [0.05],
  external_field: {hard_walls: {dims: [1]}}}
species:
- sequence: 'AAAA'
  concentration: 5e-2
- {sequence: "c", concentration: 0.02, adjustable: true}
- sequence: a
  concentration: 2.0e-2
  adjustable: yes
- sequence: Y
  pSpecies: 6.0
- sequence: Z
reactions:
  - species: [A, Y, B]
    coeffs: [-1, +1, +1]
    pK: 4.0
  - {species: [Y, Z], coeffs: [1, 1], pK: 14.0}
monomers:
  A: {diameter: 1.0, valence: 0.0}
  B: {diameter: 1.0, valence: -1.0}
  c: {diameter: 1.0, valence: 1.0}
  a: {diameter: 1.0, valence: -1.0}
  Y: {diameter: 1.0, valence: 1.0}
  Z: {diameter: 1.0, valence: -1.0}
constraints:
  temperature: 310.0
  dielectric_constant: 70.0
reduced_units: {l_sc: 0.4}
numerical:
  tole: 1e-7
  anderm: 4
model: [ideal, TPT1mfmt, TPT1msa]
"""
    _compare(text)


def test_repeated_keys_take_the_last_value():
    """YAML.jl and PyYAML keep the last value of a repeated key; so does the
    library's reader, in block and flow mappings alike."""
    text = YAML.replace("  tole: 1e-6\n", "  tole: 1e-6\n  tole: 1e-7\n")
    text = text.replace("A: {diameter: 1.0, valence: 0.0}", "A: {diameter: 0.9, valence: 0.0, diameter: 1.0}")
    text += "numerical: {damping: 0.01, tole: 1e-5, mixing_max: 0.001, tole: 1e-6, anderm: 4}\n"
    assert yamlio.load_text(text)["numerical"] == {"damping": 0.01, "tole": 1e-6, "mixing_max": 0.001, "anderm": 4}
    _compare(text)
    num = native.Input(text).numerics()
    assert (num.tole, num.anderm) == (1e-6, 4)


def test_plain_keys_may_hold_brackets_and_quotes():
    """In block context a plain scalar key may contain ], } and quotes; such a
    key is read as text (here an unknown monomer property, which both hosts
    ignore)."""
    text = YAML.replace("  a: {diameter: 1.0, valence: -1.0}",
                        "  a:\n    diameter: 1.0\n    valence: -1.0\n    note]s: 1\n    it's: 2\n    'x: y': 3")
    d = yamlio.load_text(text)["monomers"]["a"]
    assert d == {"diameter": 1.0, "valence": -1.0, "note]s": 1, "it's": 2, "x: y": 3}
    _compare(text)


def test_errors_carry_the_reference_messages():
    bad = YAML.split("species:")[0] + "model: [ideal]\n"
    with pytest.raises(native.SdftError) as e:
        native.Input(bad)
    assert "missing the required 'species' section" in str(e.value)
    # temperature must be a Float64 (get_temperature.jl:14-21)
    with pytest.raises(native.SdftError) as e:
        native.Input(YAML + "constraints:\n  temperature: 300\n")
    assert "must be a Float64 value" in str(e.value)
    with pytest.raises(native.SdftError) as e:
        native.Input(YAML.replace("[ideal, TPT1mfmt, TPT1msa]", "[ideal, vdw]"))
    assert e.value.code in (native.SDFT_ERR_UNSUPPORTED, 2)
    with pytest.raises(native.SdftError) as e:
        native.Input("geometry: [1, 2\n")
    assert e.value.code == 2


@pytest.mark.parametrize("text,why", [
    ("geometry:\n\tcoordinate_system: Cartesian\n", "tabs in indentation"),
    ("base: &b {x: 1}\nother: *b\n", "anchors"),
    ("note: |\n  text\n", "block scalars"),
    ("geometry: {coordinate_system: Cartesian\n", "flow"),
    ("geometry:\n  !external_field: 1\n", "cannot start with '!'"),
    ("monomers: {A: {%diameter: 1.0}}\n", "cannot start with '%'"),
    ("procedure: - iDFT\n", "sequence entry after a key"),
])
def test_yaml_subset_refuses_what_it_does_not_read(text, why):
    with pytest.raises(native.SdftError) as e:
        native.Input(text)
    assert e.value.code == 2 and why in str(e.value)


@pytest.mark.parametrize("dims,bw", [("[10.0]", "[0.0]"), ("[1.0e12]", "[1.0e-3]"), ("[-1.0]", "[0.05]")])
def test_slit_sizes_out_of_range_are_refused(dims, bw):
    text = YAML.replace("dimensions: [10.0]", "dimensions: " + dims).replace("bin_width: [0.05]", "bin_width: " + bw)
    assert text != YAML
    with pytest.raises(native.SdftError) as e:
        native.Input(text)
    assert e.value.code == 2


def _refused_by_both(text, why):
    with pytest.raises(Exception):
        setup_request(yamlio.load_text(text))
    with pytest.raises(native.SdftError) as e:
        native.Input(text)
    assert why in str(e.value), str(e.value)


@pytest.mark.parametrize("old,new,why", [
    ("    hard_walls:\n      dims: [1]", "    hard_walls:\n      dims:", "Missing 'dims' key"),
    ("  A: {diameter: 1.0, valence: 0.0}", "  A: 1.0", "must be a mapping"),
    ("  tole: 1e-6", "  tole: 1e-6\n  anderm: 2.5", "anderm must be an integer"),
    ("  tole: 1e-6", "  tole: 1e-6\n  anderm: 0", "anderm must be at least 1"),
    ("  tole: 1e-6", "  tole: 1e-6\n  max_iters: .nan", "max_iters must be an integer"),
])
def test_malformed_sections_are_refused_by_both_hosts(old, new, why):
    """Inputs on which the reference raises (a wall list that is null, a
    monomer whose properties are a number, a non-integral or empty Anderson
    depth: Int(x) and zeros(n, anderm) of AndersonMixing.jl) are refused by
    both hosts, not read as something else."""
    assert old in YAML
    _refused_by_both(YAML.replace(old, new), why)


def test_scalar_dims_and_extreme_numbers_read_as_the_reference_reads_them():
    """`for dim in 1` visits 1 in Julia, so `dims: 1` is the list [1]; a
    subnormal literal parses to a subnormal float (parse(Float64, ...))."""
    text = YAML.replace("    hard_walls:\n      dims: [1]", "    hard_walls:\n      dims: 1")
    text = text.replace("  tole: 1e-6", "  tole: 1e-6\n  mixed_switch: 1e-320")
    assert text != YAML
    _compare(text)
    assert native.Input(text).numerics().mixed_switch == 1e-320
