"""Result files in the reference's text formats (host only, synthetic arrays)."""
import math
import os

import numpy as np

from softdft_b200 import output, workloads
from softdft_b200.api import geometry_system
from softdft_b200.host import molsys as molsys_mod


def test_julia_float_printing():
    cases = {0.1: "0.1", 1.0: "1.0", 100000.0: "100000.0", 1e6: "1.0e6", 1234567.8: "1.2345678e6",
             0.0001: "0.0001", 1e-5: "1.0e-5", 2.5e-7: "2.5e-7", -3.25: "-3.25", 0.0: "0.0",
             123456.7: "123456.7", 1e20: "1.0e20", 1.4297414291151598: "1.4297414291151598"}
    for v, s in cases.items():
        assert output.jl(v) == s, (v, output.jl(v), s)
    assert output.jl(-0.0) == "-0.0" and output.jl(float("nan")) == "NaN" and output.jl(7) == "7"
    for v in np.random.default_rng(1).standard_normal(200) * 10.0 ** np.random.default_rng(2).integers(-12, 12, 200):
        assert float(output.jl(v).replace("e", "e")) == v  # round-trips


def _system():
    ds = workloads.weak_acid_slit(64, 0.1, 4, 4.5, 7.0, 0.1, 0.3)
    return ds, molsys_mod.molecular_system(ds), geometry_system(ds)


def test_field_and_segment_writers(tmp_path):
    ds, ms, geom = _system()
    P = geom.NP
    beads = np.arange(P * len(ms.monomers), dtype=float).reshape(P, len(ms.monomers)) / 8.0
    output.write_field_array(beads, str(tmp_path / "rho_beads_K.txt"), names=list(ms.monomers))
    lines = open(tmp_path / "rho_beads_K.txt").read().splitlines()
    assert lines[0] == "Index_1  " + " ".join(ms.monomers)
    assert lines[1] == "1  " + " ".join(output.jl(v) for v in beads[0])
    assert len(lines) == P + 1
    segs = []
    for cfg in ms.configurations:
        S = max(len(f) for f in cfg.state_family)
        segs.append(np.random.default_rng(0).uniform(0.1, 1.0, size=(P, S, len(cfg.sequence))))
    output.write_segment_array(segs, ms, str(tmp_path))
    output.write_state_fraction_profiles(segs, ms, str(tmp_path))
    output.write_total_state_fractions(segs, ms, str(tmp_path))
    chain = [u for u, c in enumerate(ms.configurations) if len(c.sequence) > 1][0]
    name = ms.species[chain]
    fam = ms.configurations[chain].state_family
    hdr = open(tmp_path / f"rho_segments_{name}.txt").readline().split()
    assert hdr[0] == "Index_1" and hdr[1] == f"seg1_{ms.monomers[fam[0][0]]}" and len(hdr) == 1 + sum(map(len, fam))
    row = open(tmp_path / f"state_fraction_{name}.txt").read().splitlines()[1].split()
    vals = [float(v) for v in row[1:]]
    assert math.isclose(vals[0] + vals[1], 1.0, rel_tol=1e-15)
    tot = open(tmp_path / f"total_state_fractions_{name}.txt").read().splitlines()
    assert tot[0] == "segment state1 state2"
    assert tot[-2] == "# Average state fractions across all dissociating segments:" and tot[-3] == ""
    avg = [float(v) for v in tot[-1].split()[1:]]
    rho = segs[chain]
    a = np.array([rho[:, :, g].sum(axis=0) / rho[:, :, g].sum() for g in range(rho.shape[2])]).mean(axis=0)
    assert np.allclose(avg, a, rtol=1e-13)


def test_contact_value_theorem_and_brush_height(tmp_path):
    ds, ms, geom = _system()
    P = geom.NP
    beads = np.ones((P, len(ms.monomers)))
    c = output.contact_value_theorem_arrays(beads, ms, geom)
    assert np.allclose(c, [len(ms.monomers), len(ms.monomers)])
    output.write_cvt(c, str(tmp_path / "cvt.txt"))
    assert open(tmp_path / "cvt.txt").read().splitlines()[1] == f"dim1  {output.jl(c[0])}  {output.jl(c[1])}"
    # charged walls add -2 pi lB q^2 per wall
    geom.charged_walls = [0.0, geom.dimensions]
    geom.wall_charges = [-0.1, -0.2]
    c2 = output.contact_value_theorem_arrays(beads, ms, geom)
    lB = ms.bjerrum_length
    assert np.allclose(c2 - c, [-2 * math.pi * lB * 0.01, -2 * math.pi * lB * 0.04])
    # brush height of a uniform free profile with one fixed segment at the left wall
    segs = [np.zeros((P, max(len(f) for f in cfg.state_family), len(cfg.sequence))) for cfg in ms.configurations]
    chain = [u for u, cfg in enumerate(ms.configurations) if len(cfg.sequence) > 1][0]
    segs[chain][:, 0, :] = 1.0
    fixed = [np.full(len(cfg.sequence), -1) for cfg in ms.configurations]
    assert output.brush_height_values(segs, ms, geom, fixed) == {}
    fixed[chain][0] = 0
    h = output.brush_height_values(segs, ms, geom, fixed)[ms.species[chain]]
    assert 0.0 < h < 2.0 * geom.dimensions
