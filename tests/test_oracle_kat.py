"""Known-answer tests that pin the CPU oracle (the reference ships no golden
vectors and cannot run here, so these physics identities are the anchor):

* bulk fixed point: in a wall-free box the mirrored grid is an infinite
  homogeneous fluid, so G(x0) at the bulk state x0 (process_guess.jl:5-54) must
  return x0 (FMT/TPT1 weights, propagators and the bulk iLST formulas agree);
* ideal-chain limit: without excess functionals every segment density equals
  the bulk segment density;
* ideal dissociation: the B-state fraction is 1/(1 + 10^(pKa - pH));
* the k-space weights carry the analytic integrals at k = 0 (n3 of a uniform
  density is rho*pi*sigma^3/6);
* contact-value theorem: at a hard wall the contact density of a hard-sphere
  fluid equals its bulk pressure (contact_value_theorem.jl:5-20 against
  eval_pressure.jl:10-25), up to a discretisation error of order dz^2;
* segment-resolved bulk state: in a wall-free box at the bulk state every
  segment's state densities (chain ends and ionisation split included) equal
  the bulk iLST segment densities at every grid point, and the species counts
  (num_species.jl:1-38) are rho_u times the box volume;
* grand potential: in a wall-free box at the bulk state, Omega
  (grand_potential.jl:4-28) is -P_bulk times the box volume NP*dz, P_bulk from
  the independent bulk formula (eval_pressure.jl:10-25);
* electroneutrality: in a converged slit with charged walls the fluid's
  trapezoid-weighted charge cancels the wall charge (the PsiC Newton step of
  neutrality_shift.jl balances them).
"""
import math

import numpy as np
import pytest

from oracle.oracle import OracleSystem
from softdft_b200 import workloads
from softdft_b200.host.descriptor import numerics_from_dict
from softdft_b200.output import contact_value_theorem_arrays
from tests.helpers import descriptor, rel, small_slit


def test_bulk_fixed_point_fmt():
    ds = small_slit(models=["ideal", "TPT1mfmt"], walls=False)
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    x0 = o.get_x()
    g = o.objective()
    mu0, lng0, psi0, psic0 = dft.split(x0)
    mu, lng, psi, psic = dft.split(g)
    assert rel(mu, mu0) < 1e-9
    assert rel(lng, lng0) < 1e-9
    assert np.max(np.abs(psi)) < 1e-9
    assert abs(psic[0]) < 1e-8


@pytest.mark.parametrize("np_", [125, 1001])
def test_bulk_fixed_point_on_odd_grids(np_):
    """Odd NP gives a mirrored grid of 2 NP = 2 mod 4 points (250, 2002), which
    the oracle transforms with Bluestein's algorithm."""
    ds = small_slit(models=["ideal", "TPT1mfmt", "TPT1msa"], walls=False, np_=np_, dz=0.05)
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    x0 = o.get_x()
    g = o.objective()
    mu0, lng0, _, _ = dft.split(x0)
    mu, lng, psi, _ = dft.split(g)
    assert rel(mu, mu0) < 1e-8
    assert rel(lng, lng0) < 1e-8
    assert np.max(np.abs(psi)) < 1e-9


def test_bulk_fixed_point_fmt_msa():
    ds = small_slit(models=["ideal", "TPT1mfmt", "TPT1msa"], walls=False)
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    x0 = o.get_x()
    g = o.objective()
    mu0, lng0, _, _ = dft.split(x0)
    mu, lng, psi, _ = dft.split(g)
    assert rel(mu, mu0) < 1e-8
    assert rel(lng, lng0) < 1e-8
    assert np.max(np.abs(psi)) < 1e-9


def test_ideal_chain_limit():
    ds = small_slit(models=["ideal"], walls=False, n_chain=8)
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    o.objective()
    segs, beads, _ = o.densities()
    bulk = dft.bulk_system.bulk
    d = dft.descriptor
    for u in range(d.n_species):
        s = segs[u].reshape((d.n_seg[u], d.max_states[u], d.np_))
        ref = bulk.rho_segments[u]  # (S, N)
        for g in range(d.n_seg[u]):
            for i in range(d.max_states[u]):
                assert np.allclose(s[g, i], ref[i, g], rtol=1e-12, atol=1e-300)
    assert rel(beads.reshape(d.nb, d.np_)[:, d.np_ // 2], bulk.rho_beads) < 1e-12


@pytest.mark.parametrize("pH", [3.0, 4.5, 7.0])
def test_ideal_dissociation_fraction(pH):
    ds = small_slit(models=["ideal"], walls=False, pH=pH, n_chain=5)
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    o.objective()
    segs, _, _ = o.densities()
    d = dft.descriptor
    s = segs[0].reshape((d.n_seg[0], d.max_states[0], d.np_))
    alpha = s[:, 1, :].sum() / s.sum()
    assert abs(alpha - 1.0 / (1.0 + 10 ** (4.5 - pH))) < 1e-12


def test_packing_fraction_weight_at_k0():
    ds = small_slit(models=["ideal", "TPT1mfmt"], walls=False)
    dft = descriptor(ds)
    bulk = dft.bulk_system.bulk
    sig = np.asarray(dft.bulk_system.molsys.diameters)
    eta = float(np.sum(bulk.rho_beads * math.pi * sig ** 3 / 6))
    # the oracle's FMT n3 weight at k=0 is 4/3 pi (sigma/2)^3; a uniform field
    # reproduces the bulk packing fraction through the excess chemical potential
    o = OracleSystem(dft.descriptor)
    g = o.objective()
    mu, _, _, _ = dft.split(g)
    assert 0.25 < eta < 0.45
    assert rel(mu[dft.NP // 2], bulk.mu_ex) < 1e-9


def test_walls_zero_density_inside():
    ds = small_slit()
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    o.objective()
    _, beads, _ = o.densities()
    d = dft.descriptor
    b = beads.reshape(d.nb, d.np_)
    ext, tr = o.fields()
    ext = ext.reshape(d.nb, d.np_)
    assert np.all(b[ext > 1e19] == 0.0)
    # contact points carry trapezoid weight 1/2
    assert np.count_nonzero(tr.reshape(d.nb, d.np_)[0] == 0.5) == 2


def test_bulk_fixed_point_long_chain_renormalised():
    """150-segment chain in a dense fluid: the reference's unscaled propagator
    products leave the double range here; the renormalised path must still
    return the bulk state in a wall-free box."""
    ds = small_slit(models=["ideal", "TPT1mfmt"], walls=False, n_chain=150, np_=256)
    dft = descriptor(ds)
    bulk = dft.bulk_system.bulk
    # unscaled propagator products ~ exp(-(N-1)(mu_ex - lng)) fall below the double range
    assert 149 * (bulk.mu_ex[0] - bulk.lng[0]) > 745
    o = OracleSystem(dft.descriptor)
    x0 = o.get_x()
    g = o.objective()
    assert np.all(np.isfinite(g))
    mu0, lng0, _, _ = dft.split(x0)
    mu, lng, psi, _ = dft.split(g)
    assert rel(mu, mu0) < 1e-8
    assert rel(lng, lng0) < 1e-8
    segs, beads, _ = o.densities()
    d = dft.descriptor
    assert rel(beads.reshape(d.nb, d.np_)[:, d.np_ // 2], dft.bulk_system.bulk.rho_beads) < 1e-8


def _hard_sphere_slit(np_, dz, eta):
    return {"procedure": "iDFT",
            "geometry": {"coordinate_system": "Cartesian", "dimensions": [(np_ - 1) * dz], "bin_width": [dz],
                         "external_field": {"hard_walls": {"dims": [1]}}},
            "species": [{"sequence": "S", "density": eta * 6.0 / math.pi}],
            "monomers": {"S": {"diameter": 1.0, "valence": 0.0}},
            "numerical": {"tole": 1e-10, "damping": 0.1, "mixing_max": 0.5, "anderm": 5},
            "model": ["ideal", "mfmt"]}


def test_contact_value_theorem_hard_spheres():
    """A 10-sigma slit of hard spheres at packing fraction 0.2: the contact
    density at each wall equals the bulk pressure to 2e-4 at dz = 0.02, and
    the error falls fourfold with each halving of dz."""
    errors = []
    for np_, dz in ((512, 0.02), (1023, 0.01), (2047, 0.005)):
        ds = _hard_sphere_slit(np_, dz, 0.2)
        dft = descriptor(ds)
        o = OracleSystem(dft.descriptor)
        it, err, _, _ = o.solve(numerics_from_dict(ds["numerical"]))
        assert err < 1e-10, (np_, it, err)
        _, beads, _ = o.densities()
        P = dft.descriptor.desc.np
        cvt = contact_value_theorem_arrays(beads.reshape(-1, P).T, dft.bulk_system.molsys, dft.geometry)
        p_bulk = dft.bulk_system.bulk.pressure
        errors.append(np.abs(cvt - p_bulk) / p_bulk)
    errors = np.array(errors)
    assert np.all(errors[0] < 2e-4)
    ratios = errors[:-1] / errors[1:]
    assert np.all((ratios > 3.5) & (ratios < 4.5)), ratios


def test_charged_slit_is_neutral():
    """A weak-acid slit between walls of charge -0.05 each, solved to 1e-8: the
    fluid carries +0.1 to within 1e-7 relative."""
    ds = small_slit(np_=128, dz=0.05, wall_charge=-0.05)
    ds["numerical"]["max_iters"] = 20000
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    it, err, _, _ = o.solve(numerics_from_dict(ds["numerical"]))
    assert err < 1e-8, (it, err)
    _, beads, _ = o.densities()
    _, trapez = o.fields()
    P = dft.descriptor.desc.np
    z = np.asarray(dft.bulk_system.molsys.valences)
    q_fluid = float((beads.reshape(-1, P).T * trapez.reshape(-1, P).T * z[None, :]).sum() * dft.geometry.bin_width)
    q_walls = -0.05 - 0.05
    assert abs(q_fluid + q_walls) < 1e-7 * abs(q_walls), q_fluid


@pytest.mark.parametrize("models", [["ideal"], ["ideal", "mfmt", "msa"], ["ideal", "TPT1mfmt", "TPT1msa"]])
def test_bulk_grand_potential_is_minus_pressure_volume(models):
    ds = small_slit(models=models, walls=False)
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    o.objective()
    volume = dft.descriptor.desc.np * dft.geometry.bin_width
    p_bulk = dft.bulk_system.bulk.pressure
    assert abs(o.grand_potential() + p_bulk * volume) < 1e-12 * p_bulk * volume


def _bulk_box(name):
    if name == "weak_acid":
        return small_slit(models=["ideal", "TPT1mfmt", "TPT1msa"], walls=False)
    if name == "diblock_200":
        ds = workloads.diblock_slit(256)
        ds["geometry"]["external_field"] = {}
        return ds
    ds = small_slit(models=["ideal"], walls=False)
    ds["species"][0]["sequence"] = "AA(AA)AA"
    return ds


# tolerance: a 200-segment chain multiplies 200 convolved propagators
@pytest.mark.parametrize("name,tol", [("weak_acid", 1e-13), ("diblock_200", 1e-9), ("branched_ideal", 1e-13)])
def test_bulk_segment_states_and_species_counts(name, tol):
    dft = descriptor(_bulk_box(name))
    o = OracleSystem(dft.descriptor)
    o.objective()
    d = dft.descriptor.desc
    bulk = dft.bulk_system.bulk
    volume = d.np * dft.geometry.bin_width
    assert rel(o.num_species(), np.asarray(bulk.rho_species) * volume) < tol
    segs, _, _ = o.densities()
    for u in range(d.n_species):
        S, N = d.species[u].max_states, d.species[u].n_seg
        profile = segs[u].reshape(N, S, d.np).transpose(1, 0, 2)  # (state, segment, K)
        expected = np.asarray(bulk.rho_segments[u])[:, :, None]     # (state, segment)
        assert np.max(np.abs(profile - expected)) < tol * np.max(np.abs(expected)), u