"""Native bulk evaluation (sdft_bulk_eval) against the numpy restatement.

The native call evaluates eval_bulk_density followed by
bulk_chemical_potential (src/iLST/evaluation/objective/residual_bulkstate.jl:26-35)
with the operations in the numpy code's order.  numpy's vectorised exp and the
C library's exp may differ by an ulp, and a chain's partition function is a
product of one such factor per segment, so the tolerance is 64 eps N for the
longest chain of N segments (1e-13 at least).
"""
import copy
import math
import zlib

import numpy as np
import pytest

from softdft_b200 import native, workloads
from softdft_b200.host import ilst, molsys, yamlio

from test_host_setup import YAML

pytestmark = pytest.mark.skipif(not native.library_present(), reason="libsoftdft.so not built")

FIELDS = ["rho_beads", "rho_bonds", "mu_species", "mu_ex", "lng", "Xi"]


def _systems():
    return {
        "ions_tpt1": yamlio.load_text(YAML),
        "ions_plain_fmt_msa": yamlio.load_text(YAML.replace("[ideal, TPT1mfmt, TPT1msa]", "[ideal, mfmt, msa]")),
        "ideal_only": yamlio.load_text(YAML.replace("[ideal, TPT1mfmt, TPT1msa]", "[ideal]")),
        "weak_acid_20": workloads.plain_slit(),
        "diblock_200": workloads.diblock_slit(2048),
        "brush_50": workloads.grafted_brush(2048, 0.02, 50, 0.05, 4.5, 7.0, 0.1),
        "dense_300": workloads.weak_acid_slit(4096, 0.02, 300, 4.5, 3.0, 0.001, 0.4),
    }


def _evaluate_both(ms, bulk):
    a, b = copy.deepcopy(bulk), copy.deepcopy(bulk)
    ilst.eval_bulk_density(ms, a)
    ilst.bulk_chemical_potential(ms, a)
    ilst.eval_bulk_state_native(ms, b)
    return a, b


def _rtol(ms):
    n = max(len(c.sequence) for c in ms.configurations)
    return max(1e-13, 64 * np.finfo(np.float64).eps * n)


def _assert_same(a, b, rtol):
    for name in FIELDS:
        x, y = np.asarray(getattr(a, name)), np.asarray(getattr(b, name))
        assert x.shape == y.shape, name
        np.testing.assert_allclose(y, x, rtol=rtol, atol=0, err_msg=name)
    for u, (x, y) in enumerate(zip(a.rho_segments, b.rho_segments)):
        np.testing.assert_allclose(y, x, rtol=rtol, atol=0, err_msg=f"rho_segments[{u}]")


@pytest.mark.parametrize("name", list(_systems()))
@pytest.mark.parametrize("shift", [0.0, 0.7, 6.0])
def test_native_matches_numpy(name, shift):
    ms = molsys.molecular_system(_systems()[name])
    bulk = ilst.initialize_densities(ms)
    rng = np.random.default_rng(zlib.crc32(f"{name}:{shift}".encode()))
    bulk.mu_ex[:] += shift + rng.normal(0.0, 0.3, bulk.mu_ex.shape)
    bulk.lng[:] += rng.normal(0.0, 0.3, bulk.lng.shape)
    a, b = _evaluate_both(ms, bulk)
    _assert_same(a, b, _rtol(ms))
    assert np.all(np.isfinite(b.mu_ex))


def test_log_domain_path_is_taken_and_matches():
    """A 300-segment chain at mu_ex + 6 underflows the linear propagators
    (child_propagators.jl:41-50 multiplies e^-6 per segment), so both
    evaluations switch to log-domain propagators."""
    ms = molsys.molecular_system(_systems()["dense_300"])
    bulk = ilst.initialize_densities(ms)
    bulk.mu_ex[:] += 6.0
    chain = next(u for u, c in enumerate(ms.configurations) if len(c.sequence) == 300)
    with np.errstate(all="ignore"):
        gC, gP, Xi = ilst._fj_propagators(ms, bulk, chain)
    assert not (np.isfinite(Xi) and Xi > 0 and np.all(np.isfinite(gC)) and np.all(np.isfinite(gP)))
    a, b = _evaluate_both(ms, bulk)
    _assert_same(a, b, _rtol(ms))
    assert b.rho_segments[chain].sum() > 0


def test_monomer_species_only():
    y = YAML.split("species:")[0] + """species:
  - sequence: "c"
    concentration: 0.1
  - sequence: "a"
    concentration: 0.1
monomers:
  c: {diameter: 1.0, valence: 1.0}
  a: {diameter: 0.8, valence: -1.0}
numerical:
  tole: 1e-8
model: [ideal, mfmt, msa]
"""
    ms = molsys.molecular_system(yamlio.load_text(y))
    bulk = ilst.initialize_densities(ms)
    bulk.mu_ex[:] += 0.2
    a, b = _evaluate_both(ms, bulk)
    _assert_same(a, b, _rtol(ms))


def test_bulk_solve_identical_with_native_residual(monkeypatch):
    """The whole bulk solve (AndersonResidual around residual_bulkstate) reaches
    the same state with either evaluation, to well inside its tolerance."""
    ds = workloads.plain_slit()
    ms1 = molsys.molecular_system(ds)
    native_state = ilst.solve_bulk(ms1, ds["numerical"])
    monkeypatch.setattr(ilst, "_use_native", lambda: False)
    ms2 = molsys.molecular_system(ds)
    numpy_state = ilst.solve_bulk(ms2, ds["numerical"])
    assert abs(native_state.iterations - numpy_state.iterations) <= 2
    _assert_same(numpy_state, native_state, 1e-9)
    assert math.isfinite(native_state.residual)
