"""Device solve vs the CPU oracle, through the C ABI (libsoftdft.so).

Tolerances (FP64 plain form):
* one G(x) evaluation: 1e-11 relative to max|G| (the device convolves in DCT
  space, the oracle with complex FFTs of the mirrored grid, as the reference);
* densities of the evaluation: 1e-12;
* converged states at tole 1e-10: 1e-7 relative on densities, 1e-8 on Omega.
  Trajectories cannot be compared step by step: the first Anderson steps
  solve near-collinear least-squares problems and the Picard phase amplifies
  1e-16 differences, so iteration counts are reported, not matched.
"""
import copy

import numpy as np
import pytest

from oracle.oracle import OracleSystem
from softdft_b200 import native
from softdft_b200.host.descriptor import numerics_from_dict
from tests.helpers import descriptor, rel, small_slit
from softdft_b200 import workloads

pytestmark = pytest.mark.gpu

CASES = {
    "acid_salt": small_slit(),
    "charged_walls": small_slit(wall_charge=-0.05),
    "mfmt_msa": small_slit(models=["ideal", "mfmt", "msa"]),
    "no_walls": small_slit(walls=False),
    "low_pH": small_slit(pH=3.0, salt=0.01),
    "brush": workloads.grafted_brush(256, 0.05, 10, 0.05, 4.5, 7.0, 0.01),
    "diblock_small": None,
}


def _diblock_small():
    ds = workloads.diblock_slit(512)
    ds["species"][0]["sequence"] = "A" * 6 + "C" * 6
    return ds


CASES["diblock_small"] = _diblock_small()
# the benchmarked request: NP = 1024, 20-segment weak polyacid, TPT1 FMT + MSA
CASES["plain_slit"] = workloads.plain_slit()
# 200-segment diblock in a 10-sigma slit: renormalised propagators
CASES["long_diblock"] = workloads.diblock_slit(1024)
# grid sizes that exercise every FFT pass mix (log2 M = 10, 11, 12, 13: radix-8
# passes with a radix-2 / radix-4 / no tail) and 4, 2, 1 transform buffers
CASES["grid_2048_mfmt_msa"] = small_slit(np_=2048, dz=0.01, models=["ideal", "mfmt", "msa"])
CASES["grid_4096"] = small_slit(np_=4096, dz=0.005)
CASES["grid_8192"] = small_slit(np_=8192, dz=0.02)
CASES["grid_16384"] = small_slit(np_=16384, dz=0.02)
# the 200-segment diblock on the 16384-point grid (one transform buffer)
CASES["diblock_16384"] = workloads.diblock_slit(16384)
# grids that are not powers of two: mixed-radix transforms of M = NP/2 points
# (radices in brackets; 11 and 13 run the run-time-radix butterfly, odd M has
# no middle coefficient pair)
CASES["grid_1000"] = small_slit(np_=1000, dz=0.02)                 # M = 500  [4 5 5 5]
CASES["grid_250_odd_m"] = small_slit(np_=250, dz=0.05)             # M = 125  [5 5 5]
CASES["grid_286_radix_11_13"] = small_slit(np_=286, dz=0.05)       # M = 143  [11 13]
CASES["grid_770_mfmt_msa"] = small_slit(np_=770, dz=0.02, models=["ideal", "mfmt", "msa"])  # M = 385 [5 7 11]
CASES["grid_1458"] = small_slit(np_=1458, dz=0.01)                 # M = 729  [3 3 3 3 3 3]
CASES["grid_6000"] = small_slit(np_=6000, dz=0.005)                # M = 3000 [4 2 3 5 5 5]
CASES["brush_600"] = workloads.grafted_brush(600, 0.05, 10, 0.05, 4.5, 7.0, 0.01)  # M = 300 [4 3 5 5]
# odd grids: a complex FFT of M = NP points on real data, device arrays padded
# to the stride NP + 1 (H = 20 sigma at dz = 0.02 gives the reference NP = 1001)
CASES["grid_1001"] = small_slit(np_=1001, dz=0.02)                 # M = 1001 [7 11 13]
CASES["grid_125_mfmt_msa"] = small_slit(np_=125, dz=0.05, models=["ideal", "mfmt", "msa"])  # M = 125 [5 5 5]
CASES["charged_walls_1001"] = small_slit(np_=1001, dz=0.02, wall_charge=-0.05)
CASES["brush_999"] = workloads.grafted_brush(999, 0.05, 10, 0.05, 4.5, 7.0, 0.01)  # M = 999 [3 3 3 37]


def _diblock_odd():
    ds = workloads.diblock_slit(1001)
    ds["species"][0]["sequence"] = "A" * 6 + "C" * 6
    return ds


CASES["diblock_1001"] = _diblock_odd()
# lengths with a prime factor above 61: Bluestein's chirp convolution
CASES["grid_1009_bluestein"] = small_slit(np_=1009, dz=0.02)        # M = 1009 (prime), 2048-point convolution
CASES["grid_1002_bluestein"] = small_slit(np_=1002, dz=0.02)        # M = 501 = 3 * 167, 1024 points
CASES["grid_2026_bluestein_mfmt_msa"] = small_slit(np_=2026, dz=0.01, models=["ideal", "mfmt", "msa"])  # M = 1013
# the edges of the device's range: the longest Bluestein length (M = 4093, prime,
# an 8192-point convolution), the longest odd mixed-radix length (M = 12285 =
# 3^3 5 7 13) and the longest even one that fits one CTA's shared memory
# (M = 12288 = 2^12 3, one transform buffer of 221 KB)
CASES["grid_8186_bluestein"] = small_slit(np_=8186, dz=0.005)
CASES["grid_12285_odd"] = small_slit(np_=12285, dz=0.005)
CASES["grid_24576"] = small_slit(np_=24576, dz=0.002)
# G(x) bound per case: 1e-11, except where the oracle's own transform is the
# looser one -- at 24576 points its mirrored 49152-point FFT is not a power of
# two and runs through its Bluestein convolution of 131072 points (measured
# 1.1e-11 against the device)
G_TOL = {"grid_24576": 2e-11}


# branched chains (parse_topology.jl syntax: a parenthesised run is a side branch)
def _branched(seq, **kw):
    ds = small_slit(**kw)
    ds["species"][0]["sequence"] = seq
    return ds


def _branched_brush():
    ds = workloads.grafted_brush(256, 0.05, 6, 0.05, 4.5, 7.0, 0.01)
    ds["species"][0]["sequence"] = ds["species"][1]["sequence"] = "AA(AA)AA"
    return ds


CASES["branched_acid"] = _branched("AA(AA)AA")
CASES["branched_two_points"] = _branched("AAA(A)AAA(AA)A")
CASES["branched_brush"] = _branched_brush()
CASES["branched_1001"] = _branched("AA(AA)AA", np_=1001, dz=0.02)
# the branched slit converges under the reference's Anderson driver at a smaller mixing
CASES["branched_acid_mix5e-4"] = _branched("AA(AA)AA")
CASES["branched_acid_mix5e-4"]["numerical"]["mixing_max"] = 5e-4


@pytest.mark.parametrize("name", sorted(CASES))
def test_objective_matches_oracle(name):
    dft = descriptor(CASES[name])
    o = OracleSystem(dft.descriptor)
    g = native.DeviceSystem(dft.descriptor)
    assert rel(g.get_x(), o.get_x()) == 0.0
    go, gg = o.objective(), g.objective()
    assert rel(gg, go) < G_TOL.get(name, 1e-11)
    so, bo, bno = o.densities()
    sg, bg, bng = g.densities()
    assert rel(bg, bo) < 1e-12
    if bno.size:
        assert rel(bng, bno) < 1e-12
    for a, b in zip(sg, so):
        assert rel(a, b) < 1e-12


def test_objective_at_perturbed_state():
    dft = descriptor(CASES["acid_salt"])
    o = OracleSystem(dft.descriptor)
    g = native.DeviceSystem(dft.descriptor)
    rng = np.random.default_rng(7)
    x = o.get_x() + 1e-2 * rng.standard_normal(o.n)
    o.set_x(x)
    g.set_x(x)
    assert rel(g.objective(), o.objective()) < 1e-11


def test_picard_trajectory_matches():
    ds = copy.deepcopy(CASES["acid_salt"])
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    g = native.DeviceSystem(dft.descriptor)
    num = numerics_from_dict(dict(ds["numerical"], max_iters=30, switch_tole=1e-30))
    _, eo, _, _ = o.solve(num)
    _, eg, _ = g.solve(num)
    assert rel(g.get_x(), o.get_x()) < 1e-12
    assert abs(eg - eo) / eo < 1e-10


@pytest.mark.parametrize("name", ["acid_salt", "brush", "grid_1000", "brush_600", "grid_1001", "brush_999",
                                  "branched_acid_mix5e-4", "branched_brush", "grid_1009_bluestein"])
def test_converged_state_matches(name):
    ds = copy.deepcopy(CASES[name])
    ds["numerical"]["tole"] = 1e-10
    ds["numerical"]["max_iters"] = 5000
    dft = descriptor(ds)
    o = OracleSystem(dft.descriptor)
    g = native.DeviceSystem(dft.descriptor)
    num = numerics_from_dict(ds["numerical"])
    it_o, err_o, rc_o, _ = o.solve(num)
    it_g, err_g, rc_g = g.solve(num)
    assert rc_o == 0 and rc_g == 0, (it_o, err_o, it_g, err_g)
    assert err_g < 1e-10
    _, bo, _ = o.densities()
    _, bg, _ = g.densities()
    assert rel(bg, bo) < 1e-7
    om_o, om_g = o.grand_potential(), g.grand_potential()
    assert abs(om_g - om_o) / abs(om_o) < 1e-8
    assert rel(g.num_species(), o.num_species()) < 1e-7


def test_batch_equals_single():
    ds = copy.deepcopy(CASES["acid_salt"])
    num = numerics_from_dict(dict(ds["numerical"], max_iters=60))
    systems = []
    for pH in (5.0, 7.0, 9.0):
        d2 = copy.deepcopy(ds)
        d2["species"][4]["pSpecies"] = pH
        systems.append(descriptor(d2))
    singles = []
    for dft in systems:
        s = native.DeviceSystem(dft.descriptor)
        s.solve(num)
        singles.append(s.get_x())
    batch = [native.DeviceSystem(dft.descriptor) for dft in systems]
    iters, errs, status = native.solve_batch(batch, num)
    for b, x in zip(batch, singles):
        assert rel(b.get_x(), x) == 0.0


def test_max_iters_status_and_nonfinite():
    ds = copy.deepcopy(CASES["acid_salt"])
    dft = descriptor(ds)
    g = native.DeviceSystem(dft.descriptor)
    num = numerics_from_dict(dict(ds["numerical"], max_iters=3))
    it, err, rc = g.solve(num)
    assert it == 3 and rc == native.SDFT_MAX_ITERS
    x = g.get_x()
    x[5] = np.nan
    g.set_x(x)
    with pytest.raises(native.SdftError) as e:
        g.solve(num)
    assert e.value.code == 7


def test_batch_mixes_grid_kinds():
    """One batch over power-of-two and general-length requests (one launch of
    each kernel build) gives each request the state of its own single solve."""
    num = numerics_from_dict(dict(CASES["acid_salt"]["numerical"], max_iters=40))
    dss = [CASES["acid_salt"], CASES["grid_250_odd_m"], CASES["grid_1000"], CASES["grid_286_radix_11_13"],
           CASES["grid_1001"]]
    singles = []
    for ds in dss:
        s = native.DeviceSystem(descriptor(ds).descriptor)
        s.solve(num)
        singles.append(s.get_x())
    batch = [native.DeviceSystem(descriptor(ds).descriptor) for ds in dss]
    native.solve_batch(batch, num)
    for b, x in zip(batch, singles):
        assert rel(b.get_x(), x) == 0.0


@pytest.mark.parametrize("np_,why", [(4099, "Bluestein transform of 16384 points"),
                                     (8198, "Bluestein transform of 16384 points")])
def test_unsupported_grids_are_refused(np_, why):
    dft = descriptor(small_slit(np_=np_, dz=0.02))
    with pytest.raises(native.SdftError) as e:
        native.DeviceSystem(dft.descriptor)
    assert e.value.code == native.SDFT_ERR_UNSUPPORTED
    assert why in str(e.value)


def test_branched_topology_beyond_the_reference_arrays_is_refused():
    """A branch point with more children than states: the reference's
    other-children index (parent_propagators.jl:150) leaves its array."""
    dft = descriptor(_branched("A(AA)(AA)A"))
    with pytest.raises(native.SdftError) as e:
        native.DeviceSystem(dft.descriptor)
    assert e.value.code == native.SDFT_ERR_UNSUPPORTED and "index out of range" in str(e.value)
