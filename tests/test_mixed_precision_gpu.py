"""Mixed precision (SDFT_PREC_MIXED): FP32 chain convolutions, and on even
grids FP32 propagator storage, while the residual is above the switch in the
Anderson phase; FP64 for everything else, for the Picard phase and for the
final iterations.  One mixed G(x) stays within 1e-5 (max-norm, relative to
max|G|) of the FP64 one; a mixed solve converges to the FP64 fixed point, so
its densities and grand potential match the FP64 oracle's converged state to
1e-7 and 1e-8 (the served mixed form is asked for 1e-6 and 1e-8).

The Picard phase stays in FP64: the reference's Anderson driver starts from a
history of tiny Picard steps (mixing 0.002) whose first least-squares problem
amplifies 1e-7-level noise, and the small acid slit diverged at its first
Anderson step when those steps were FP32."""
import copy

import numpy as np
import pytest

from oracle.oracle import OracleSystem
from softdft_b200 import native, workloads
from softdft_b200.host.descriptor import numerics_from_dict
from tests.helpers import descriptor, rel, small_slit

pytestmark = pytest.mark.gpu

MIXED = 1

CASES = {
    "acid_salt": small_slit(),
    "brush": workloads.grafted_brush(256, 0.05, 10, 0.05, 4.5, 7.0, 0.01),
    "long_diblock": workloads.diblock_slit(1024),
    "plain_slit": workloads.plain_slit(),
    # FP32 mixed-radix transforms: an even grid (M = 500) and an odd one (M = 1001, complex FFT of real data)
    "grid_1000": small_slit(np_=1000, dz=0.02),
    "grid_1001": small_slit(np_=1001, dz=0.02),
    "brush_999": workloads.grafted_brush(999, 0.05, 10, 0.05, 4.5, 7.0, 0.01),
    # FP32 Bluestein transforms (M = 1009, prime)
    "grid_1009_bluestein": small_slit(np_=1009, dz=0.02),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_objective_close_to_fp64(name):
    dft = descriptor(CASES[name])
    g64 = native.DeviceSystem(dft.descriptor)
    g32 = native.DeviceSystem(dft.descriptor, precision=MIXED)
    a, b = g64.objective(), g32.objective()
    d = rel(b, a)
    print(f"{name}: mixed G(x) max-norm deviation {d:.3e}")
    assert np.all(np.isfinite(b)) and d < 1e-5


@pytest.mark.parametrize("name", ["acid_salt", "brush", "plain_slit", "brush_999"])
def test_mixed_solve_reaches_fp64_fixed_point(name):
    ds = copy.deepcopy(CASES[name])
    ds["numerical"]["tole"] = 1e-10
    ds["numerical"]["max_iters"] = 8000
    dft = descriptor(ds)
    num = numerics_from_dict(ds["numerical"])
    o = OracleSystem(dft.descriptor)
    g = native.DeviceSystem(dft.descriptor, precision=MIXED)
    it_o, err_o, rc_o, _ = o.solve(num)
    it_g, err_g, rc_g = g.solve(num)
    assert rc_o == 0 and rc_g == 0, (it_o, err_o, it_g, err_g)
    assert err_g < 1e-10
    _, bo, _ = o.densities()
    _, bg, _ = g.densities()
    om_o, om_g = o.grand_potential(), g.grand_potential()
    print(f"{name}: iterations mixed {it_g} oracle {it_o}; densities {rel(bg, bo):.2e}, "
          f"Omega {abs(om_g - om_o) / abs(om_o):.2e}")
    assert rel(bg, bo) < 1e-7
    assert abs(om_g - om_o) / abs(om_o) < 1e-8
