"""Batched wall-separation continuation on the device: every step of all
branches in one launch gives the same numbers as each branch swept alone, and
each step's grand potential matches the CPU oracle solving the same
warm-started state (converged-state tolerance)."""
import copy

import numpy as np
import pytest

from oracle.oracle import OracleSystem
from softdft_b200 import continuation as ct
from softdft_b200 import native, workloads
from softdft_b200.api import geometry_system, iLST, setup_iDFT
from softdft_b200.host.descriptor import numerics_from_dict

pytestmark = pytest.mark.gpu


def _branches():
    out = []
    for pH in (6.0, 8.0):
        ds = workloads.grafted_brush(128, 0.05, 8, 0.05, 4.5, pH, 0.01)
        ds["numerical"] = dict(ds["numerical"], tole=1e-10, max_iters=8000)
        out.append(ds)
    return out


DIST = [6.0, 5.4, 4.8]


def test_batched_sweep_equals_branches_alone():
    br = _branches()
    together = ct.batched_distance_sweep(br, DIST, dz=0.05)
    for b, ds in enumerate(br):
        alone = ct.batched_distance_sweep([ds], DIST, dz=0.05)[0]
        for s_t, s_a in zip(together[b], alone):
            assert s_t["status"] == 0 and s_t["iterations"] == s_a["iterations"]
            assert s_t["omega"] == s_a["omega"] and s_t["Pressure"] == s_a["Pressure"]
    # warm starts: later steps need fewer iterations than the cold first step
    for b in range(len(br)):
        assert together[b][-1]["iterations"] < together[b][0]["iterations"]


def test_sweep_grand_potential_matches_oracle():
    ds = _branches()[0]
    num = numerics_from_dict(ds["numerical"])
    data = copy.deepcopy(ds)
    bulk = iLST(data)
    prev = None
    for H in DIST:
        ct.set_distance(data, H, 0.05)
        geom = geometry_system(data)
        dft = setup_iDFT(data, bulk, geom)
        o = OracleSystem(dft.descriptor)
        if prev is not None:
            dft.state = ct.resample_state(prev[0], prev[1], geom)
            o.set_x(dft.handle().get_x())
        it_o, _, rc_o, _ = o.solve(num, 0)
        it_d, err_d, rc_d = dft.handle().solve(num)
        assert rc_o == 0 and rc_d == 0
        om_d, om_o = dft.handle().grand_potential(), o.grand_potential()
        assert abs(om_d - om_o) <= 1e-8 * abs(om_o)
        prev = (dft.state, geom)
        dft.handle().close()


def test_adjust_pH_sweep_writes_the_routine_files(tmp_path):
    ds = workloads.grafted_brush(128, 0.05, 8, 0.05, 4.5, 5.0, 0.01)
    ds["numerical"] = dict(ds["numerical"], max_iters=8000)
    res = ct.adjust_pH(ds, startZ=5.0, stopZ=6.0, stepZ=0.5, out_root=str(tmp_path / "pH_sweep"))
    assert [r["step"] for r in res] == [1, 2, 3] and all(r["status"] == 0 for r in res)
    alphas = [r["alpha"] for r in res]
    assert alphas[0] < alphas[1] < alphas[2]          # ionisation grows with pH
    assert all(r["brush_height"] > 0 for r in res)
    lines = open(tmp_path / "pH_sweep" / "summary_brush_alpha.csv").read().splitlines()
    assert lines[0] == "step,pH,brush_height,alpha" and len(lines) == 4
    for name in ("cvt.txt", "grand_potential.txt", "brush_height.txt", "MEP.txt", "rho_beads_K.txt"):
        assert (tmp_path / "pH_sweep" / "pH_5.50" / name).is_file(), name


# ---- pseudo-arclength continuation in pH ----

def _pac_branches():
    out = []
    for pH in (4.0, 5.0):
        ds = workloads.grafted_brush(128, 0.05, 8, 0.05, 4.5, pH, 0.01)
        ds["numerical"] = dict(ds["numerical"], tole=1e-10, max_iters=8000)
        out.append(ds)
    return out


def test_pac_points_are_solutions_on_the_constraint_hyperplane():
    res = ct.pac_pH_branches(_pac_branches(), ds_init=0.2, max_steps=5)
    for pts in res:
        assert len(pts) == 5
        for p in pts:
            assert p["status"] == 0 and p["residual"] < 1e-10
            assert 0.0 <= p["alpha"] <= 1.0
        for p in pts[2:]:
            assert p["corrector_converged"]
            assert abs(p["constraint_residual"]) <= 1e-6 * p["dS"]
        # the two natural steps point up in pH; the brush ionises as pH grows
        assert np.all(np.diff([p["pH"] for p in pts]) > 0)
        assert np.all(np.diff([p["alpha"] for p in pts]) > 0)


def test_pac_batched_branches_equal_branches_alone():
    br = _pac_branches()
    together = ct.pac_pH_branches(br, ds_init=0.2, max_steps=4)
    for b, ds in enumerate(br):
        alone = ct.pac_pH_branches([ds], ds_init=0.2, max_steps=4)[0]
        assert len(alone) == len(together[b])
        for p_t, p_a in zip(together[b], alone):
            assert p_t["pH"] == p_a["pH"] and p_t["omega"] == p_a["omega"]


def test_pac_graft_density_branch():
    """Continuation in ln(graft density) of the first grafted species: converged
    points on the constraint hyperplane; the denser left brush grows taller."""
    ds = _pac_branches()[1]
    pts = ct.pac_graft_branches([ds], ds_init=0.2, max_steps=4)[0]
    assert len(pts) == 4
    for p in pts:
        assert p["status"] == 0 and p["residual"] < 1e-10
    for p in pts[2:]:
        assert p["corrector_converged"] and abs(p["constraint_residual"]) <= 1e-6 * p["dS"]
    dens = [p["graft_density"] for p in pts]
    assert dens[0] == pytest.approx(0.05, rel=1e-12) and np.all(np.diff(dens) > 0)
    assert np.all(np.diff([p["brush_height"] for p in pts]) > 0)
