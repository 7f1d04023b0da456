"""Continuation helpers on the host: grid rule, warm-start resampling, the
float range of the pH sweep and the readers of the routine's files."""
import math

import numpy as np

from softdft_b200 import continuation as ct
from softdft_b200 import workloads
from softdft_b200.api import geometry_system
from softdft_b200.host.geometry import cld


def test_pow2_bin_width_gives_power_of_two_grids():
    for H in [2.0, 5.3, 19.97, 40.0, 40.0 - 1e-9]:
        for dz in [0.05, 40.0 / 8191, 0.02]:
            w = ct.pow2_bin_width(H, dz)
            NP = cld(H, w) + 1
            assert NP & (NP - 1) == 0 and w <= dz * (1 + 1e-12)
            assert NP < 2 * (cld(H, dz) + 1)


def _geom(H, dz):
    ds = workloads.weak_acid_slit(64, dz, 4, 4.5, 7.0, 0.1, 0.3)
    ds["geometry"]["dimensions"] = [H]
    ds["geometry"]["bin_width"] = [dz]
    return geometry_system(ds)


def test_resample_is_identity_on_the_same_grid():
    g = _geom(6.3, 0.1)
    rng = np.random.default_rng(0)
    st = (rng.standard_normal((g.NP, 3)), rng.standard_normal((g.NP, 2, 2)), rng.standard_normal(g.NP), np.array([0.3]))
    out = ct.resample_state(st, g, g)
    for a, b in zip(out, st):
        assert np.array_equal(np.asarray(a), np.asarray(b))


def test_resample_copies_near_wall_halves_when_the_slit_grows_by_grid_steps():
    g0, g1 = _geom(6.0, 0.1), _geom(6.4, 0.1)  # 61 -> 65 points
    rng = np.random.default_rng(1)
    psi = rng.standard_normal(g0.NP)
    st = (psi[:, None].copy(), np.zeros((g0.NP, 2, 0)), psi.copy(), np.array([1.5]))
    mu, _, p1, c1 = ct.resample_state(st, g0, g1)
    half = g1.NP // 2
    assert np.array_equal(p1[:31], psi[:31])            # left wall side: index copy
    assert np.array_equal(p1[-31:], psi[-31:])          # right wall side
    assert np.array_equal(p1[31:half + 1], np.full(half - 30, psi[30]))  # beyond the old half width: midpoint
    assert c1[0] == 1.5 and np.array_equal(mu[:, 0], p1)


def test_julia_float_range():
    assert ct.julia_range(3.0, 0.5, 5.0) == [3.0, 3.5, 4.0, 4.5, 5.0]
    r = ct.julia_range(3.0, 0.05, 10.0)
    assert len(r) == 141 and math.isclose(r[-1], 10.0)
    assert ct.julia_range(9.0, -1.0, 7.0) == [9.0, 8.0, 7.0]


def test_readers_of_the_routine_files(tmp_path):
    (tmp_path / "brush_height.txt").write_text("# Brush heights per species (computed as 2 * <z>)\n"
                                               "# Format: species brush_height\nAAAA 3.25\n")
    assert ct.read_brush_height(str(tmp_path / "brush_height.txt")) == {"AAAA": 3.25}
    assert ct.read_brush_height(str(tmp_path / "missing.txt")) == {}
    (tmp_path / "t.txt").write_text("segment state1 state2\n1 0.25 0.75\n\n"
                                    "# Average state fractions across all dissociating segments:\navg 0.3 0.7\n")
    assert ct.read_avg_state_fraction(str(tmp_path / "t.txt"), 2) == 0.7
