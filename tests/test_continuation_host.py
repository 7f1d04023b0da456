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


def test_grid_supported_matches_the_device_rule():
    """sdft_grid_supported (host-only): NP >= 16 whose FFT length M (NP/2 for
    even NP, NP for odd NP) fits one CTA's shared memory: directly when M has no
    prime factor above 61, else through Bluestein's chirp convolution of length
    2^k >= 2M - 1 (at most 8192 points, so M <= 4096)."""
    from softdft_b200 import native
    ok = native.grid_supported
    assert [n for n in (8, 15, 16, 17, 1000, 1001, 1024, 16384) if ok(n)] == [16, 17, 1000, 1001, 1024, 16384]
    assert ok(1009)                # prime: Bluestein over 2048 points
    assert ok(2018)                # NP/2 = 1009
    assert ok(1002)                # NP/2 = 3 * 167: Bluestein over 1024 points
    assert ok(2 * 61 * 64)         # mixed radix
    assert not ok(2 * 67 * 64)     # M = 4288 = 67 * 64: Bluestein over 16384 points, beyond one CTA
    assert not ok(4099) and not ok(8198)  # M = 4099 (prime): the same
    assert b"Bluestein transform of 16384 points" in native.lib().sdft_last_error()
    assert ok(24576) and not ok(24696) and not ok(32768)  # one CTA's shared memory: M = 12288 fits, 12348 does not


def test_supported_bin_width_keeps_the_reference_grid():
    # H = 20 sigma at dz = 0.02: the reference's NP = 1001 runs as is
    assert ct.supported_bin_width(20.0, 0.02) == 0.02
    for H, dz in [(20.0, 0.02), (19.97, 0.05), (40.0, 40.0 / 8191), (10.16, 0.01), (workloads.slit_length(4099, 0.01), 0.01)]:
        w = ct.supported_bin_width(H, dz)
        NP = cld(H, w) + 1
        from softdft_b200 import native
        assert native.grid_supported(NP) and w <= dz
        NP0 = cld(H, dz) + 1
        assert all(not native.grid_supported(n) for n in range(NP0, NP))
    # 4099 points (prime, beyond a Bluestein transform in one CTA) move to the
    # next supported size, 4100 (NP/2 = 2 * 5^2 * 41)
    H = workloads.slit_length(4099, 0.01)
    assert cld(H, 0.01) + 1 == 4099
    w = ct.supported_bin_width(H, 0.01)
    assert cld(H, w) + 1 == 4100 and w < 0.01


def test_set_distance_grid_policies():
    ds = workloads.weak_acid_slit(64, 0.02, 4, 4.5, 7.0, 0.1, 0.3)
    ct.set_distance(ds, 20.0, 0.02)
    assert ds["geometry"]["bin_width"] == [0.02]
    ct.set_distance(ds, 20.0, 0.02, grid="pow2")
    assert cld(20.0, ds["geometry"]["bin_width"][0]) + 1 == 1024
    ct.set_distance(ds, 20.0, 0.025, grid="exact")
    assert ds["geometry"]["bin_width"] == [0.025]


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


def test_pac_tangent_secant_and_three_point_difference():
    rng = np.random.default_rng(5)
    a, b, c = rng.normal(size=(3, 7))
    S = [0.0, 0.7, 1.6]
    X = [a + b * s + c * s * s for s in S]
    t2 = ct._pac_tangent(X[:2], S[:2])
    assert np.allclose(t2, (X[1] - X[0]) / np.linalg.norm(X[1] - X[0]), rtol=0, atol=1e-15)
    # the three-point backward difference is exact for a quadratic in arclength
    d = b + 2 * c * S[2]
    assert np.allclose(ct._pac_tangent(X, S), d / np.linalg.norm(d), rtol=0, atol=1e-12)
