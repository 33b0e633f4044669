"""The oracle's restatement of fractal.F90 (oracle/fractal.py), pinned by
the reference's own test/fractal/test_fractal_radii_conversion.F90 and by
the limits the formulas must reach.  CPU only."""
import math

import pytest

from oracle import fractal as F

TEMP, PRESSURE = 300.0, 1e5  # test_fractal_radii_conversion.F90:18-19


def test_radii_round_trips_over_the_reference_grid():
    """test_fractal_radii_conversion.F90: for R0 in 1e-10..1e-7 m, f in
    {1, 1.43}, d_f in 1.8..3, and 100 radii from R0 to 1000 R0, the round
    trips R_me -> V -> R_me and R_geo -> V -> R_geo agree to util.F90's
    almost_equal (relative 1e-8); every Newton solve converges in under 10
    steps (an error otherwise)."""
    bad = []
    for r0 in (1e-10, 1e-9, 1e-8, 1e-7):
        radii = F.logspace(r0, r0 * 1e3, 100)
        for f in (1.0, 1.43):
            for df in (1.8, 2.0, 2.2, 2.4, 2.6, 2.8, 3.0):
                fr = F.Fractal(df, r0, f)
                for r in radii:
                    rme = F.vol_to_mobility_rad(fr, F.mobility_rad_to_vol(fr, r, TEMP, PRESSURE), TEMP, PRESSURE)
                    rgeo = F.vol2rad(fr, F.rad2vol(fr, r))
                    if not F.almost_equal(r, rme) or not F.almost_equal(r, rgeo):
                        bad.append((r0, f, df, r, rme, rgeo))
    assert not bad, bad[:5]


def test_spherical_particles_keep_the_geometric_radius():
    """fractal_set_spherical (d_f 3, f 1): the mobility radius is the radius
    of the volume-equivalent sphere."""
    fr = F.Fractal()
    for v in (1e-27, 4e-21, 3e-18):
        assert F.vol_to_mobility_rad(fr, v, TEMP, PRESSURE) == F.sphere_vol2rad(v)


def test_continuum_limit():
    """Far above the mean free path the slip correction goes to 1 and the
    mobility radius to the continuum one (Kirkwood-Riseman ratio times the
    geometric radius).  Compact clusters (d_f 2.4, 2.8) are there within
    1e-3 at a geometric radius of 0.3 mm; open ones (d_f 1.8, whose
    effective radius grows slowly) approach it monotonically."""
    for df in (2.4, 2.8):
        fr = F.Fractal(df, 1e-8, 1.0)
        v = F.rad2vol(fr, 3e-4)
        assert F.vol_to_mobility_rad(fr, v, TEMP, PRESSURE) == pytest.approx(
            F.vol_to_mobility_rad_in_continuum(fr, v), rel=1e-3)
    fr = F.Fractal(1.8, 1e-8, 1.0)
    gaps = []
    for rg in (1e-6, 1e-5, 1e-4, 3e-4):
        v = F.rad2vol(fr, rg)
        gaps.append(abs(F.vol_to_mobility_rad(fr, v, TEMP, PRESSURE) / F.vol_to_mobility_rad_in_continuum(fr, v) - 1))
    assert all(a > b for a, b in zip(gaps, gaps[1:])) and gaps[-1] < 0.02


def test_mean_free_path_at_standard_conditions():
    """util.F90:289-312 at 300 K and 1e5 Pa: about 68 nm."""
    assert F.air_mean_free_path(TEMP, PRESSURE) == pytest.approx(6.8e-8, rel=0.03)


def test_surface_fractal_dimension():
    """fractal_surface_frac_dim: 3 up to d_f 2, 6 / d_f up to 3, an error above."""
    assert F.surface_frac_dim(F.Fractal(1.8)) == 3.0
    assert F.surface_frac_dim(F.Fractal(2.4)) == pytest.approx(2.5)
    with pytest.raises(ValueError):
        F.surface_frac_dim(F.Fractal(3.2))
