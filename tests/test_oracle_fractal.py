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


def test_c_oracle_radii_match_the_pinned_restatement():
    """The C oracle's fractal_vol2rad and fractal_vol_to_mobility_rad (the
    checker of the device path) against oracle/fractal.py, which the
    reference's radii round trips pin, over the reference test's grid."""
    from oracle import oracle as O
    worst = 0.0
    for r0 in (1e-10, 1e-9, 1e-8, 1e-7):
        for f in (1.0, 1.43):
            for df in (1.8, 2.0, 2.4, 2.8, 3.0):
                fr = F.Fractal(df, r0, f)
                for r in F.logspace(r0, r0 * 1e3, 25):
                    v = F.rad2vol(fr, r)
                    rg, rme = O.fractal_radius(v, df, r0, f, TEMP, PRESSURE)
                    worst = max(worst, abs(rg / F.vol2rad(fr, v) - 1),
                                abs(rme / F.vol_to_mobility_rad(fr, v, TEMP, PRESSURE) - 1))
    assert worst < 1e-12, worst


def test_c_oracle_fractal_kernels():
    """Free-molecular and continuum kernels of clusters (d_f 2.4 and 1.8, the
    shapes of test/fractal) against their formulas written out here, and the
    Brownian and sedimentation kernels reduce to the spherical ones at
    d_f = 3."""
    from oracle import oracle as O
    kB, visc = 1.3806505e-23, 1.78e-5
    for df, r0, temp in ((2.4, 5e-10, 1800.0), (1.8, 2.5e-7, 300.0)):
        v0 = 4.0 / 3.0 * math.pi * r0 ** 3
        for n1, n2 in ((1.0, 1.0), (7.0, 300.0), (2e4, 5e5)):
            v1, v2 = n1 * v0, n2 * v0
            free = O.kernel_value_fractal(O.KERNEL_BROWN_FREE, v1, 4200.0, v2, 4200.0, df, r0, 1.0, temp)
            want = math.sqrt(6 * kB * temp * r0 / 4200.0 * (1 / n1 + 1 / n2)) * (n1 ** (1 / df) + n2 ** (1 / df)) ** 2
            assert free == pytest.approx(want, rel=1e-12)
            cont = O.kernel_value_fractal(O.KERNEL_BROWN_CONT, v1, 4200.0, v2, 4200.0, df, r0, 1.0, temp)
            a, b = n1 ** (1 / df), n2 ** (1 / df)
            assert cont == pytest.approx(2 * kB * temp / 3 / visc * (1 / a + 1 / b) * (a + b), rel=1e-12)
    for kt in (O.KERNEL_BROWN, O.KERNEL_SEDI):
        v1, v2 = (1e-24, 3e-22) if kt == O.KERNEL_BROWN else (4e-15, 3e-14)
        assert O.kernel_value_fractal(kt, v1, 1500.0, v2, 1500.0, 3.0, 1e-8) == O.kernel_value(kt, v1, 1500.0, v2,
                                                                                                1500.0)
    # the cluster shape reaches the transition-regime kernel (through the
    # geometric and mobility radii)
    k_sph = O.kernel_value(O.KERNEL_BROWN, 1e-24, 1500.0, 3e-22, 1500.0)
    k_frac = O.kernel_value_fractal(O.KERNEL_BROWN, 1e-24, 1500.0, 3e-22, 1500.0, 1.8, 1e-9)
    assert k_frac != k_sph and math.isfinite(k_frac)
