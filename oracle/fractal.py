"""Fractal particle radii of the reference, restated for the CPU.

TEST INFRASTRUCTURE ONLY: the checker for a device mobility radius, never the
product.

Follows fractal.F90 (after Naumann 2003, J. Aerosol Sci. 34, 1371-1397): the
geometric radius of a cluster of N monomers of radius R0 with fractal
dimension d_f and filling factor f (fractal.F90:90-172), the accessible
surface (:199-216), the Kirkwood-Riseman ratio (:223-231), the continuum and
effective radii (:239-268), the slip correction (:276-291), and the two
Newton solves between mass-equivalent volume and mobility-equivalent radius
(:315-428), with the reference's tolerance (relative step 1e-14) and step
limit (10).  The air mean free path is util.F90:289-312 with the constants of
constants.F90.

Pinned by the reference's own test/fractal/test_fractal_radii_conversion.F90:
the round trips R_me -> V -> R_me and R_geo -> V -> R_geo over its grid of
R0, f and d_f agree to the relative tolerance of util.F90:318-339.
"""
import math

PI = 3.14159265358979323846
BOLTZMANN = 1.3806505e-23
AVOGADRO = 6.02214179e23
UNIV_GAS_CONST = 8.314472
AIR_MOLEC_WEIGHT = 2.89644e-2

A_SLIP, Q_SLIP, B_SLIP = 1.142, 0.588, 0.999  # fractal.F90:40-45
SCALE_FACTOR_S_ACC, SCALE_EXPONENT_S_ACC = 1.0, 0.86  # fractal.F90:46-51
NEWTON_REL_TOL, NEWTON_MAX_STEPS = 1e-14, 10


class Fractal:
    """fractal_t: volume fractal dimension, primary radius (m), volume
    filling factor.  The defaults are fractal_set_spherical (fractal.F90:73-82)."""

    def __init__(self, frac_dim=3.0, prime_radius=1e-8, vol_fill_factor=1.0):
        self.frac_dim, self.prime_radius, self.vol_fill_factor = float(frac_dim), float(prime_radius), \
            float(vol_fill_factor)

    def is_spherical(self):
        return self.frac_dim == 3.0 and self.vol_fill_factor == 1.0


def sphere_vol2rad(v):
    return (3.0 * v / 4.0 / PI) ** (1.0 / 3.0)


def sphere_rad2vol(r):
    return 4.0 * PI * r ** 3 / 3.0


def air_mean_free_path(temp, pressure):
    """util.F90:289-312"""
    rhoair = pressure * AIR_MOLEC_WEIGHT / (UNIV_GAS_CONST * temp)
    viscosd = 1.8325e-5 * (296.16 + 120.0) / (temp + 120.0) * (temp / 296.16) ** 1.5
    viscosk = viscosd / rhoair
    gasspeed = math.sqrt(8.0 * BOLTZMANN * temp * AVOGADRO / (PI * AIR_MOLEC_WEIGHT))
    return 2.0 * viscosk / gasspeed


def vol_to_num_of_monomers(fr, v):
    return (sphere_vol2rad(v) / fr.prime_radius) ** 3


def vol2rad(fr, v):
    if fr.is_spherical():
        return sphere_vol2rad(v)
    return fr.prime_radius * (vol_to_num_of_monomers(fr, v) * fr.vol_fill_factor) ** (1.0 / fr.frac_dim)


def rad2vol(fr, r):
    if fr.is_spherical():
        return sphere_rad2vol(r)
    return sphere_rad2vol(fr.prime_radius) * (r / fr.prime_radius) ** fr.frac_dim / fr.vol_fill_factor


def surface_frac_dim(fr):
    if fr.frac_dim <= 2.0:
        return 3.0
    if fr.frac_dim <= 3.0:
        return 6.0 / fr.frac_dim
    raise ValueError("volume fractal dimension larger than 3")


def vol_to_accessible_surface(fr, v):
    ds = surface_frac_dim(fr)
    n = vol_to_num_of_monomers(fr, v)
    return 4.0 * PI * fr.prime_radius ** 2 * n ** (ds / 3.0) * (
        (ds - 2.0) * (SCALE_FACTOR_S_ACC / n) ** (1.0 - SCALE_EXPONENT_S_ACC) - ds + 3.0)


def kirkwood_riseman(fr):
    return -0.06483 * fr.frac_dim ** 2 + 0.6353 * fr.frac_dim - 0.4898


def vol_to_mobility_rad_in_continuum(fr, v):
    return kirkwood_riseman(fr) * vol2rad(fr, v)


def vol_to_effective_rad(fr, v):
    return vol_to_accessible_surface(fr, v) / 4.0 / PI / vol_to_mobility_rad_in_continuum(fr, v)


def slip_correct(r_eff, temp, pressure):
    fp = air_mean_free_path(temp, pressure)
    return 1.0 + A_SLIP * fp / r_eff + Q_SLIP * fp / r_eff * math.exp(-B_SLIP * r_eff / fp)


def _newton(f_df, x):
    """The reference's loop: at most 10 steps, stop when the relative step
    is below 1e-14; not converging by the last step is an error."""
    for step in range(1, NEWTON_MAX_STEPS + 1):
        f, df = f_df(x)
        x = x - f / df
        if abs(f / df) / (abs(x + f / df) + abs(x)) < NEWTON_REL_TOL:
            break
    if not step < NEWTON_MAX_STEPS:
        raise ArithmeticError("fractal Newton loop failed to converge")
    return x


def vol_to_mobility_rad(fr, v, temp, pressure):
    """fractal_vol_to_mobility_rad, fractal.F90:315-362"""
    if fr.is_spherical():
        return vol2rad(fr, v)
    rmec = vol_to_mobility_rad_in_continuum(fr, v)
    c_reff = slip_correct(vol_to_effective_rad(fr, v), temp, pressure)
    fp = air_mean_free_path(temp, pressure)
    a1, a2, a3, a4, a5 = c_reff, -rmec, -rmec * Q_SLIP * fp, -B_SLIP / fp, -rmec * A_SLIP * fp

    def f_df(x):
        e = math.exp(a4 * x)
        return a1 * x ** 2 + a2 * x + a3 * e + a5, 2.0 * a1 * x + a2 + a3 * a4 * e

    return _newton(f_df, rmec)


def mobility_rad_to_mobility_rad_in_continuum(fr, rme, temp, pressure):
    """fractal.F90:370-428"""
    c_rme = slip_correct(rme, temp, pressure)
    fp = air_mean_free_path(temp, pressure)
    ds = surface_frac_dim(fr)
    base = fr.vol_fill_factor * kirkwood_riseman(fr) ** fr.frac_dim * fr.prime_radius ** fr.frac_dim
    phi = fr.prime_radius ** 2 / base ** (ds / 3.0)
    psi = 1.0 / base ** (SCALE_EXPONENT_S_ACC - 1.0)
    c1 = fr.frac_dim * ds / 3.0 + (SCALE_EXPONENT_S_ACC - 1.0) * fr.frac_dim - 1.0
    c2 = fr.frac_dim * ds / 3.0 - 1.0
    a1 = c_rme / rme * phi * psi * (ds - 2.0)
    a2 = c_rme / rme * phi * (3.0 - ds)
    a3 = -phi * psi * (ds - 2.0)
    a4 = phi * (ds - 3.0)
    a5 = -Q_SLIP * fp
    a6 = -B_SLIP / fp * phi * psi * (ds - 2.0)
    a7 = -B_SLIP / fp * phi * (3.0 - ds)
    a8 = -A_SLIP * fp

    def f_df(x):
        e = math.exp(a6 * x ** c1 + a7 * x ** c2)
        f = a1 * x ** (c1 + 1.0) + a2 * x ** (c2 + 1.0) + a3 * x ** c1 + a4 * x ** c2 + a5 * e + a8
        df = (a1 * (c1 + 1.0) * x ** c1 + a2 * (c2 + 1.0) * x ** c2 + a3 * c1 * x ** (c1 - 1.0)
              + a4 * c2 * x ** (c2 - 1.0) + a5 * (a6 * c1 * x ** (c1 - 1.0) + a7 * c2 * x ** (c2 - 1.0)) * e)
        return f, df

    return _newton(f_df, rme)


def mobility_rad_to_geometric_rad(fr, rme, temp, pressure):
    if fr.is_spherical():
        return rme
    return mobility_rad_to_mobility_rad_in_continuum(fr, rme, temp, pressure) / kirkwood_riseman(fr)


def mobility_rad_to_vol(fr, rme, temp, pressure):
    return rad2vol(fr, mobility_rad_to_geometric_rad(fr, rme, temp, pressure))


def logspace(lo, hi, n):
    """util.F90:492-518, end points exact"""
    if n == 1:
        return [lo]
    la, lb = math.log(lo), math.log(hi)
    out = [math.exp((1.0 - i / (n - 1)) * la + i / (n - 1) * lb) for i in range(n)]  # linspace, util.F90:460-488
    out[0], out[-1] = lo, hi
    return out


def almost_equal(d1, d2, eps=1e-8):
    """util.F90:318-339"""
    return d1 == d2 or abs(d1 - d2) / (abs(d1) + abs(d2)) < eps
