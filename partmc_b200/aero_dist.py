"""Initial particle populations for the benchmark and test workloads.

Restates the reference's sampling of a mode (aero_mode_sample_radius,
aero_mode.F90:549-632) and the number of computational particles a weighted
mode yields (aero_mode_number, aero_mode.F90:496-545), so that weight
magnitudes can be set for a target particle count the way
aero_state_add_aero_dist_sample does (aero_state.F90:758-831).  Sampling
uses numpy's generator, not the reference's uniform stream.
"""
import numpy as np

from .coagulation import (AERO_WEIGHT_TYPE_NONE, AERO_WEIGHT_TYPE_POWER, AeroData, AeroWeightArray)

PI = 3.14159265358979323846


def rad2vol(r):
    return 4.0 * PI * np.asarray(r, dtype=np.float64) ** 3 / 3.0


def vol2rad(v):
    return (3.0 * np.asarray(v, dtype=np.float64) / 4.0 / PI) ** (1.0 / 3.0)


def lognormal_number(num_conc, char_radius, log10_std, w_type, w_mag, w_exp):
    """aero_mode_number for a log-normal mode."""
    if w_type == AERO_WEIGHT_TYPE_NONE:
        return num_conc / w_mag
    x = np.log10(char_radius)
    xp = x - w_exp * log10_std ** 2 * np.log(10.0)
    return num_conc / w_mag * np.exp((xp ** 2 - x ** 2) / (2.0 * log10_std ** 2))


def sample_lognormal(rng, n, char_radius, log10_std, w_type, w_exp):
    """aero_mode_sample_radius for a log-normal mode under a weight."""
    x = np.log10(char_radius)
    xp = x if w_type == AERO_WEIGHT_TYPE_NONE else x - w_exp * log10_std ** 2 * np.log(10.0)
    return 10.0 ** rng.normal(xp, log10_std, size=n)


def sample_exp(rng, n, char_radius):
    """aero_mode_sample_radius for an exponential mode (flat weight only)."""
    return vol2rad(-rad2vol(char_radius) * np.log(rng.random(n)))


class Population:
    """A population ready to upload: per-particle volumes and weights."""

    def __init__(self, aero_data, awa, vol, group, cls=None, label=""):
        self.aero_data = aero_data
        self.awa = awa
        self.vol = np.ascontiguousarray(vol, dtype=np.float64)
        self.group = np.ascontiguousarray(group, dtype=np.int32)
        self.cls = np.ones(self.vol.shape[0], dtype=np.int32) if cls is None else np.ascontiguousarray(cls, np.int32)
        self.label = label

    @property
    def n_part(self):
        return self.vol.shape[0]


def _modes_population(rng, n_part, modes, awa_kind, exponent, density, mass_fracs=None):
    """Sample n_part particles (in expectation, one Poisson draw per group and
    mode as in aero_state_add_aero_dist_sample) from log-normal modes
    (num_conc, char_radius, log10_std) under flat, power or nummass weights."""
    if awa_kind == "flat":
        groups = [(AERO_WEIGHT_TYPE_NONE, 0.0)]
    elif awa_kind == "power":
        groups = [(AERO_WEIGHT_TYPE_POWER, float(exponent))]
    elif awa_kind == "nummass":
        groups = [(AERO_WEIGHT_TYPE_NONE, 0.0), (AERO_WEIGHT_TYPE_POWER, -3.0)]
    else:
        raise ValueError(awa_kind)
    n_ideal = n_part / len(groups)
    mags = []
    vols, grp = [], []
    for gi, (wt, we) in enumerate(groups):
        tot = sum(lognormal_number(nc, r, s, wt, 1.0, we) for nc, r, s in modes)
        mag = tot / n_ideal
        mags.append(mag)
        for nc, r, s in modes:
            n = rng.poisson(lognormal_number(nc, r, s, wt, mag, we))
            rad = sample_lognormal(rng, n, r, s, wt, we)
            vols.append(rad2vol(rad))
            grp.append(np.full(n, gi + 1, dtype=np.int32))
    vtot = np.concatenate(vols)
    group = np.concatenate(grp)
    n_spec = len(density)
    if n_spec == 1:
        vol = vtot[:, None]
    else:
        f = mass_fracs(vtot.size) if mass_fracs is not None else np.full((vtot.size, n_spec), 1.0 / n_spec)
        phi = f / np.asarray(density)[None, :]
        phi = phi / phi.sum(axis=1, keepdims=True)
        vol = phi * vtot[:, None]
    if awa_kind == "flat":
        awa = AeroWeightArray.flat(magnitude=mags[0])
    elif awa_kind == "power":
        awa = AeroWeightArray.power(exponent, magnitude=mags[0])
    else:
        awa = AeroWeightArray.nummass(magnitudes=(mags[0], mags[1]))
    return AeroData(density), awa, vol, group


def additive_exp(n_part=10000, seed=1, num_conc=1e9, radius_at_mean_vol=1e-5):
    """Exponential volume distribution, flat weighting, 1 species of density
    1000 kg/m^3 (test/additive: aero_init_dist.dat, run_part.spec)."""
    rng = np.random.default_rng(seed)
    rad = sample_exp(rng, rng.poisson(n_part), radius_at_mean_vol)
    ad = AeroData([1000.0])
    awa = AeroWeightArray.flat(magnitude=num_conc / n_part)
    return Population(ad, awa, rad2vol(rad)[:, None], np.ones(rad.size, np.int32), label="additive_exp")


def brown_bimodal(n_part=100000, seed=1, exponent=-1.0, modes=None, density=1800.0):
    """Two log-normal modes, D_g 0.05 um (sigma_g 1.6, 3.2e9 m^-3) and 0.2 um
    (sigma_g 1.8, 1e8 m^-3), one species of 1800 kg/m^3, power weight."""
    rng = np.random.default_rng(seed)
    if modes is None:
        modes = [(3.2e9, 0.025e-6, np.log10(1.6)), (1e8, 0.1e-6, np.log10(1.8))]
    ad, awa, vol, grp = _modes_population(rng, n_part, modes, "power", exponent, [density])
    return Population(ad, awa, vol, grp, label="brown_bimodal")


def brown_20spec(n_part=1000000, seed=1, num_concs=(1e10, 1e9, 1e8)):
    """Twenty species with per-particle Dirichlet(1) mass fractions and
    densities U(1000, 2000) kg/m^3, three log-normal modes with D_g 0.02,
    0.1, 0.5 um and seeded sigma_g in [1.5, 2.0], nummass weighting."""
    rng = np.random.default_rng(seed)
    density = rng.uniform(1000.0, 2000.0, size=20)
    sig = rng.uniform(1.5, 2.0, size=3)
    modes = [(num_concs[k], d / 2.0, np.log10(sig[k])) for k, d in enumerate((0.02e-6, 0.1e-6, 0.5e-6))]
    fr = lambda n: rng.dirichlet(np.ones(20), size=n)
    ad, awa, vol, grp = _modes_population(rng, n_part, modes, "nummass", 0.0, density, mass_fracs=fr)
    return Population(ad, awa, vol, grp, label="brown_20spec")


def batched_bimodal(n_pop=256, seed=1, n_min=1e3, n_max=1e5, exponent=-1.0):
    """Independent bimodal populations with log-uniform particle counts,
    seeded mode diameters and widths, and per-population T and p."""
    rng = np.random.default_rng(seed)
    pops, temps, press = [], [], []
    for k in range(n_pop):
        n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        da = rng.uniform(0.03e-6, 0.08e-6)
        db = rng.uniform(0.15e-6, 0.3e-6)
        sa, sb = rng.uniform(1.4, 1.9, size=2)
        pops.append(brown_bimodal(n, seed=int(rng.integers(1 << 30)), exponent=exponent,
                                  modes=[(3.2e9, da / 2, np.log10(sa)), (1e8, db / 2, np.log10(sb))]))
        temps.append(rng.uniform(250.0, 300.0))
        press.append(rng.uniform(5e4, 1e5))
    return pops, np.array(temps), np.array(press)
