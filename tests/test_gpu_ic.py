"""The initial-condition sampler on the device (pmc_coag_gpu_add_dist_sample,
aero_state_add_aero_dist_sample of aero_state.F90:758-831) against the
oracle's restatement (oracle/ic_sampler.py), through the C ABI.

The device and the oracle draw from different random streams, so particles
are compared as distributions: two-sample Kolmogorov-Smirnov tests of the
radii and the species fractions against oracle samples of the same modes
(p > 1e-4 each), interval frequencies against the weighted probabilities,
and per-mode number concentrations estimated from the weighted particles.
What the reference fixes exactly is checked exactly: the prepared weight
magnitude of an empty state, the truncation bound of the normal sampler,
mono-disperse volumes, volume sums, IDs, groups, classes, components, the
size of a halving and the copies of a doubling."""
import math

import numpy as np
import pytest
from scipy import stats

import partmc_b200 as pm
from oracle import fractal as OF
from oracle import ic_sampler as S

pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("gpu_lib")]

WT = {pm.coagulation.AERO_WEIGHT_TYPE_NONE: S.WEIGHT_NONE, pm.coagulation.AERO_WEIGHT_TYPE_POWER: S.WEIGHT_POWER,
      pm.coagulation.AERO_WEIGHT_TYPE_MFA: S.WEIGHT_MFA}
MT = {pm.AERO_MODE_TYPE_LOG_NORMAL: S.MODE_LOG_NORMAL, pm.AERO_MODE_TYPE_EXP: S.MODE_EXP,
      pm.AERO_MODE_TYPE_MONO: S.MODE_MONO, pm.AERO_MODE_TYPE_SAMPLED: S.MODE_SAMPLED}


def oracle_mode(m):
    return S.Mode(MT[m.type], m.char_radius, m.log10_std_dev_radius, m.num_conc, m.vol_frac, m.vol_frac_std,
                  m.sample_radius, m.sample_num_conc)


def oracle_state(awa, n_part_ideal=None):
    ws = [[S.Weight(WT[int(awa.type[g, c])], awa.magnitude[g, c], awa.exponent[g, c]) for c in range(awa.n_class)]
          for g in range(awa.n_group)]
    return S.SampleState(1, ws, n_part_ideal)


def device_sample(modes, awa, density=(1000.0,), n_part_ideal=None, seed=1, fractal=None, **kw):
    st = pm.AeroState(pm.AeroData(np.array(density), fractal=fractal), awa, seed=seed)
    if n_part_ideal is not None:
        st.set_n_part_ideal(n_part_ideal)
    n = st.add_aero_dist_sample(pm.AeroDist(modes), **kw)
    return st, n


def ks(a, b):
    return stats.ks_2samp(a, b).pvalue


def test_empty_state_weight_and_count_follow_the_reference():
    """One log-normal mode into an empty state under r^-1 weighting with an
    ideal of 20,000: aero_state_prepare_weight_for_add scales the weight by
    n_add / ideal (exact, the same FP64 expression as the oracle's), and the
    count is Poisson with mean 20,000."""
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 5e-8, 0.2, 1e10)
    awa = pm.AeroWeightArray.power(-1.0, magnitude=1.0)
    st, n = device_sample([mode], awa, n_part_ideal=20000)
    o = oracle_state(awa, [[20000.0]])
    S.add_aero_dist_sample(np.random.default_rng(0), o, [oracle_mode(mode)], 1.0)
    assert st.weight_magnitudes()[0, 0] == o.weights[0][0].magnitude
    assert n == st.n_part() and abs(n - 20000) < 5 * math.sqrt(20000)


@pytest.mark.parametrize("alpha", [0.0, -1.0, -3.0])
def test_lognormal_radii_match_the_oracle(alpha):
    """Radii of a weighted log-normal mode (x_mean_prime shifted by the
    weight's exponent) against the oracle's, ~30,000 particles each."""
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 4e-8, 0.25, 1e10)
    awa = pm.AeroWeightArray.power(alpha) if alpha else pm.AeroWeightArray.flat()
    st, n = device_sample([mode], awa, n_part_ideal=30000, seed=7)
    r_dev = S.vol2rad(st.particles()["vol"][:, 0])
    o = oracle_state(awa, [[30000.0]])
    S.add_aero_dist_sample(np.random.default_rng(int(1 - alpha)), o, [oracle_mode(mode)], 1.0)
    r_orc = S.vol2rad(o.arrays()[0][:, 0])
    assert ks(np.log(r_dev), np.log(r_orc)) > 1e-4
    xp = math.log10(4e-8) - alpha * 0.25 ** 2 * math.log(10.0)
    x = np.log10(r_dev)
    assert abs(x.mean() - xp) < 4.5 * 0.25 / math.sqrt(n)


def test_truncated_normal_keeps_the_reference_bound():
    """A characteristic factor that makes the size factor 0.32 truncates the
    log-normal draws at 1 - |erf(z / 2.0**.5)| >= 0.32 (|z| <= 0.9944...):
    every device radius is inside, the bound is reached, and the truncated
    radii match the oracle's."""
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 1e-7, 0.3, 1e10)
    awa = pm.AeroWeightArray.flat()
    st, n = device_sample([mode], awa, n_part_ideal=20000, characteristic_factor=1e-6, seed=3)
    x = np.log10(S.vol2rad(st.particles()["vol"][:, 0]))
    z = (x - math.log10(1e-7)) / 0.3
    zmax = 0.99446  # 1 - erf(z / sqrt 2) = 0.32, plus rounding of log10(10**x)
    assert np.abs(z).max() < zmax and np.abs(z).max() > 0.98
    o = oracle_state(awa, [[20000.0]])
    S.add_aero_dist_sample(np.random.default_rng(4), o, [oracle_mode(mode)], 1.0, characteristic_factor=1e-6)
    zo = (np.log10(S.vol2rad(o.arrays()[0][:, 0])) - math.log10(1e-7)) / 0.3
    assert ks(z, zo) > 1e-4


def test_exponential_mode_matches_the_oracle_and_the_exponential_law():
    """aero_mode_sample_radius for an exponential mode (flat weight only):
    volumes are exponential with mean rad2vol(char_radius)."""
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_EXP, 2e-6, 0.0, 1e8)
    awa = pm.AeroWeightArray.flat()
    st, n = device_sample([mode], awa, n_part_ideal=20000, seed=9)
    v = st.particles()["vol"][:, 0]
    v0 = S.rad2vol(2e-6)
    assert stats.kstest(v / v0, "expon").pvalue > 1e-4
    o = oracle_state(awa, [[20000.0]])
    S.add_aero_dist_sample(np.random.default_rng(2), o, [oracle_mode(mode)], 1.0)
    assert ks(v, o.arrays()[0][:, 0]) > 1e-4
    # weighting other than flat is refused, as die_msg(822252601) stops the reference
    with pytest.raises(pm.PmcError):
        device_sample([mode], pm.AeroWeightArray.power(-1.0), n_part_ideal=1000)


@pytest.mark.parametrize("fractal", [None, pm.Fractal(2.2, 1e-8, 1.2)])
def test_mono_mode_volumes_are_exact(fractal):
    """A mono-disperse mode: every particle has aero_data_rad2vol(char
    radius), through the particle shape when it is fractal."""
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_MONO, 3e-7, 0.0, 1e9)
    st, n = device_sample([mode], pm.AeroWeightArray.power(-3.0), n_part_ideal=5000, fractal=fractal)
    fr = OF.Fractal() if fractal is None else OF.Fractal(2.2, 1e-8, 1.2)
    v = st.particles()["vol"][:, 0]
    assert n > 0 and np.allclose(v, OF.rad2vol(fr, 3e-7), rtol=1e-14, atol=0.0)


def test_sampled_mode_intervals_and_radii():
    """A sampled mode under r^-1 weighting: interval frequencies follow the
    weighted concentrations (aero_mode_weighted_sampled_num_conc), radii
    stay inside their interval and match the oracle's."""
    edges = np.array([1e-8, 3e-8, 1e-7, 4e-7, 1e-6])
    conc = np.array([1e9, 4e9, 2e8, 5e7])
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_SAMPLED, sample_radius=edges, sample_num_conc=conc)
    awa = pm.AeroWeightArray.power(-1.0)
    st, n = device_sample([mode], awa, n_part_ideal=40000, seed=11)
    r = S.vol2rad(st.particles()["vol"][:, 0])
    idx = np.searchsorted(edges, r) - 1
    assert idx.min() >= 0 and idx.max() < 4
    p = S.weighted_sampled_num_conc(oracle_mode(mode), S.Weight(S.WEIGHT_POWER, 1.0, -1.0))
    p = p / p.sum()
    frac = np.bincount(idx, minlength=4) / n
    assert np.all(np.abs(frac - p) <= 4.5 * np.sqrt(p * (1 - p) / n))
    o = oracle_state(awa, [[40000.0]])
    S.add_aero_dist_sample(np.random.default_rng(5), o, [oracle_mode(mode)], 1.0)
    assert ks(np.log(r), np.log(S.vol2rad(o.arrays()[0][:, 0]))) > 1e-4


def test_species_volumes_match_the_oracle():
    """aero_mode_sample_vols with non-zero fraction deviations: volumes sum
    to the particle's, none negative, the per-species fractions distributed
    as the oracle's."""
    dens = (1800.0, 1000.0, 1500.0)
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 6e-8, 0.2, 1e10, vol_frac=[0.6, 0.3, 0.1],
                       vol_frac_std=[0.2, 0.1, 0.05])
    awa = pm.AeroWeightArray.flat()
    st, n = device_sample([mode], awa, density=dens, n_part_ideal=20000, seed=13)
    vol = st.particles()["vol"]
    assert vol.min() >= 0.0
    r = S.vol2rad(vol.sum(1))
    assert ks(np.log(r), np.log(10.0) * np.random.default_rng(1).normal(math.log10(6e-8), 0.2, 20000)) > 1e-4
    o = S.SampleState(3, [[S.Weight(S.WEIGHT_NONE, 1.0, 0.0)]], [[20000.0]])
    S.add_aero_dist_sample(np.random.default_rng(6), o, [oracle_mode(mode)], 1.0)
    vo = o.arrays()[0]
    for s in range(3):
        assert ks(vol[:, s] / vol.sum(1), vo[:, s] / vo.sum(1)) > 1e-4, s
    # without deviations the fractions are the mode's, up to rounding
    mode0 = pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 6e-8, 0.2, 1e10, vol_frac=[0.6, 0.3, 0.1])
    st0, _ = device_sample([mode0], awa, density=dens, n_part_ideal=2000)
    v0 = st0.particles()["vol"]
    assert np.allclose(v0 / v0.sum(1, keepdims=True), [0.6, 0.3, 0.1], rtol=1e-13, atol=0.0)


def test_ids_groups_classes_and_components():
    """Particles come in the reference's order (group, then mode) with
    consecutive new IDs, the class of their source (n_class > 1), one
    component with the mode's source and the creation time, and one primary
    particle."""
    modes = [pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 3e-8, 0.2, 1e10, source=2),
             pm.AeroMode(pm.AERO_MODE_TYPE_MONO, 2e-7, 0.0, 1e8, source=1)]
    awa = pm.AeroWeightArray(np.full((2, 2), pm.coagulation.AERO_WEIGHT_TYPE_POWER), np.ones((2, 2)),
                             np.array([[0.0, 0.0], [-3.0, -3.0]]))
    st = pm.AeroState(pm.AeroData(np.array([1000.0])), awa, seed=3)
    st.set_next_id(101)
    st.set_n_part_ideal(8000)
    n = st.add_aero_dist_sample(pm.AeroDist(modes), create_time=42.0)
    p = st.particles(components=True)
    assert n == len(p["id"]) > 0
    assert np.array_equal(p["id"], 101 + np.arange(n))
    assert st.next_id() == 101 + n
    g, c = p["weight_group"], p["weight_class"]
    # order: group 1 (mode 1, mode 2), group 2 (mode 1, mode 2)
    key = (g - 1) * 2 + np.where(c == 2, 0, 1)
    assert np.all(np.diff(key) >= 0) and set(g) == {1, 2} and set(c) == {1, 2}
    assert np.array_equal(p["comp_source"][:, 0], c)  # class = source
    assert np.all(p["n_comp"] == 1) and np.all(p["comp_create_time"][:, 0] == 42.0)
    assert np.all(p["n_primary_parts"] == 1)
    mono = c == 1
    assert np.allclose(p["vol"][mono, 0], S.rad2vol(2e-7), rtol=1e-14)


def test_multi_mode_halving_estimates_every_mode_without_bias():
    """Three modes under nummass weights (flat and r^-3 groups) with an
    ideal of 2000: the later modes push a group past twice its ideal and
    the device halves it (a uniform subset removed, each recorded as
    AERO_INFO_HALVED).  Per source, the sum of the particles' combined
    number concentrations estimates the mode's concentration without bias,
    on the device as in the oracle (16 runs each, 4.5 standard errors)."""
    modes = [pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 2e-8, 0.2, 3e9),
             pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 1.2e-7, 0.25, 5e9),
             pm.AeroMode(pm.AERO_MODE_TYPE_MONO, 3e-7, 0.0, 2e8)]
    awa = pm.AeroWeightArray.nummass()
    truth = np.array([m.num_conc for m in modes])
    dev, orc = [], []
    halved = 0
    for k in range(16):
        st = pm.AeroState(pm.AeroData(np.array([1000.0])), awa, seed=50 + k)
        st.set_record_removals(True)
        st.set_n_part_ideal(2000)
        st.add_aero_dist_sample(pm.AeroDist(modes))
        rm = st.removals()
        halved += len(rm["id"])
        assert np.all(rm["action"] == 3)
        p = st.particles(components=True)
        assert not np.isin(p["id"], rm["id"]).any()
        w = pm.AeroWeightArray(awa.type, st.weight_magnitudes(), awa.exponent)
        nc = w.num_conc_at_radius(1, S.vol2rad(p["vol"][:, 0]))
        src = p["comp_source"][:, 0]
        dev.append([nc[src == s + 1].sum() for s in range(3)])
        o = oracle_state(awa, [[1000.0], [1000.0]])
        S.add_aero_dist_sample(np.random.default_rng(80 + k), o, [oracle_mode(m) for m in modes], 1.0)
        vo, _, _, so, _ = o.arrays()
        wo = pm.AeroWeightArray(awa.type, np.array([[o.weights[0][0].magnitude], [o.weights[1][0].magnitude]]),
                                awa.exponent)
        nco = wo.num_conc_at_radius(1, S.vol2rad(vo[:, 0]))
        orc.append([nco[so == s + 1].sum() for s in range(3)])
    assert halved > 0
    for est in (np.array(dev), np.array(orc)):
        z = np.abs(est.mean(0) - truth) / (est.std(0, ddof=1) / math.sqrt(len(est)))
        assert z.max() < 4.5, z


def test_doubling_copies_existing_members():
    """Existing particles, then a distribution whose expected count leaves
    the group below half its ideal: with allow_doubling the weight is scaled
    by ratio = n_new / ideal and every member ends as prob_round(1/ratio)
    particles (copies with the member's volumes and new IDs); without it
    nothing is copied and the weight is kept."""
    rng = np.random.default_rng(4)
    n0 = 3000
    vol = S.rad2vol(10.0 ** rng.normal(-7.0, 0.2, n0))
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_MONO, 1e-6, 0.0, 1e-30)  # adds nothing, n_add ~ 0
    for allow in (True, False):
        awa = pm.AeroWeightArray.power(-1.0, magnitude=2.0)
        st = pm.AeroState(pm.AeroData(np.array([1000.0])), awa, seed=8)
        st.add_particles(vol)
        st.set_n_part_ideal(10000)
        st.add_aero_dist_sample(pm.AeroDist([mode]), allow_doubling=allow)
        p = st.particles()
        n_add = 1e-30 / (2.0 * 1e-6 ** -1.0)
        ratio = (n0 + n_add) / 10000.0
        if not allow:
            assert len(p["id"]) == n0 and st.weight_magnitudes()[0, 0] == 2.0
            continue
        assert st.weight_magnitudes()[0, 0] == 2.0 * ratio
        m = len(p["id"])
        q = 1.0 / ratio - math.floor(1.0 / ratio)
        assert abs(m / n0 - 1.0 / ratio) < 5 * math.sqrt(q * (1 - q) / n0)
        assert len(np.unique(p["id"])) == m
        _, k = np.unique(p["vol"][:, 0], return_counts=True)
        assert set(k) <= {math.floor(1.0 / ratio), math.ceil(1.0 / ratio)}


def test_halving_removes_the_drawn_number_uniformly():
    """An existing group far above twice its ideal: the device removes
    prob_round(n (1 - 1/ratio)) members (floor or ceiling), records each,
    and the survivors' sizes follow the population's (uniform removal)."""
    rng = np.random.default_rng(9)
    n0 = 50000
    vol = S.rad2vol(10.0 ** rng.normal(-7.0, 0.3, n0))
    mode = pm.AeroMode(pm.AERO_MODE_TYPE_MONO, 1e-6, 0.0, 1e-30)
    st = pm.AeroState(pm.AeroData(np.array([1000.0])), pm.AeroWeightArray.flat(magnitude=1.0), seed=21)
    st.set_record_removals(True)
    st.add_particles(vol)
    st.set_n_part_ideal(7000)
    st.add_aero_dist_sample(pm.AeroDist([mode]))
    p = st.particles()
    ratio = (n0 + 1e-30) / 7000.0
    removed = n0 - len(p["id"])
    assert removed in (math.floor(n0 * (1 - 1 / ratio)), math.ceil(n0 * (1 - 1 / ratio)))
    assert len(st.removals()["id"]) == removed
    assert st.weight_magnitudes()[0, 0] == ratio
    assert ks(np.log(p["vol"][:, 0]), np.log(vol)) > 1e-4


def test_sample_then_step():
    """A sampled population steps like an uploaded one: the Brownian step
    runs and conserves the weighted volume within its statistics."""
    modes = [pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 2e-8, 0.2, 3e9),
             pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, 1.2e-7, 0.25, 5e9)]
    st = pm.AeroState(pm.AeroData(np.array([1000.0])), pm.AeroWeightArray.nummass(), seed=2)
    st.set_n_part_ideal(50000)
    st.add_aero_dist_sample(pm.AeroDist(modes))
    env = pm.EnvState(288.0, 1e5)
    n0 = st.n_part()
    tot = 0
    for _ in range(5):
        s, c = pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, st.aero_data, st, 60.0)
        tot += c
    assert tot > 0 and st.n_part() <= n0
