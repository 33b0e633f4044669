"""The oracle's restatement of the reference's initial-condition sampler
(oracle/ic_sampler.py: aero_state.F90:758-831, aero_mode.F90:495-665,
rand.F90:410-487 and 550-576), pinned by answers that follow from the
mathematics: quadrature of the weighted mode densities, the moments of the
sampled radii, the truncation rule of the normal sampler, and the volume
constraints.  CPU only."""
import math

import numpy as np
import pytest
from scipy import integrate

from oracle import ic_sampler as S

LOG10 = math.log(10.0)


def lognormal_density_log10(x, num_conc, mu, sigma):
    """number concentration per unit log10 r of a log-normal mode"""
    return num_conc / (sigma * math.sqrt(2.0 * math.pi)) * math.exp(-(x - mu) ** 2 / (2.0 * sigma ** 2))


@pytest.mark.parametrize("kind,alpha", [(S.WEIGHT_NONE, 0.0), (S.WEIGHT_POWER, -1.0), (S.WEIGHT_POWER, -3.0),
                                        (S.WEIGHT_POWER, 0.5), (S.WEIGHT_MFA, -3.0)])
def test_mode_number_matches_quadrature(kind, alpha):
    """aero_mode_number of a log-normal mode is the integral of its density
    divided by the weight at each radius."""
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=5e-8, log10_std=math.log10(1.7), num_conc=3.2e9)
    w = S.Weight(kind, magnitude=1e7 if kind == S.WEIGHT_NONE else 2.5, exponent=alpha)
    mu, sigma = math.log10(mode.char_radius), mode.log10_std

    def f(x):
        return lognormal_density_log10(x, mode.num_conc, mu, sigma) / float(w.num_conc_at_radius(10.0 ** x))

    ref, _ = integrate.quad(f, mu - 12 * sigma, mu + 12 * sigma, epsabs=0.0, epsrel=1e-12, limit=200)
    assert S.mode_number(mode, w) == pytest.approx(ref, rel=1e-9)


@pytest.mark.parametrize("alpha", [0.0, -1.0, -3.0])
def test_sampled_mode_number_matches_quadrature(alpha):
    """A sampled mode spreads each interval's concentration uniformly in
    ln r; its weighted number is the integral of that over the weight."""
    edges = np.array([1e-8, 3e-8, 1e-7, 4e-7])
    nc = np.array([1e9, 4e9, 2e8])
    mode = S.Mode(S.MODE_SAMPLED, sample_radius=edges, sample_num_conc=nc)
    w = S.Weight(S.WEIGHT_POWER, magnitude=3.0, exponent=alpha)
    ref = 0.0
    for i in range(len(nc)):
        x0, x1 = math.log(edges[i]), math.log(edges[i + 1])
        val, _ = integrate.quad(lambda x: nc[i] / (x1 - x0) / float(w.num_conc_at_radius(math.exp(x))), x0, x1,
                                epsabs=0.0, epsrel=1e-12)
        ref += val
    assert S.mode_number(mode, w) == pytest.approx(ref, rel=1e-9)


@pytest.mark.parametrize("alpha", [0.0, -1.0, -3.0])
def test_lognormal_radii_follow_the_weighted_density(alpha):
    """Under a power weight the computational particles' log10 radius is
    normal with mean log10 r_c - alpha sigma^2 ln 10 and the mode's sigma."""
    rng = np.random.default_rng(11)
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=1e-7, log10_std=0.25, num_conc=1e9)
    w = S.Weight(S.WEIGHT_POWER, magnitude=1.0, exponent=alpha)
    n = 40000
    x = np.log10([S.sample_radius(rng, mode, w, 0.0) for _ in range(n)])
    mean = math.log10(mode.char_radius) - alpha * mode.log10_std ** 2 * LOG10
    assert abs(x.mean() - mean) < 4 * mode.log10_std / math.sqrt(n)
    assert abs(x.std() / mode.log10_std - 1.0) < 4 / math.sqrt(2 * n)


def test_normal_truncation_rule():
    """rand_normal with a probability threshold keeps only draws with
    1 - |erf(z / sqrt 2)| >= threshold, which for 0.32 is |z| <= 0.994."""
    rng = np.random.default_rng(5)
    z = np.array([S.rand_normal(rng, 0.0, 1.0, 0.32) for _ in range(20000)])
    assert np.all([1.0 - abs(math.erf(v / math.sqrt(2.0))) >= 0.32 for v in z])
    assert np.abs(z).max() < 0.9945 and np.abs(z).max() > 0.98


def test_sampled_mode_radii_fall_in_intervals_by_weighted_number():
    """sample_cts_pdf picks an interval with probability proportional to its
    weighted number, and under a power weight r^-alpha is uniform inside it."""
    rng = np.random.default_rng(7)
    edges = np.array([1e-8, 3e-8, 1e-7, 4e-7])
    mode = S.Mode(S.MODE_SAMPLED, sample_radius=edges, sample_num_conc=np.array([1e9, 4e9, 2e8]))
    w = S.Weight(S.WEIGHT_POWER, magnitude=1.0, exponent=-1.0)
    n = 30000
    r = np.array([S.sample_radius(rng, mode, w, 0.0) for _ in range(n)])
    idx = np.searchsorted(edges, r) - 1
    assert idx.min() >= 0 and idx.max() < 3
    p = S.weighted_sampled_num_conc(mode, w)
    p = p / p.sum()
    frac = np.bincount(idx, minlength=3) / n
    assert np.all(np.abs(frac - p) < 4 * np.sqrt(p * (1 - p) / n))
    inside = idx == 1
    u = (r[inside] - edges[1]) / (edges[2] - edges[1])  # r^-alpha = r is uniform on the interval
    assert abs(u.mean() - 0.5) < 4 * math.sqrt(1 / 12 / inside.sum())


def test_volumes_sum_to_the_particle_and_stay_non_negative():
    """aero_mode_sample_vols: perturbed fractions projected onto sum 1,
    redrawn while any is negative; their mean stays at vol_frac."""
    rng = np.random.default_rng(3)
    mode = S.Mode(S.MODE_LOG_NORMAL, vol_frac=[0.6, 0.3, 0.1], vol_frac_std=[0.2, 0.1, 0.05])
    v = np.array([S.sample_vols(rng, mode, 2.0) for _ in range(20000)])
    assert np.allclose(v.sum(1), 2.0, rtol=1e-12, atol=0.0)
    assert v.min() >= 0.0
    assert np.allclose(v.mean(0) / 2.0, mode.vol_frac, atol=0.01)


def test_dist_sample_counts_and_groups():
    """aero_state_add_aero_dist_sample: per group and mode a Poisson count
    with mean sample_prop * aero_mode_number."""
    modes = [S.Mode(S.MODE_LOG_NORMAL, char_radius=2.5e-8, log10_std=0.2, num_conc=3.2e9),
             S.Mode(S.MODE_MONO, char_radius=1e-7, num_conc=1e8)]
    weights = [S.Weight(S.WEIGHT_POWER, magnitude=1e4, exponent=-1.0),
               S.Weight(S.WEIGHT_POWER, magnitude=3e3, exponent=-1.0)]
    prop = 1e-3
    means = np.array([[prop * S.mode_number(m, w) for m in modes] for w in weights])
    rng = np.random.default_rng(2)
    reps = 40
    counts = np.zeros((2, 2))
    for _ in range(reps):
        vols, grp, mode_of = S.add_dist_sample(rng, modes, weights, prop)
        assert vols.shape == (len(grp), 1)
        for g in range(2):
            for m in range(2):
                counts[g, m] += np.sum((grp == g) & (mode_of == m))
    assert np.all(np.abs(counts / reps - means) < 4 * np.sqrt(means / reps))
    mono = vols[mode_of == 1, 0]
    assert np.allclose(mono, S.rad2vol(1e-7), rtol=1e-12)


@pytest.mark.parametrize("alpha", [0.0, -1.0, -3.0])
def test_sampled_distribution_matches_the_mode_under_any_weighting(alpha):
    """The starting point of the reference's test/weighting: test/weighting's
    initial mode (log-normal, 3.2e9 m^-3, geometric mean diameter 20 nm,
    log10 of the geometric standard deviation 0.161), sampled with about
    10,000 computational particles under a flat or power weighting, gives
    the mode's number distribution on the test's grid (160 log bins of
    diameter from 1e-8 to 1e-3 m, extract_aero_size --num) within the test's
    relative 2-norm tolerance of 0.1 (numeric_diff --by col --rel-tol 0.1),
    each particle counted at the weight at its radius."""
    from oracle import exact as E
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=1e-8, log10_std=0.161, num_conc=3.2e9)
    unit = S.Weight(S.WEIGHT_POWER, magnitude=1.0, exponent=alpha)
    w = S.Weight(S.WEIGHT_POWER, magnitude=S.mode_number(mode, unit) / 10000.0, exponent=alpha)
    rng = np.random.default_rng(17)
    vols, grp, _ = S.add_dist_sample(rng, [mode], [w], 1.0)
    r = S.vol2rad(vols[:, 0])
    h, centers = E.size_histogram(2.0 * r, w.num_conc_at_radius(r))
    ln_sigma = mode.log10_std * LOG10
    exact = mode.num_conc / (math.sqrt(2.0 * math.pi) * ln_sigma) * np.exp(
        -(np.log(centers) - math.log(2.0 * mode.char_radius)) ** 2 / (2.0 * ln_sigma ** 2))
    assert abs(len(r) - 10000) < 5 * math.sqrt(10000)
    assert E.rel_err_by_col(exact, h)[0] < 0.1


def _state(n, weights, ideal=None, seed=0):
    """a SampleState holding n log-normal particles in group 1, class 1"""
    rng = np.random.default_rng(seed)
    st = S.SampleState(1, weights, ideal)
    for r in 10.0 ** rng.normal(-7.0, 0.2, n):
        st.add([S.rad2vol(r)], 1, 1, 1, 0.0)
    return st


def test_scale_weight_halving_removes_a_uniform_subset_of_exact_size():
    """aero_state_scale_weight, ratio > 1: prob_round(n (1 - 1/ratio))
    members removed, each recorded as halved, the weight scaled by ratio;
    the removed members are a uniform subset (their sizes follow the
    population's)."""
    n, ratio = 4000, 2.5
    kept_small = []
    for seed in range(6):
        st = _state(n, [[S.Weight(S.WEIGHT_POWER, 3.0, -1.0)]], seed=seed)
        v0 = np.array(st.vols)[:, 0]
        S.scale_weight(np.random.default_rng(100 + seed), st, 1, 1, ratio, False, True)
        left = len(st.id)
        assert n - left in (math.floor(n * (1 - 1 / ratio)), math.ceil(n * (1 - 1 / ratio)))
        assert len(st.removed) == n - left and all(a == S.INFO_HALVED for _, a in st.removed)
        assert st.weights[0][0].magnitude == 3.0 * ratio
        kept_small.append(np.mean(np.array(st.vols)[:, 0] < np.median(v0)))
    # half of the population is below the median: a uniform subset keeps half of those
    assert abs(np.mean(kept_small) - 0.5) < 4 * math.sqrt(0.25 / (6 * n / ratio))


def test_scale_weight_doubling_copies_each_member():
    """aero_state_scale_weight, ratio < 1: each member ends as
    prob_round(1/ratio) particles (aero_state_dup_particle), copies with
    new IDs and the member's volumes."""
    n, ratio = 3000, 0.3
    st = _state(n, [[S.Weight(S.WEIGHT_POWER, 3.0, -1.0)]], seed=1)
    ids0 = list(st.id)
    S.scale_weight(np.random.default_rng(5), st, 1, 1, ratio, True, False)
    m = len(st.id)
    assert abs(m / n - 1 / ratio) < 4 * math.sqrt((1 / 3) * (2 / 3) / n)
    assert st.id[:n] == ids0 and len(set(st.id)) == m
    vols = np.array(st.vols)[:, 0]
    _, k = np.unique(vols, return_counts=True)
    assert set(k) <= {3, 4}
    assert st.weights[0][0].magnitude == 3.0 * ratio


def test_prepare_weight_for_an_empty_state_sets_the_magnitude():
    """With no particles, the weight is scaled by n_add / ideal whatever
    allow_doubling / allow_halving say (aero_state.F90:1890, :1910)."""
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=5e-8, log10_std=0.2, num_conc=1e10)
    for allow in (False, True):
        st = S.SampleState(1, [[S.Weight(S.WEIGHT_POWER, 1.0, -3.0)]], [[5000.0]])
        n_avg = S.mode_number(mode, st.weights[0][0])
        S.add_aero_dist_sample(np.random.default_rng(3), st, [mode], 1.0, allow_doubling=allow,
                               allow_halving=allow)
        assert st.weights[0][0].magnitude == 1.0 * (n_avg / 5000.0)
        assert abs(len(st.id) - 5000) < 5 * math.sqrt(5000)


def combined_num_conc(weights, cls, r):
    """aero_weight_array_num_conc_at_radius: harmonic combination of the
    groups' weights of class cls (1-based) at r"""
    return 1.0 / sum(1.0 / w[cls - 1].num_conc_at_radius(r) for w in weights)


def test_multi_mode_sample_with_halving_estimates_every_mode_without_bias():
    """Three modes under two weight groups (flat and r^-3) with an ideal of
    2000 particles: the second and third modes push the groups past twice
    the ideal, so aero_state_prepare_weight_for_add halves them.  Summing
    each particle's combined number concentration per source still gives
    every mode's number concentration (an unbiased estimate)."""
    modes = [S.Mode(S.MODE_LOG_NORMAL, char_radius=2e-8, log10_std=0.2, num_conc=3e9),
             S.Mode(S.MODE_LOG_NORMAL, char_radius=1.2e-7, log10_std=0.25, num_conc=5e9),
             S.Mode(S.MODE_MONO, char_radius=3e-7, num_conc=2e8)]
    est = []
    n_halved = 0
    for seed in range(24):
        st = S.SampleState(1, [[S.Weight(S.WEIGHT_NONE, 1.0, 0.0)], [S.Weight(S.WEIGHT_POWER, 1.0, -3.0)]],
                           [[1000.0], [1000.0]])
        S.add_aero_dist_sample(np.random.default_rng(seed), st, modes, 1.0)
        n_halved += len(st.removed)
        vols, grp, cls, src, _ = st.arrays()
        r = S.vol2rad(vols[:, 0])
        nc = combined_num_conc(st.weights, 1, r)
        est.append([nc[src == k + 1].sum() for k in range(3)])
    assert n_halved > 0
    est = np.array(est)
    truth = np.array([m.num_conc for m in modes])
    z = np.abs(est.mean(0) - truth) / (est.std(0, ddof=1) / math.sqrt(len(est)))
    assert z.max() < 4.5, z
