"""aero_state_rebalance on the device (aero_state.F90:1722-1852).

Doubling copies every member of a (group, class) with a new ID and halves the
weight magnitude; halving removes each member with probability 1/2 and
doubles the magnitude.  End to end, the additive kernel's exact solution
(test/additive) must hold with rebalancing after every step, as run_part does
(run_part.F90:982), the check the oracle passes in test_oracle_exact.py."""
import numpy as np
import pytest

import partmc_b200 as pm
from oracle import exact as E

pytestmark = pytest.mark.gpu

N0, R = 1e9, 1e-5


def flat_population(n, seed):
    rng = np.random.default_rng(seed)
    vols = -E.rad2vol(R) * np.log(rng.random(n))
    return pm.AeroData([1000.0]), pm.AeroWeightArray.flat(magnitude=N0 / n), vols[:, None]


def test_doubling_copies_every_particle(gpu_lib):
    ad, awa, vol = flat_population(1000, 1)
    st = pm.AeroState(ad, awa, seed=3)
    st.add_particles(vol)
    before = st.particles()
    mag = st.rebalance(8000)  # 1000 -> 2000 -> 4000: two doublings reach ideal/2
    after = st.particles()
    assert st.n_part() == 4000
    assert np.isclose(mag[0, 0], N0 / 1000 / 4, rtol=0, atol=0)
    # every original volume appears four times; IDs are all distinct
    assert np.array_equal(np.sort(np.tile(before["vol"][:, 0], 4)), np.sort(after["vol"][:, 0]))
    assert len(np.unique(after["id"])) == 4000
    assert st.next_id() == 4001
    # the number concentration represented is unchanged
    assert np.isclose(st.n_part() * mag[0, 0], N0, rtol=1e-15)


def test_halving_removes_half(gpu_lib):
    """40 000 particles with an ideal of 10 000: halved while above 20 000;
    each halving keeps a member with probability 1/2 and doubles the
    magnitude, so the represented number concentration is kept in
    expectation."""
    ad, awa, vol = flat_population(40000, 2)
    st = pm.AeroState(ad, awa, seed=4)
    st.add_particles(vol)
    mag = st.rebalance(10000)
    n = st.n_part()
    halvings = int(round(np.log2(mag[0, 0] / (N0 / 40000))))
    assert halvings >= 1 and n <= 20000
    p = 0.5 ** halvings
    sd = np.sqrt(40000 * p * (1 - p))
    assert abs(n - 40000 * p) < 5 * sd, (n, 40000 * p, sd)
    assert len(np.unique(st.particles()["id"])) == n


def test_additive_exact_solution_with_rebalance(gpu_lib):
    """Twenty ensemble members of 1e4 particles (one batched context),
    additive kernel, 600 s of 1 s steps, each member rebalanced (doubling)
    to 1e4 after every step: within the reference test's tolerance of the
    exact solution (test_additive_1.sh / _2.sh: 0.05 in number, 0.2 in
    mass).  The mass distribution at late times rests on a few large
    particles, so the ensemble is twice the oracle's (test_oracle_exact.py)."""
    n_part, n_runs, times = 10000, 20, [60.0, 300.0, 600.0]
    hs = {t: [] for t in times}
    ms = {t: [] for t in times}
    pops = [flat_population(n_part, 1000 + k) for k in range(n_runs)]
    ad, awa, _ = pops[0]
    st = pm.AeroState(ad, awa, mode=pm.MODE_FP64, n_pop=n_runs, seeds=np.arange(77, 77 + n_runs, dtype=np.uint64))
    for k, (_, awa_k, vol) in enumerate(pops):
        st.set_weight_pop(k, awa_k)
        st.add_particles(vol, pop=k)
    for step in range(1, 601):
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_ADDITIVE, 288.0, 1e5, 1000.0, st, 1.0)
        mags = [st.rebalance(n_part, allow_halving=False, pop=k) for k in range(n_runs)]
        t = float(step)
        if t in hs:
            for k in range(n_runs):
                v = st.particles(pop=k)["vol"].sum(1)
                d = 2 * E.vol2rad(v)
                h, dc = E.size_histogram(d, np.full(len(d), mags[k][0, 0]))
                hm, _ = E.size_histogram(d, np.full(len(d), mags[k][0, 0]) * v * 1000.0)
                hs[t].append(h)
                ms[t].append(hm)
    for t in times:
        ex = E.soln_additive_exp(dc / 2, t, N0, R, 1000.0)
        exm = ex * E.rad2vol(dc / 2) * 1000.0
        num_err = E.rel_err_by_col(ex, np.mean(hs[t], axis=0))[0]
        mass_err = E.rel_err_by_col(exm, np.mean(ms[t], axis=0))[0]
        assert num_err < 0.05, (t, num_err)
        assert mass_err < 0.2, (t, mass_err)
