"""Batched contexts: every population advances exactly as it would alone.

All random decisions are keyed by (population seed, step, round, pair,
sample), claims and slot allocation are per population, so a population's
particle list after several batched steps must equal, bit for bit, the list
it reaches in a context of its own with the same seed."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [pm.MODE_FP64, pm.MODE_MIXED])
def test_population_same_alone_and_in_batch(gpu_lib, mode):
    pops, temps, press = aero_dist.batched_bimodal(n_pop=4, seed=9, n_min=2e3, n_max=2e4)
    seeds = np.array([11, 22, 33, 44], dtype=np.uint64)
    ad = pops[0].aero_data
    batch = pm.AeroState(ad, pops[0].awa, mode=mode, n_pop=4, seeds=seeds)
    for k, p in enumerate(pops):
        batch.set_weight_pop(k, p.awa)
        batch.add_particles(p.vol, p.group, pop=k)
    tot = pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, batch, 600.0, n_steps=6)
    assert tot[0] > 0 and tot[1] > 0
    for k, p in enumerate(pops):
        alone = pm.AeroState(ad, p.awa, seed=int(seeds[k]), mode=mode)
        alone.add_particles(p.vol, p.group)
        for _ in range(6):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, pm.EnvState(temps[k], press[k]), ad, alone, 600.0)
        a, b = alone.particles(), batch.particles(pop=k)
        for key in a:
            assert np.array_equal(a[key], b[key]), (k, key)


def test_batch_counters_sum_over_populations(gpu_lib):
    pops, temps, press = aero_dist.batched_bimodal(n_pop=3, seed=4, n_min=1e3, n_max=5e3)
    ad = pops[0].aero_data
    batch = pm.AeroState(ad, pops[0].awa, n_pop=3, seeds=np.array([5, 6, 7], dtype=np.uint64))
    n0 = []
    for k, p in enumerate(pops):
        batch.set_weight_pop(k, p.awa)
        batch.add_particles(p.vol, p.group, pop=k)
        n0.append(p.n_part)
    s, c = pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, batch, 600.0, n_steps=2)
    assert s >= c >= 0
    assert all(batch.n_part(pop=k) > 0 for k in range(3))


def test_many_chunks_per_sort_block(gpu_lib):
    """48 populations of 60 000 particles: more sort chunks (30 each, 1440 in
    all) than the sort's co-resident blocks, so blocks sort several chunks.
    Selected populations still match their runs alone bit for bit."""
    n_pop, n = 48, 60000
    pops = [aero_dist.brown_bimodal(int(n * 1.05), seed=900 + k) for k in range(n_pop)]
    assert all(p.n_part >= n for p in pops)  # trimmed to exactly n below
    ad = pops[0].aero_data
    seeds = np.arange(1, n_pop + 1, dtype=np.uint64)
    batch = pm.AeroState(ad, pops[0].awa, n_pop=n_pop, seeds=seeds)
    for k, p in enumerate(pops):
        batch.set_weight_pop(k, p.awa)
        batch.add_particles(p.vol[:n], p.group[:n], pop=k)
    temps, press = np.full(n_pop, 288.0), np.full(n_pop, 1e5)
    pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, batch, 600.0, n_steps=2)
    for k in (0, 17, 47):
        p = pops[k]
        alone = pm.AeroState(ad, p.awa, seed=int(seeds[k]))
        alone.add_particles(p.vol[:n], p.group[:n])
        for _ in range(2):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, pm.EnvState(288.0, 1e5), ad, alone, 600.0)
        a, b = alone.particles(), batch.particles(pop=k)
        for key in a:
            assert np.array_equal(a[key], b[key]), (k, key)


def test_batched_per_particle_rounds_keep_every_population_consistent(gpu_lib):
    """test/sedi's population under number-and-mass weights, 64 members in
    one batched context, 5 s steps: the per-particle path's target
    operations, and the walkers they make, come from every population in
    the later rounds.  Each population's slots and IDs are allocated from
    its own range (the operations and events are grouped by population
    first), so after every step each member's live count matches its slots
    and its IDs are unique.  Every list of a round is built in an order that
    does not depend on scheduling, so a second run with the same seeds gives
    the same particles bit for bit, and a member ends as it would alone."""
    import reference_cases as RC
    from oracle import ic_sampler as S
    from oracle import oracle as O
    sc = RC.SEDI
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=sc["r_geom"], log10_std=sc["log10_sigma"], num_conc=sc["num_conc"])
    ws = [S.Weight(S.WEIGHT_POWER, S.mode_number(mode, S.Weight(S.WEIGHT_POWER, 1.0, a)) / 500, a)
          for a in RC.ALPHAS]
    n_pop = 64
    awa = pm.AeroWeightArray(np.array([[O.WEIGHT_POWER], [O.WEIGHT_POWER]]),
                             np.array([[ws[0].magnitude], [ws[1].magnitude]]), np.array([[0.0], [-3.0]]))
    inits = [S.add_dist_sample(np.random.default_rng(100 + k), [mode], ws, 1.0) for k in range(n_pop)]
    finals = []
    for run in range(2):
        st = pm.AeroState(pm.AeroData([1000.0]), awa, mode=pm.MODE_FP64, n_pop=n_pop,
                          seeds=np.arange(900, 900 + n_pop, dtype=np.uint64))
        for k, (vols, grp, _) in enumerate(inits):
            st.add_particles(vols, grp + 1, pop=k)
        ops = 0
        for _ in range(4):
            pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_SEDI, 288.0, 1e5, 0.0, st, 5.0)
            ops += st.conflicts()["target_ops"]
            for k in range(n_pop):
                p = st.particles(pop=k)  # the download checks the live count against the slots
                assert len(np.unique(p["id"])) == len(p["id"]) == st.n_part(pop=k)
        assert ops > 0
        finals.append([st.particles(pop=k) for k in range(n_pop)])
        st.close()
    for a, b in zip(*finals):
        for key in ("vol", "id", "weight_group"):
            assert np.array_equal(a[key], b[key]), key
    # and each member as it would run alone
    for k in (0, 17, 63):
        alone = pm.AeroState(pm.AeroData([1000.0]), awa, seed=900 + k, mode=pm.MODE_FP64)
        alone.add_particles(inits[k][0], inits[k][1] + 1)
        for _ in range(4):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_SEDI, pm.EnvState(288.0, 1e5), pm.AeroData([1000.0]), alone, 5.0)
        a = alone.particles()
        for key in ("vol", "id", "weight_group"):
            assert np.array_equal(a[key], finals[0][k][key]), (k, key)
