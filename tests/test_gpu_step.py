"""The parallel CUDA step against the reference's invariants and the oracle's
statistics, through the C ABI."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist
from oracle import exact as E
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_flat_weights_conserve_volume_and_count(gpu_lib):
    pop = aero_dist.additive_exp(20000, seed=1)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=3)
    st.add_particles(pop.vol, pop.group)
    env = pm.EnvState(288.0, 1e5, 1000.0)
    v0 = pop.vol.sum()
    n = pop.n_part
    for _ in range(50):
        ns, nc = pm.mc_coag(pm.COAG_KERNEL_TYPE_ADDITIVE, env, pop.aero_data, st, 1.0)
        assert ns >= nc >= 0
        n -= nc  # flat weights: every event removes both and creates one
        assert st.n_part() == n
    p = st.particles()
    assert abs(p["vol"].sum() / v0 - 1) < 1e-12
    assert len(np.unique(p["id"])) == len(p["id"])


@pytest.mark.parametrize("mode", [pm.MODE_FP64, pm.MODE_MIXED])
def test_additive_matches_exact_solution(gpu_lib, mode):
    N0, R, n_part = 1e9, 1e-5, 20000
    times = [60.0, 180.0, 300.0]
    hs = {t: [] for t in times}
    for k in range(6):
        pop = aero_dist.additive_exp(n_part, seed=100 + k, num_conc=N0, radius_at_mean_vol=R)
        st = pm.AeroState(pop.aero_data, pop.awa, seed=11 + k, mode=mode)
        st.add_particles(pop.vol, pop.group)
        env = pm.EnvState(288.0, 1e5, 1000.0)
        for step in range(1, 301):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_ADDITIVE, env, pop.aero_data, st, 1.0)
            if float(step) in hs:
                p = st.particles()
                d = 2 * E.vol2rad(p["vol"].sum(1))
                h, dc = E.size_histogram(d, np.full(len(d), pop.awa.magnitude[0, 0]))
                hs[float(step)].append(h)
    for t in times:
        ex = E.soln_additive_exp(dc / 2, t, N0, R, 1000.0)
        err = E.rel_err_by_col(ex, np.mean(hs[t], axis=0))[0]
        assert err < 0.05, (t, err)


@pytest.mark.parametrize("kt", [pm.COAG_KERNEL_TYPE_BROWN, pm.COAG_KERNEL_TYPE_BROWN_FREE,
                                pm.COAG_KERNEL_TYPE_BROWN_CONT])
def test_brownian_matches_oracle_ensemble(gpu_lib, kt):
    """Number and mass distributions of a power-weighted run with each of
    the Brownian kernels (transition regime, free molecular, continuum)
    agree with the oracle's ensemble within 3 sigma of the Monte Carlo
    error."""
    n_part, n_runs, n_steps = 4000, 8, 30
    env = pm.EnvState(288.0, 1e5)
    hist = {"gpu": [], "cpu": []}
    for k in range(n_runs):
        pop = aero_dist.brown_bimodal(n_part, seed=200 + k)
        st = pm.AeroState(pop.aero_data, pop.awa, seed=300 + k)
        st.add_particles(pop.vol, pop.group)
        orc = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=400 + k)
        orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
        orc.set_next_id(pop.n_part + 1)
        for _ in range(n_steps):
            pm.mc_coag(kt, env, pop.aero_data, st, 600.0)
            orc.mc_coag(kt, 288.0, 1e5, 0.0, 600.0)
        for key, vol in (("gpu", st.particles()["vol"]), ("cpu", orc.particles()[0])):
            r = E.vol2rad(vol.sum(1))
            nc = pop.awa.num_conc_at_radius(1, r)
            h, dc = E.size_histogram(2 * r, nc, n_bin=40, dmin=1e-8, dmax=1e-6)
            hist[key].append(h)
    g, c = np.array(hist["gpu"]), np.array(hist["cpu"])
    se = np.sqrt(g.var(0, ddof=1) / n_runs + c.var(0, ddof=1) / n_runs)
    ok = se > 0
    z = (g.mean(0) - c.mean(0))[ok] / se[ok]
    assert np.abs(z).max() < 4.0, np.abs(z).max()
    tot_g, tot_c = g.sum(1), c.sum(1)
    se_t = np.sqrt(tot_g.var(ddof=1) / n_runs + tot_c.var(ddof=1) / n_runs)
    assert abs(tot_g.mean() - tot_c.mean()) < 3 * se_t + 1e-9 * tot_c.mean()


def test_step_is_deterministic(gpu_lib):
    pop = aero_dist.brown_bimodal(20000, seed=7)
    env = pm.EnvState(288.0, 1e5)
    outs = []
    for _ in range(2):
        st = pm.AeroState(pop.aero_data, pop.awa, seed=5)
        st.add_particles(pop.vol, pop.group)
        for _ in range(5):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, 600.0)
        outs.append(st.particles())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_host_round_trip_each_step(gpu_lib):
    """The drop-in use: the state lives on the host; every step uploads it,
    steps it and downloads it into preallocated buffers.  Particle IDs and
    weight groups survive the round trip, volume is conserved under flat
    weights, and the download into ``out`` equals a fresh download."""
    pop = aero_dist.additive_exp(20000, seed=2)
    env = pm.EnvState(288.0, 1e5, 1000.0)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=8)
    n = pop.n_part
    cap = n + 100
    hb = {"vol": np.zeros((cap, 1)), "weight_group": np.zeros(cap, np.int32),
          "weight_class": np.zeros(cap, np.int32), "id": np.zeros(cap, np.int64),
          "n_primary_parts": np.zeros(cap, np.int32)}
    hb["vol"][:n] = pop.vol
    hb["weight_group"][:n] = pop.group
    hb["weight_class"][:n] = 1
    hb["id"][:n] = np.arange(1, n + 1)
    hb["n_primary_parts"][:n] = 1
    v0 = pop.vol.sum()
    coag = 0
    for _ in range(4):
        st.add_particles(hb["vol"][:n], hb["weight_group"][:n], hb["weight_class"][:n], ids=hb["id"][:n],
                         n_primary_parts=hb["n_primary_parts"][:n])
        _, k = pm.mc_coag(pm.COAG_KERNEL_TYPE_ADDITIVE, env, pop.aero_data, st, 60.0)
        coag += k
        got = st.particles(out=hb)
        fresh = st.particles()
        for key in fresh:
            assert np.array_equal(got[key], fresh[key]), key
        assert got["id"].shape[0] == n - k
        n = got["id"].shape[0]
    assert coag > 0
    assert np.isclose(hb["vol"][:n].sum(), v0, rtol=1e-12)
    assert len(np.unique(hb["id"][:n])) == n
    assert hb["n_primary_parts"][:n].sum() == pop.n_part
    with pytest.raises(ValueError):
        st.particles(out={**hb, "id": np.zeros(3, np.int64)})


@pytest.mark.parametrize("del_t,n_runs", [(600.0, 16), (37.5, 8)])
def test_per_particle_path_matches_oracle_ensemble(gpu_lib, del_t, n_runs):
    """A bimodal population of many 10 nm particles and few 0.5 um particles
    under power weights: the large-target / small-source bin pairs take the
    per-particle (accelerated) path of try_per_particle_coag
    (coagulation.F90:150-241).  The GPU's target operations must run, and the
    number distribution and total number must agree with the oracle's
    ensemble within the Monte Carlo error over 2400 s, at test/brownian's
    600 s steps and at short ones.  In the reference's sequential pair loop a
    target that grew into another bin, and its copies, are handled again by
    later pairs of the same step; the device's walks carry them on (before
    they did, the number came out 2.2% high at 600 s, 4.6 sigma)."""
    modes = [(1e11, 0.01e-6, np.log10(1.5)), (1e8, 0.5e-6, np.log10(1.5))]
    n_part = 8000
    n_steps = int(round(2400 / del_t))
    env = pm.EnvState(288.0, 1e5)
    hist = {"gpu": [], "cpu": []}
    ops = pp_cpu = 0
    for k in range(n_runs):
        pop = aero_dist.brown_bimodal(n_part, seed=500 + k, modes=modes)
        st = pm.AeroState(pop.aero_data, pop.awa, seed=600 + k)
        st.add_particles(pop.vol, pop.group)
        orc = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=700 + k)
        orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
        orc.set_next_id(pop.n_part + 1)
        for _ in range(n_steps):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, del_t)
            ops += st.conflicts()["target_ops"]
            orc.mc_coag(O.KERNEL_BROWN, 288.0, 1e5, 0.0, del_t)
        pp_cpu += orc.pp_targets()
        for key, vol in (("gpu", st.particles()["vol"]), ("cpu", orc.particles()[0])):
            r = E.vol2rad(vol.sum(1))
            nc = pop.awa.num_conc_at_radius(1, r)
            h, dc = E.size_histogram(2 * r, nc, n_bin=30, dmin=5e-9, dmax=5e-6)
            hist[key].append(h)
    assert pp_cpu > 0 and ops > 0, (pp_cpu, ops)
    g, c = np.array(hist["gpu"]), np.array(hist["cpu"])
    se = np.sqrt(g.var(0, ddof=1) / n_runs + c.var(0, ddof=1) / n_runs)
    ok = se > 0
    z = (g.mean(0) - c.mean(0))[ok] / se[ok]
    assert np.abs(z).max() < 4.5, np.abs(z).max()
    tot_g, tot_c = g.sum(1), c.sum(1)
    se_t = np.sqrt(tot_g.var(ddof=1) / n_runs + tot_c.var(ddof=1) / n_runs)
    assert abs(tot_g.mean() - tot_c.mean()) < 3 * se_t + 1e-9 * tot_c.mean()


def check_mirror_steps(st, pop, kt, env, del_t, n_steps):
    mirror = pm.HostMirror(st, cap=256)  # too small: the first sync regrows it
    n, full = mirror.sync()
    assert full and n == pop.n_part
    fulls = 0
    for _ in range(n_steps):
        pm.mc_coag(kt, env, pop.aero_data, st, del_t)
        n, full = mirror.sync()
        fulls += full
        a, b = mirror.particles(), st.particles()
        for key in b:
            assert np.array_equal(a[key], b[key]), key
    return fulls


@pytest.mark.parametrize("mode", [pm.MODE_MIXED, pm.MODE_REPLAY])
def test_host_mirror_tracks_every_step(gpu_lib, mode):
    """A host copy kept slot by slot and updated with only the changed slots
    equals a full download after every step: per-set events and the
    per-particle path's removals and copies, and in replay mode the
    reference's swap-last removals that shrink the slot count."""
    modes = [(1e11, 0.01e-6, np.log10(1.5)), (1e8, 0.5e-6, np.log10(1.5))]
    pop = aero_dist.brown_bimodal(6000, seed=31, modes=modes)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=4, mode=mode)
    st.add_particles(pop.vol, pop.group)
    if mode == pm.MODE_REPLAY:
        st.set_replay(np.random.default_rng(5).random(20_000_000))
    check_mirror_steps(st, pop, pm.COAG_KERNEL_TYPE_BROWN, pm.EnvState(288.0, 1e5), 600.0, 8)


def test_host_mirror_after_compaction(gpu_lib):
    """Flat-weight additive coagulation removing most particles: the library
    compacts its slots, which renumbers them, and the next sync copies every
    slot; the copy still equals a full download after every step.  Steps of
    120 s (at 600 s a particle leaves the bin grid within the first step,
    in the oracle's sequential loop as on the device)."""
    pop = aero_dist.additive_exp(20000, seed=6)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=2, mode=pm.MODE_MIXED)
    st.add_particles(pop.vol, pop.group)
    fulls = check_mirror_steps(st, pop, pm.COAG_KERNEL_TYPE_ADDITIVE, pm.EnvState(288.0, 1e5, 1000.0), 120.0, 6)
    assert st.n_part() < pop.n_part // 2
    assert fulls >= 1  # a compaction happened and forced one full copy
