"""Order of events within one step, against the oracle's sequential loop.

The parallel step draws every pair's samples from the state at the start of
the step.  In the reference's loop (coagulation.F90:43-96) a particle that
an event creates at one bin pair is tested again by every later pair of the
step, so a particle can coagulate several times per step, and a runaway
collector can absorb hundreds of droplets in one step.  The device carries
this on with walks and chains.  Both tests compare ensembles of independent
runs, the GPU's against the oracle's, within 4 sigma of their combined
Monte Carlo error."""
import numpy as np
import pytest

import partmc_b200 as pm
from oracle import exact as E
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_BATCH = 256


def compare(name, a, b, n_sigma=4.0):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    sem = np.sqrt(a.var() / len(a) + b.var() / len(b))
    assert abs(a.mean() - b.mean()) < n_sigma * sem, (name, a.mean(), b.mean(), sem)


def test_one_step_moments_match_oracle(gpu_lib):
    """One step of the additive kernel from one fixed state of 1e4
    particles (flat weights, mean volume 40 times the initial one of
    test/additive): the growth of the second and third volume moments and
    the number of events, 4096 runs each.  Without the tests of particles
    made earlier in the step, the second moment grew about 2% too slowly,
    several sigma at this ensemble size."""
    n, vbar, dt = 10000, 40.0, 1.0
    v0 = E.rad2vol(1e-5)
    vols = -vbar * v0 * np.log(np.random.default_rng(1).random(n))
    w = 1e9 / vbar / n
    m2, m3 = (vols ** 2).sum(), (vols ** 3).sum()
    reps = 16 * N_BATCH

    def stats(v):
        return (v ** 2).sum() / m2 - 1.0, (v ** 3).sum() / m3 - 1.0, n - len(v)

    cpu = []
    for k in range(reps):
        orc = O.Oracle([1000.0], ([[1]], [[w]], [[0.0]]), seed=1000 + k)
        orc.add_particles(vols[:, None], O.make_meta(n))
        orc.mc_coag(O.KERNEL_ADDITIVE, 288.0, 1e5, 1000.0, dt)
        cpu.append(stats(orc.particles()[0].sum(1)))
    gpu = []
    for it in range(reps // N_BATCH):
        st = pm.AeroState(pm.AeroData([1000.0]), pm.AeroWeightArray.flat(magnitude=w), mode=pm.MODE_FP64,
                          n_pop=N_BATCH, seeds=np.arange(1 + it * N_BATCH, 1 + (it + 1) * N_BATCH, dtype=np.uint64))
        for p in range(N_BATCH):
            st.add_particles(vols[:, None], pop=p)
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_ADDITIVE, 288.0, 1e5, 1000.0, st, dt)
        for p in range(N_BATCH):
            gpu.append(stats(st.particles(pop=p)["vol"].sum(1)))
        st.close()
    cpu, gpu = np.array(cpu), np.array(gpu)
    for j, name in enumerate(("dM2/M2", "dM3/M3", "events")):
        compare(name, gpu[:, j], cpu[:, j])


def sedi_population(seed, n_part=1000):
    """test/sedi's initial condition (aero_init_dist.dat): one log-normal
    mode, geometric mean diameter 20 um, log10 of the geometric standard
    deviation 0.2, 1e9 m^-3, water density, flat weights."""
    rng = np.random.default_rng(seed)
    d = np.exp(np.log(2e-5) + np.log(10 ** 0.2) * rng.standard_normal(n_part))
    return np.pi / 6 * d ** 3


def test_sedi_runaway_matches_oracle_ensemble(gpu_lib):
    """test/sedi's initial condition (1000 particles): the sedimentation
    kernel's runaway collector holds half the mass after 60 s and absorbs
    droplets in chains.  Particles left, the largest particle's share of the
    mass and the second moment at 20, 40 and 60 s, 256 runs each, with steps
    of 0.2 s; the volume is conserved exactly and IDs stay unique.  (At the
    test's own 5 s steps the device's collector grows about 12% slower by
    60 s than the sequential loop's, which itself runs about 9% faster at
    5 s than at 0.2 s: the loop counts a pair's members at the pair's start,
    after every earlier pair but before every later one.)"""
    n_part, dt, times = 1000, 0.2, (20, 40, 60)
    n_steps = int(round(times[-1] / dt))
    members = [sedi_population(s, n_part) for s in range(N_BATCH)]

    def stats(v, v_init):
        return len(v), v.max() / v_init.sum(), (v ** 2).sum() / (v_init ** 2).sum()

    def at(step):
        t = step * dt
        return round(t) if abs(t - round(t)) < 1e-9 and round(t) in times else None

    cpu = {t: [] for t in times}
    for k, vol in enumerate(members):
        orc = O.Oracle([1000.0], ([[1]], [[1e9 / n_part]], [[0.0]]), seed=k + 7)
        orc.add_particles(vol[:, None], O.make_meta(n_part))
        orc.set_next_id(n_part + 1)
        for step in range(1, n_steps + 1):
            orc.mc_coag(O.KERNEL_SEDI, 288.0, 1e5, 0.0, dt)
            if at(step) is not None:
                cpu[at(step)].append(stats(orc.particles()[0].sum(1), vol))
    st = pm.AeroState(pm.AeroData([1000.0]), pm.AeroWeightArray.flat(magnitude=1e9 / n_part), mode=pm.MODE_FP64,
                      n_pop=N_BATCH, seeds=np.arange(501, 501 + N_BATCH, dtype=np.uint64))
    for p, vol in enumerate(members):
        st.add_particles(vol[:, None], pop=p)
    gpu = {t: [] for t in times}
    for step in range(1, n_steps + 1):
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_SEDI, 288.0, 1e5, 0.0, st, dt)
        if at(step) is not None:
            for p, vol in enumerate(members):
                part = st.particles(pop=p)
                v = part["vol"].sum(1)
                gpu[at(step)].append(stats(v, vol))
                assert len(np.unique(part["id"])) == len(v)
                assert abs(v.sum() / vol.sum() - 1.0) < 1e-12
    for t in times:
        c, g = np.array(cpu[t]), np.array(gpu[t])
        for j, name in enumerate(("particles left", "largest share", "M2")):
            compare(f"{name} at {t} s", g[:, j], c[:, j])
