"""Serving: jobs that arrive over time share batched steps with other jobs,
yet each job's particles equal those of the same job run alone, bit for bit
(every draw is keyed by the job's seed and its own step count)."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import serve

pytestmark = pytest.mark.gpu


def test_job_same_served_and_alone(gpu_lib):
    jobs = serve.poisson_jobs(9, rate=200.0, seed=3, n_min=1e3, n_max=2e4, steps=(3, 12))
    server = serve.Server([pm.COAG_KERNEL_TYPE_ADDITIVE, pm.COAG_KERNEL_TYPE_BROWN, pm.COAG_KERNEL_TYPE_SEDI],
                          slots=4, keep_results=True)
    m = serve.run(jobs, server)
    assert m["jobs"] == len(jobs)
    assert m["tick_latency_ms"]["p99"] >= m["tick_latency_ms"]["p50"] > 0
    for j in jobs:
        alone = pm.AeroState(serve.species_of(j.kernel), j.pop.awa, seed=j.seed, mode=pm.MODE_MIXED)
        alone.add_particles(j.pop.vol, j.pop.group)
        for _ in range(j.n_steps):
            pm.mc_coag(j.kernel, pm.EnvState(j.temp, j.pressure, 1000.0), alone.aero_data, alone, server.del_t[j.kernel])
        a = alone.particles()
        for key in a:
            assert np.array_equal(a[key], j.result[key]), (j.jid, key)


def test_admission_respects_the_hbm_budget(gpu_lib):
    jobs = serve.poisson_jobs(4, rate=1000.0, seed=8, n_min=5e3, n_max=6e3, steps=(2, 3),
                              kernels=(pm.COAG_KERNEL_TYPE_ADDITIVE,))
    budget = 1.5 * max(j.n_part for j in jobs) * serve.BYTES_PER_PARTICLE
    server = serve.Server([pm.COAG_KERNEL_TYPE_ADDITIVE], slots=4, hbm_budget=budget)
    peak = 0.0
    orig = server.admit

    def admit(job):
        nonlocal peak
        ok = orig(job)
        peak = max(peak, server.used)
        return ok

    server.admit = admit
    m = serve.run(jobs, server)
    assert m["jobs"] == 4 and peak <= budget
