"""Serving many coagulation jobs on one GPU with continuous batching.

A job is one particle population advanced by a number of mc_coag steps
with one coagulation kernel (the reference's run_part loop with only
coagulation on, run_part.F90:917-931).  The step length of each kernel type
is the one of the reference's own test for it (DEL_T).  Jobs arrive over time; the
server keeps one batched context per kernel type with a fixed number of
population slots and, every tick:

  1. admits arrived jobs into free slots while the HBM budget allows
     (upload, weights, and a fresh seed and ID counter for the slot);
  2. advances every context that holds jobs by one step (one batched launch
     sequence per context);
  3. retires jobs whose steps are done (their slot is emptied).

Because every random draw is keyed by the population's seed and its own step
count (pmc_coag_gpu_set_seed restarts it), a job's particles do not depend on
which other jobs shared its ticks.

The metrics are the ones of a server: throughput (pair tests, simulated
seconds), tick latency percentiles, and job turnaround and queueing
percentiles.
"""
import time

import numpy as np

from . import aero_dist
from . import coagulation as C

# device bytes per particle slot at one species, for admission: volumes and
# caches (vol, vtot, mass, rad: 32 B), records (48 + 32 B), scalar fields
# (about 80 B), components (20 x 12 B), sort and claim words (20 B), at the
# library's 1.5x capacity
BYTES_PER_PARTICLE = int(1.5 * (32 + 80 + 80 + 240 + 20))

# step length per kernel type: del_t of test/additive, test/sedi and
# test/brownian (run_part.spec of each)
DEL_T = {C.COAG_KERNEL_TYPE_ADDITIVE: 1.0, C.COAG_KERNEL_TYPE_SEDI: 5.0, C.COAG_KERNEL_TYPE_BROWN: 600.0}


class Job:
    def __init__(self, jid, arrival, kernel, n_steps, pop, seed, temp=288.0, pressure=1e5):
        self.jid, self.arrival, self.kernel, self.n_steps = jid, arrival, kernel, n_steps
        self.pop, self.seed, self.temp, self.pressure = pop, seed, temp, pressure
        self.start = self.finish = None
        self.steps_done = 0
        self.n_samp = self.n_coag = 0

    @property
    def n_part(self):
        return self.pop.n_part


def make_population(kernel, n_part, seed):
    """One job's population: exponential volumes with flat weights for the
    additive kernel, cloud-drop sizes for sedimentation, two log-normal modes
    with power weights for the Brownian kernel."""
    if kernel == C.COAG_KERNEL_TYPE_ADDITIVE:
        return aero_dist.additive_exp(n_part, seed=seed)
    if kernel == C.COAG_KERNEL_TYPE_SEDI:
        return aero_dist.additive_exp(n_part, seed=seed, radius_at_mean_vol=1e-5)
    return aero_dist.brown_bimodal(n_part, seed=seed)


def poisson_jobs(n_jobs, rate, seed=1, n_min=1e3, n_max=1e6, steps=(10, 200),
                 kernels=(C.COAG_KERNEL_TYPE_ADDITIVE, C.COAG_KERNEL_TYPE_BROWN, C.COAG_KERNEL_TYPE_SEDI)):
    """Seeded job stream: exponential inter-arrival times of mean 1/rate,
    particle counts log-uniform in [n_min, n_max], steps uniform in steps,
    kernels uniform over kernels."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_jobs))
    jobs = []
    for j in range(n_jobs):
        kernel = int(rng.choice(kernels))
        n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        ns = int(rng.integers(steps[0], steps[1] + 1))
        pseed = int(rng.integers(1, 2**31 - 1))
        jobs.append(Job(j, float(t[j]), kernel, ns, make_population(kernel, n, pseed), seed=pseed + 17))
    return jobs


def species_of(kernel):
    """The species of a kernel's jobs (make_population): one species of
    1800 kg/m^3 for the Brownian populations, 1000 kg/m^3 otherwise."""
    return C.AeroData([1800.0 if kernel == C.COAG_KERNEL_TYPE_BROWN else 1000.0])


class Server:
    """Batched contexts per kernel type, `slots` populations each.  All jobs
    of one kernel type share its species (species_of)."""

    def __init__(self, kernels, slots=32, hbm_budget=150e9, del_t=None, mode=C.MODE_MIXED, keep_results=False):
        # del_t: one step length for every kernel, or None for DEL_T
        self.del_t = {k: float(del_t) if del_t is not None else DEL_T.get(k, 60.0) for k in kernels}
        self.budget, self.used = float(hbm_budget), 0.0
        self.keep_results = keep_results
        self.n_samp_total = 0
        self.ctx, self.jobs = {}, {}
        for k in kernels:
            ad = species_of(k)
            st = C.AeroState(ad, C.AeroWeightArray.flat(), mode=mode, n_pop=slots,
                             seeds=np.arange(1, slots + 1, dtype=np.uint64))
            for p in range(slots):
                st.add_particles(np.zeros((0, 1)), pop=p)
            self.ctx[k] = st
            self.jobs[k] = [None] * slots

    def admit(self, job):
        """Place a job in a free slot of its kernel's context; False if there
        is none or the HBM budget would be exceeded."""
        need = job.n_part * BYTES_PER_PARTICLE
        if self.used + need > self.budget:
            return False
        slots = self.jobs[job.kernel]
        try:
            k = slots.index(None)
        except ValueError:
            return False
        st = self.ctx[job.kernel]
        st.set_weight_pop(k, job.pop.awa)
        st.set_next_id(1, pop=k)  # IDs as in a fresh run of the job (aero_particle.F90:72)
        st.add_particles(job.pop.vol, job.pop.group, pop=k)
        st.set_seed(job.seed, pop=k)
        slots[k] = job
        self.used += need
        return True

    def tick(self):
        """One step of every context that holds jobs; returns the finished
        jobs and the wall time of each context's step."""
        done, lat = [], []
        for kern, st in self.ctx.items():
            slots = self.jobs[kern]
            if not any(slots):
                continue
            temps = np.array([j.temp if j else 288.0 for j in slots])
            press = np.array([j.pressure if j else 1e5 for j in slots])
            t0 = time.perf_counter()
            s, c = C.mc_coag_batch(kern, temps, press, 1000.0, st, self.del_t[kern])
            lat.append(time.perf_counter() - t0)
            for k, j in enumerate(slots):
                if j is None:
                    continue
                j.steps_done += 1
                if j.steps_done == j.n_steps:
                    done.append((kern, k, j))
            self.n_samp_total += s
        for kern, k, j in done:
            j.result = self.ctx[kern].particles(pop=k) if self.keep_results else None
            self.ctx[kern].add_particles(np.zeros((0, 1)), pop=k)  # empty the slot
            self.jobs[kern][k] = None
            self.used -= j.n_part * BYTES_PER_PARTICLE
        return [j for _, _, j in done], lat


def warm_up(server, seed=99):
    """Run a few small jobs of every kernel type through the server, so that
    first launches (module loading, buffer growth, graph capture) fall
    outside a timed run."""
    kernels = tuple(server.ctx)
    jobs = poisson_jobs(4 * len(kernels), rate=1e4, seed=seed, n_min=2e3, n_max=2e5, steps=(4, 8), kernels=kernels)
    run(jobs, server)
    server.n_samp_total = 0


def run(jobs, server):
    """Serve a job stream in wall-clock time (arrival times are seconds after
    the start).  Returns the metrics."""
    queue = sorted(jobs, key=lambda j: j.arrival)
    pending, qi, finished, tick_lat = [], 0, [], []
    t_start = time.perf_counter()
    while len(finished) < len(jobs):
        now = time.perf_counter() - t_start
        while qi < len(queue) and queue[qi].arrival <= now:
            pending.append(queue[qi])
            qi += 1
        still = []
        for j in pending:
            if server.admit(j):
                j.start = time.perf_counter() - t_start
            else:
                still.append(j)
        pending = still
        done, lat = server.tick()
        tick_lat.extend(lat)
        now = time.perf_counter() - t_start
        for j in done:
            j.finish = now
        finished.extend(done)
        if not done and not lat and qi < len(queue):
            time.sleep(max(0.0, min(0.002, queue[qi].arrival - now)))
    wall = time.perf_counter() - t_start
    turn = np.array([j.finish - j.arrival for j in finished])
    wait = np.array([j.start - j.arrival for j in finished])
    lat = np.array(tick_lat) * 1e3
    sim_s = sum(j.n_steps * server.del_t[j.kernel] for j in finished)
    return {"jobs": len(finished), "wall_s": wall, "sim_s_per_s": sim_s / wall,
            "pair_tests_per_s": server.n_samp_total / wall,
            "particle_steps_per_s": sum(j.n_part * j.n_steps for j in finished) / wall,
            "tick_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                "max": float(lat.max())},
            "job_turnaround_s": {"p50": float(np.percentile(turn, 50)), "p99": float(np.percentile(turn, 99))},
            "queue_wait_s": {"p50": float(np.percentile(wait, 50)), "p99": float(np.percentile(wait, 99))}}
