"""The serving loop's host logic (partmc_b200/serve.py) on CPU: admission
into free population slots within the HBM budget, retirement after a job's
steps, and a full run over a job stream.  The batched device context and its
step are replaced by a stand-in that counts calls, so no GPU is needed; the
device side of serving is tested in test_gpu_serve.py."""
import numpy as np
import pytest

from partmc_b200 import serve
from partmc_b200 import coagulation as C


class FakeState:
    """Stands in for a batched AeroState: records what the server does to
    each population slot."""

    def __init__(self, aero_data, awa, mode=None, n_pop=1, seeds=None):
        self.n_pop = n_pop
        self.n_part = [0] * n_pop
        self.seed = list(seeds) if seeds is not None else [0] * n_pop
        self.steps = 0

    def add_particles(self, vol, group=None, pop=0):
        self.n_part[pop] = len(vol)

    def set_weight_pop(self, pop, awa):
        pass

    def set_next_id(self, next_id, pop=0):
        pass

    def set_seed(self, seed, pop=0):
        self.seed[pop] = seed

    def particles(self, pop=0):
        return {"n": self.n_part[pop]}


def fake_step(kernel, temps, pressures, coeff, st, del_t, n_steps=1):
    st.steps += 1
    return 10 * sum(1 for n in st.n_part if n), 1


@pytest.fixture
def fake_device(monkeypatch):
    monkeypatch.setattr(serve.C, "AeroState", FakeState)
    monkeypatch.setattr(serve.C, "mc_coag_batch", fake_step)


def job(jid, n_part, n_steps, kernel=C.COAG_KERNEL_TYPE_ADDITIVE, arrival=0.0):
    return serve.Job(jid, arrival, kernel, n_steps, serve.make_population(kernel, n_part, seed=jid + 1),
                     seed=100 + jid)


def test_admission_limited_by_slots(fake_device):
    s = serve.Server((C.COAG_KERNEL_TYPE_ADDITIVE,), slots=2, hbm_budget=1e15)
    jobs = [job(j, 200, 3) for j in range(3)]
    assert s.admit(jobs[0]) and s.admit(jobs[1])
    assert not s.admit(jobs[2])  # both slots taken
    st = s.ctx[C.COAG_KERNEL_TYPE_ADDITIVE]
    assert st.seed[:2] == [100, 101]  # each slot restarts its stream with the job's seed


def test_admission_limited_by_budget_and_freed_on_retirement(fake_device):
    j0, j1, j2 = job(0, 200, 2), job(1, 200, 5), job(2, 200, 1)
    per_job = j0.n_part * serve.BYTES_PER_PARTICLE
    s = serve.Server((C.COAG_KERNEL_TYPE_ADDITIVE,), slots=8, hbm_budget=2.5 * per_job)
    assert s.admit(j0) and s.admit(j1)
    assert not s.admit(j2)  # a third would exceed the budget
    done, _ = s.tick()
    assert done == []
    done, lat = s.tick()  # j0's second and last step
    assert done == [j0] and len(lat) == 1
    assert s.used == pytest.approx(j1.n_part * serve.BYTES_PER_PARTICLE)
    assert s.admit(j2)  # its slot and budget came back
    st = s.ctx[C.COAG_KERNEL_TYPE_ADDITIVE]
    assert st.n_part[s.jobs[C.COAG_KERNEL_TYPE_ADDITIVE].index(j2)] == j2.n_part


def test_contexts_per_kernel_step_only_when_holding_jobs(fake_device):
    kernels = (C.COAG_KERNEL_TYPE_ADDITIVE, C.COAG_KERNEL_TYPE_BROWN)
    s = serve.Server(kernels, slots=4, hbm_budget=1e15)
    assert s.admit(job(0, 150, 2, kernel=C.COAG_KERNEL_TYPE_BROWN))
    s.tick()
    assert s.ctx[C.COAG_KERNEL_TYPE_BROWN].steps == 1
    assert s.ctx[C.COAG_KERNEL_TYPE_ADDITIVE].steps == 0
    assert s.del_t[C.COAG_KERNEL_TYPE_BROWN] == serve.DEL_T[C.COAG_KERNEL_TYPE_BROWN]


def test_run_serves_every_job(fake_device):
    jobs = serve.poisson_jobs(12, rate=2000.0, seed=4, n_min=100, n_max=400, steps=(2, 5),
                              kernels=(C.COAG_KERNEL_TYPE_ADDITIVE, C.COAG_KERNEL_TYPE_SEDI))
    s = serve.Server((C.COAG_KERNEL_TYPE_ADDITIVE, C.COAG_KERNEL_TYPE_SEDI), slots=3, hbm_budget=1e15)
    m = serve.run(jobs, s)
    assert m["jobs"] == len(jobs)
    assert all(j.steps_done == j.n_steps for j in jobs)
    assert all(j.finish >= j.start >= j.arrival - 1e-9 for j in jobs)
    assert s.used == pytest.approx(0.0)
    assert all(x is None for slots in s.jobs.values() for x in slots)
    expected = sum(j.n_steps * serve.DEL_T[j.kernel] for j in jobs)
    assert m["sim_s_per_s"] * m["wall_s"] == pytest.approx(expected)
