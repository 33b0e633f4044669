"""Ensembles over several ranks (the multi-GPU host logic), on CPU with gloo.

Two ranks each step their shard of independent populations; the stepper is
the oracle (standing in for a rank's GPU, which these tests do not need).
Whole-job counters and binned ensemble totals reduced over the two ranks must
equal those of one process stepping every population, because populations
are independent and each is seeded by its own seed."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from partmc_b200 import aero_dist
from partmc_b200 import ensemble as ens
from oracle import oracle as O

N_POP, N_STEPS, DEL_T = 5, 3, 600.0
EDGES = np.logspace(-9, -5, 41)


class OracleShard:
    """Stepper for Ensemble: one oracle per population (test stand-in for a GPU)."""

    def __init__(self, pops, temps, pressures, seeds, mode):
        self.pops, self.temps, self.pressures = pops, temps, pressures
        self.orcs = []
        for p, s in zip(pops, seeds):
            o = O.Oracle(p.aero_data.density, (p.awa.type, p.awa.magnitude, p.awa.exponent), seed=int(s))
            o.add_particles(p.vol, O.make_meta(p.n_part, group=p.group))
            o.set_next_id(p.n_part + 1)
            self.orcs.append(o)

    def step(self, kernel_type, del_t, n_steps):
        s = c = 0
        for _ in range(n_steps):
            for o, t, pr in zip(self.orcs, self.temps, self.pressures):
                a, b = o.mc_coag(kernel_type, float(t), float(pr), 0.0, del_t)
                s += a
                c += b
        return s, c

    def histogram(self, k, edges):
        vol = self.orcs[k].particles()[0]
        r = np.cbrt(3.0 * vol.sum(1) / (4.0 * np.pi))
        p = self.pops[k]
        return ens.binned_totals(vol, p.awa.num_conc_at_radius(1, r), edges, p.aero_data.density)


def problem():
    pops = [aero_dist.brown_bimodal(n, seed=40 + k) for k, n in enumerate((800, 3000, 1500, 2200, 600))]
    temps = np.linspace(270.0, 300.0, N_POP)
    press = np.linspace(8e4, 1e5, N_POP)
    seeds = np.arange(11, 11 + N_POP, dtype=np.uint64)
    return pops, temps, press, seeds


def problem_20spec(n_pop):
    """n_pop populations of 20 species (nummass weights), small."""
    pops = [aero_dist.brown_20spec(n, seed=60 + k) for k, n in enumerate((700, 900, 500)[:n_pop])]
    return pops, np.full(n_pop, 288.0), np.full(n_pop, 1e5), np.arange(21, 21 + n_pop, dtype=np.uint64)


def run_ensemble(rank, world, n_pop=N_POP):
    if n_pop == N_POP:
        pops, temps, press, seeds = problem()
    else:
        pops, temps, press, seeds = problem_20spec(n_pop)
    e = ens.Ensemble(pops, temps, press, seeds, rank=rank, world_size=world, stepper=OracleShard)
    s, c = e.step(O.KERNEL_BROWN, DEL_T, N_STEPS)
    tot = ens.reduce_counters(s, c, seconds=1.0 + rank)
    hist = ens.reduce_histograms(e.histogram(EDGES))
    return tot, hist, e.index


def _worker(rank, world, port, out_dir, n_pop=N_POP):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tot, hist, idx = run_ensemble(rank, world, n_pop)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), hist=hist, idx=np.array(idx),
                 tot=np.array([tot["n_samp"], tot["n_coag"], tot["seconds"]]))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_partitions_and_balances():
    n = [100, 5, 40, 40, 60, 1, 30]
    for w in (1, 2, 3, 7, 9):
        parts = ens.shard(n, w)
        assert sorted(i for p in parts for i in p) == list(range(len(n)))
        loads = [sum(n[i] for i in p) for p in parts]
        # greedy LPT: the most loaded rank exceeds the least by at most the largest job
        assert max(loads) - min(loads) <= max(n)
    assert ens.shard(n, 2) == ens.shard(n, 2)  # deterministic


def test_binned_totals_conserve():
    rng = np.random.default_rng(3)
    vol = rng.uniform(1e-24, 1e-21, size=(500, 3))
    nc = rng.uniform(1e8, 1e9, size=500)
    rho = np.array([1000.0, 1500.0, 2000.0])
    edges = np.logspace(-9, -5, 30)
    width = np.log(edges[-1] / edges[0]) / 29
    h = ens.binned_totals(vol, nc, edges, rho) * width  # per unit ln D, times the width
    assert np.isclose(h[:, 0].sum(), nc.sum())
    for s in range(3):
        assert np.isclose(h[:, 1 + s].sum(), (nc * vol[:, s] * rho[s]).sum())


def test_two_gloo_ranks_match_one_process():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, free_port(), d), nprocs=world, join=True, start_method="spawn")
        r = [np.load(os.path.join(d, f"rank{k}.npz")) for k in range(world)]
    # every population stepped exactly once across the ranks
    idx = sorted(np.concatenate([x["idx"] for x in r]).tolist())
    assert idx == list(range(N_POP))
    tot1, hist1, _ = run_ensemble(0, 1)
    for x in r:  # the reduced values are the same on every rank
        assert x["tot"][0] == tot1["n_samp"] and x["tot"][1] == tot1["n_coag"]
        assert x["tot"][2] == 2.0  # max over ranks of 1.0 + rank
        assert np.allclose(x["hist"], hist1, rtol=1e-12, atol=0.0)


def test_more_ranks_than_populations():
    """Three ranks, two populations of 20 species: the rank without a
    population still takes part in both reductions with histograms of the
    shared shape (number plus 20 species), and the sums equal one
    process's."""
    world, n_pop = 3, 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(world, free_port(), d, n_pop), nprocs=world, join=True,
                           start_method="spawn")
        r = [np.load(os.path.join(d, f"rank{k}.npz")) for k in range(world)]
    assert sorted(len(x["idx"]) for x in r) == [0, 1, 1]
    tot1, hist1, _ = run_ensemble(0, 1, n_pop)
    for x in r:
        assert x["hist"].shape == hist1.shape == (len(EDGES) - 1, 21)
        assert x["tot"][0] == tot1["n_samp"] and x["tot"][1] == tot1["n_coag"]
        assert np.allclose(x["hist"], hist1, rtol=1e-12, atol=0.0)
