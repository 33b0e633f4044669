"""Ensembles of independent populations over several GPUs.

A single population of PartMC's particle-resolved model does not shard: its
coagulation step couples every particle pair of the population.  Independent
populations (ensemble members of one scenario, or the cells of a column
model) do: each rank steps a shard of them with no exchange during the step.
One process drives one GPU (torch.distributed, NCCL on GPUs, gloo on CPU).

  shard(n_parts, world_size)       populations to ranks, balanced by particles
  Ensemble(...)                    this rank's shard as one batched context
  reduce_counters(...)             whole-job pair tests / events / time
  reduce_histograms(...)           ensemble sums of binned number and volume

The binned sums are the quantities PartMC's ensemble post-processing averages
(aero_state_num_conc / aero_state_masses per bin, aero_state.F90:987-1022),
reduced across ranks with one all_reduce per output time.
"""
import numpy as np


def shard(n_parts, world_size):
    """Assign populations to ranks, largest first, each to the rank with the
    fewest particles so far (ties: lowest rank).  Deterministic; returns one
    sorted list of population indices per rank."""
    n_parts = [int(n) for n in n_parts]
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    load = [0] * world_size
    out = [[] for _ in range(world_size)]
    for i in sorted(range(len(n_parts)), key=lambda i: (-n_parts[i], i)):
        r = min(range(world_size), key=lambda r: (load[r], r))
        out[r].append(i)
        load[r] += n_parts[i]
    return [sorted(x) for x in out]


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def reduce_counters(n_samp, n_coag, seconds, device="cpu"):
    """Whole-job counters: pair tests and events summed over ranks, time as
    the slowest rank's.  Without a process group the local values return."""
    dist = _dist()
    if dist is None:
        return {"n_samp": int(n_samp), "n_coag": int(n_coag), "seconds": float(seconds)}
    import torch
    work = torch.tensor([float(n_samp), float(n_coag)], dtype=torch.float64, device=device)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(work, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return {"n_samp": int(work[0].item()), "n_coag": int(work[1].item()), "seconds": float(t.item())}


def binned_totals(vol, num_conc, edges, density):
    """Number and per-species mass distributions of one population per unit
    ln(D) on the diameter grid `edges` (n_bin + 1, log-spaced), as
    bin_grid_histogram_1d (bin_grid.F90:225-248) weights them: vol (n_part,
    n_spec) m^3, num_conc (n_part,) m^-3, density (n_spec,) kg m^-3.
    Returns an (n_bin, 1 + n_spec) array (number, then species masses).  The
    GPU shard computes the same on the device (pmc_coag_gpu_size_dist)."""
    vol = np.asarray(vol, dtype=np.float64)
    if vol.ndim == 1:
        vol = vol[:, None]
    n_bin = len(edges) - 1
    width = (np.log(edges[-1]) - np.log(edges[0])) / n_bin
    d = 2.0 * np.cbrt(3.0 * vol.sum(1) / (4.0 * np.pi))
    k = np.floor((np.log(d) - np.log(edges[0])) / (np.log(edges[-1]) - np.log(edges[0])) * n_bin).astype(np.int64)
    ok = (k >= 0) & (k < n_bin)
    out = np.zeros((n_bin, 1 + vol.shape[1]))
    np.add.at(out[:, 0], k[ok], num_conc[ok] / width)
    for s in range(vol.shape[1]):
        np.add.at(out[:, 1 + s], k[ok], num_conc[ok] * vol[ok, s] * density[s] / width)
    return out


def reduce_histograms(hist, device="cpu"):
    """Sum binned totals over ranks (one all_reduce)."""
    dist = _dist()
    if dist is None:
        return np.asarray(hist, dtype=np.float64)
    import torch
    t = torch.as_tensor(np.asarray(hist, dtype=np.float64), device=device).clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def _n_spec(populations):
    """Species count shared by every population of an ensemble (taken from
    aero_data, which all members share)."""
    counts = {int(len(p.aero_data.density)) for p in populations}
    if len(counts) != 1:
        raise ValueError("ensemble members must share one aero_data (species count)")
    return counts.pop()


class Ensemble:
    """This rank's shard of independent populations, stepped together.

    populations: list of objects with .vol, .group, .awa, .aero_data (as made
    by partmc_b200.aero_dist); temps, pressures, seeds: per population.  The
    default stepper is a batched AeroState on this rank's GPU; `stepper` can
    replace it (a callable factory taking the shard's populations, their
    temperatures, pressures and seeds, and returning an object with
    step(kernel_type, del_t, n_steps) -> (n_samp, n_coag) and
    histogram(k, edges) -> binned_totals of population k)."""

    def __init__(self, populations, temps, pressures, seeds, rank=0, world_size=1, mode=None, stepper=None):
        self.index = shard([p.vol.shape[0] for p in populations], world_size)[rank]
        self.pops = [populations[i] for i in self.index]
        # species count from the whole ensemble, not this rank's shard: a rank
        # with no populations still returns histograms of the shared shape,
        # so every rank's all_reduce in reduce_histograms matches
        self.n_spec = _n_spec(populations)
        t = np.asarray(temps, dtype=np.float64)[self.index]
        p = np.asarray(pressures, dtype=np.float64)[self.index]
        s = np.asarray(seeds, dtype=np.uint64)[self.index]
        if stepper is None:
            stepper = _GpuShard
        self.engine = stepper(self.pops, t, p, s, mode) if self.pops else None

    def step(self, kernel_type, del_t, n_steps=1):
        if self.engine is None:
            return 0, 0
        return self.engine.step(kernel_type, del_t, n_steps)

    def histogram(self, edges):
        """Size distributions (binned_totals layout) summed over this rank's
        populations."""
        out = np.zeros((len(edges) - 1, 1 + self.n_spec))
        for k in range(len(self.pops)):
            out += self.engine.histogram(k, edges)
        return out


class _GpuShard:
    """A shard as one batched context on the current GPU."""

    def __init__(self, pops, temps, pressures, seeds, mode):
        from . import coagulation as C
        self.C = C
        self.temps, self.pressures = temps, pressures
        self.pops = pops
        self.st = C.AeroState(pops[0].aero_data, pops[0].awa, mode=C.MODE_MIXED if mode is None else mode,
                              n_pop=len(pops), seeds=seeds)
        for k, p in enumerate(pops):
            self.st.set_weight_pop(k, p.awa)
            self.st.add_particles(p.vol, p.group, pop=k)

    def step(self, kernel_type, del_t, n_steps):
        return self.C.mc_coag_batch(kernel_type, self.temps, self.pressures, 0.0, self.st, del_t, n_steps=n_steps)

    def histogram(self, k, edges):
        """On the device, without a download (log-spaced edges)."""
        num, mass = self.st.size_dist(len(edges) - 1, edges[0], edges[-1], pop=k)
        return np.concatenate([num[:, None], mass], axis=1)
