"""The device against the oracle on the benchmark set's own configurations,
through the C ABI: ensembles of independent runs, compared per size bin.

  - the 20-species benchmark workload in miniature: per-particle Dirichlet(1)
    mass fractions over 20 species of densities U(1000, 2000), three
    log-normal modes, nummass weights, the Brownian kernel at 288 K, 60 s
    steps; 20,000 particles, 16 runs, FP64 and MIXED;
  - the bimodal Brownian population with power weights (alpha = -1) at 288 K
    for 24 h of 60 s steps; 5000 particles, 16 runs (one batched context on
    the device);
  - the additive kernel's exact solution with 1e4 particles, 1 s steps to
    600 s, is in test_gpu_rebalance.py.

Each run of the device and of the oracle has its own seed.  Per bin, the
ensemble means of the number and of each species' mass must agree within
4.5 standard errors of their difference (about 300 bins per configuration:
the family-wise false-alarm rate is under 0.2%), and the totals within 3.
The device results are deterministic for fixed seeds, so a pass is
repeatable."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist
from oracle import exact as E
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_RUNS = 16
Z_BIN, Z_TOT = 4.5, 3.0


def histograms(vol, awa, density, n_bin=30, dmin=5e-9, dmax=5e-6):
    """Number and per-species mass per unit ln D of one population."""
    r = E.vol2rad(vol.sum(1))
    nc = awa.num_conc_at_radius(1, r)
    out = [E.size_histogram(2 * r, nc, n_bin=n_bin, dmin=dmin, dmax=dmax)[0]]
    for s in range(vol.shape[1]):
        out.append(E.size_histogram(2 * r, nc * vol[:, s] * density[s], n_bin=n_bin, dmin=dmin, dmax=dmax)[0])
    return np.array(out)  # (1 + n_spec, n_bin)


def compare(dev, orc, label):
    """z-scores of the ensemble means, per bin and for the totals."""
    g, c = np.array(dev), np.array(orc)  # (runs, 1 + n_spec, n_bin)
    n = len(g)
    se = np.sqrt(g.var(0, ddof=1) / n + c.var(0, ddof=1) / n)
    ok = se > 0
    z = np.abs(g.mean(0) - c.mean(0))[ok] / se[ok]
    tg, tc = g.sum(2), c.sum(2)  # totals per moment
    se_t = np.sqrt(tg.var(0, ddof=1) / n + tc.var(0, ddof=1) / n)
    zt = np.abs(tg.mean(0) - tc.mean(0)) / np.maximum(se_t, 1e-300)
    print(f"{label}: {ok.sum()} bins, max |z| {z.max():.2f}; totals max |z| {zt.max():.2f}")
    assert z.max() < Z_BIN, (label, z.max())
    assert zt.max() < Z_TOT, (label, zt.max())


def oracle_run(pop, seed):
    o = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=seed)
    o.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
    o.set_next_id(pop.n_part + 1)
    return o


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_20spec_nummass_brownian_matches_oracle(gpu_lib, mode):
    n_part, n_steps, del_t = 20000, 10, 60.0
    m = pm.MODE_FP64 if mode == "fp64" else pm.MODE_MIXED
    dev, orc = [], []
    env = pm.EnvState(288.0, 1e5)
    for k in range(N_RUNS):
        pop = aero_dist.brown_20spec(n_part, seed=500 + k)
        st = pm.AeroState(pop.aero_data, pop.awa, seed=600 + k, mode=m)
        st.add_particles(pop.vol, pop.group)
        o = oracle_run(pop, 700 + k)
        for _ in range(n_steps):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, del_t)
            o.mc_coag(O.KERNEL_BROWN, 288.0, 1e5, 0.0, del_t)
        dev.append(histograms(st.particles()["vol"], pop.awa, pop.aero_data.density))
        orc.append(histograms(o.particles()[0], pop.awa, pop.aero_data.density))
    compare(dev, orc, f"20spec nummass {mode}")


def test_bimodal_power_24h_matches_oracle(gpu_lib):
    n_part, del_t = 5000, 60.0
    checks = {360: [], 720: [], 1440: []}  # steps: 6 h, 12 h, 24 h
    pops = [aero_dist.brown_bimodal(n_part, seed=800 + k) for k in range(N_RUNS)]
    st = pm.AeroState(pops[0].aero_data, pops[0].awa, mode=pm.MODE_FP64, n_pop=N_RUNS,
                      seeds=np.arange(900, 900 + N_RUNS, dtype=np.uint64))
    for k, p in enumerate(pops):
        st.set_weight_pop(k, p.awa)
        st.add_particles(p.vol, p.group, pop=k)
    orcs = [oracle_run(p, 1000 + k) for k, p in enumerate(pops)]
    dev = {s: [] for s in checks}
    orc = {s: [] for s in checks}
    for step in range(1, 1441):
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, 288.0, 1e5, 0.0, st, del_t)
        for o in orcs:
            o.mc_coag(O.KERNEL_BROWN, 288.0, 1e5, 0.0, del_t)
        if step in checks:
            for k, p in enumerate(pops):
                dev[step].append(histograms(st.particles(pop=k)["vol"], p.awa, p.aero_data.density))
                orc[step].append(histograms(orcs[k].particles()[0], p.awa, p.aero_data.density))
    for s in checks:
        compare(dev[s], orc[s], f"bimodal power {s * del_t / 3600:.0f} h")
