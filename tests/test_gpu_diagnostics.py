"""Binned diagnostics on the device (pmc_coag_gpu_size_dist) against the
oracle's restatement of extract_aero_size (oracle/exact.py size_histogram:
bin_grid_histogram_1d, bin_grid.F90:225-248, as extract_aero_size.F90:132-138
uses it) and against the package's host histogram of a full download, and
the ensemble on one GPU rank."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist
from partmc_b200 import ensemble as ens
from oracle import exact as E

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["brown_20spec", "brown_bimodal"])
def test_size_dist_matches_host_histogram(gpu_lib, name):
    pop = aero_dist.brown_20spec(20000, seed=3) if name == "brown_20spec" else aero_dist.brown_bimodal(20000, seed=3)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=2)
    st.add_particles(pop.vol, pop.group)
    pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, pm.EnvState(288.0, 1e5), pop.aero_data, st, 600.0)
    edges = np.logspace(-9, -5, 81)
    for _ in range(2):  # two calls in a row give the same sums up to rounding order
        num, mass = st.size_dist(80, edges[0], edges[-1])
        p = st.particles()
        r = np.cbrt(3.0 * p["vol"].sum(1) / (4.0 * np.pi))
        # the number concentration of each particle (aero_state_num_concs)
        nc = pop.awa.num_conc_at_radius(1, r)
        ref = ens.binned_totals(p["vol"], nc, edges, pop.aero_data.density)
        assert np.allclose(num, ref[:, 0], rtol=1e-12, atol=0.0)
        assert np.allclose(mass, ref[:, 1:], rtol=1e-12, atol=1e-300)
        assert num.sum() > 0


@pytest.mark.parametrize("n_bin,dmin,dmax", [(160, 1e-8, 1e-3), (50, 2e-9, 2e-6)])
def test_size_dist_matches_the_extract_aero_size_oracle(gpu_lib, n_bin, dmin, dmax):
    """Number and per-species mass distributions of a stepped 20-species
    nummass population against size_histogram, the oracle's restatement of
    extract_aero_size --num / --mass (per unit ln D, each particle at its
    number concentration), on test/weighting's grid (160 bins, 10 nm to
    1 mm) and on a grid that cuts the population at both ends."""
    pop = aero_dist.brown_20spec(30000, seed=8)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=4)
    st.add_particles(pop.vol, pop.group)
    for _ in range(3):
        pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, pm.EnvState(288.0, 1e5), pop.aero_data, st, 60.0)
    num, mass = st.size_dist(n_bin, dmin, dmax)
    p = st.particles()
    d = 2.0 * E.vol2rad(p["vol"].sum(1))
    nc = pop.awa.num_conc_at_radius(1, d / 2.0)
    ref_num, _ = E.size_histogram(d, nc, n_bin=n_bin, dmin=dmin, dmax=dmax)
    assert np.allclose(num, ref_num, rtol=1e-12, atol=0.0)
    for s_ in range(pop.aero_data.n_spec):
        ref_m, _ = E.size_histogram(d, nc * p["vol"][:, s_] * pop.aero_data.density[s_], n_bin=n_bin, dmin=dmin,
                                    dmax=dmax)
        assert np.allclose(mass[:, s_], ref_m, rtol=1e-12, atol=1e-300), s_
    assert num.sum() > 0


def test_ensemble_on_one_gpu(gpu_lib):
    pops = [aero_dist.brown_bimodal(n, seed=60 + k) for k, n in enumerate((3000, 5000, 2000))]
    e = ens.Ensemble(pops, [288.0] * 3, [1e5] * 3, [7, 8, 9], rank=0, world_size=1)
    s, c = e.step(pm.COAG_KERNEL_TYPE_BROWN, 600.0, 3)
    assert s >= c > 0
    edges = np.logspace(-9, -5, 41)
    h = e.histogram(edges)
    total = 0.0
    for k, p in enumerate(e.pops):
        out = e.engine.st.particles(pop=k)
        r = np.cbrt(3.0 * out["vol"].sum(1) / (4.0 * np.pi))
        total += ens.binned_totals(out["vol"], p.awa.num_conc_at_radius(1, r), edges, p.aero_data.density)
    assert np.allclose(h, total, rtol=1e-12, atol=1e-300)
