"""Binned diagnostics on the device (pmc_coag_gpu_size_dist) against the same
histograms computed on the host from a full download (bin_grid_histogram_1d,
bin_grid.F90:225-248, as extract_aero_size.F90:132-138 uses it), and the
ensemble on one GPU rank."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist
from partmc_b200 import ensemble as ens

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
