"""Parity of the CUDA path with the CPU oracle, through the C ABI.

Bit-exact: bin grid, per-particle bins and per-cell counts.  1e-12 relative:
FP64 kernel values (num_conc_weighted_kernel) and the k_max table.  FP32 mode:
kernel values within 2e-5 relative."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ENV = pm.EnvState(288.0, 1e5, 1000.0)
KERNELS = [pm.COAG_KERNEL_TYPE_ADDITIVE, pm.COAG_KERNEL_TYPE_CONSTANT, pm.COAG_KERNEL_TYPE_BROWN,
           pm.COAG_KERNEL_TYPE_SEDI, pm.COAG_KERNEL_TYPE_BROWN_FREE, pm.COAG_KERNEL_TYPE_BROWN_CONT]


def populations():
    return {
        "additive_flat": aero_dist.additive_exp(3000, seed=2),
        "brown_power": aero_dist.brown_bimodal(4000, seed=3),
        "brown_20spec_nummass": aero_dist.brown_20spec(4000, seed=4),
    }


def oracle_for(pop, seed=1):
    return O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=seed)


@pytest.mark.parametrize("name", ["additive_flat", "brown_power", "brown_20spec_nummass"])
@pytest.mark.parametrize("kt", KERNELS)
def test_kernel_values_fp64(gpu_lib, name, kt):
    pop = populations()[name]
    if kt == pm.COAG_KERNEL_TYPE_SEDI:
        # the Hall table covers drops up to mm size; use cloud-drop sizes
        pop = aero_dist.additive_exp(3000, seed=5, radius_at_mean_vol=1e-5)
    st = pm.AeroState(pop.aero_data, pop.awa)
    orc = oracle_for(pop)
    rng = np.random.default_rng(kt)
    i = rng.integers(0, pop.n_part, 256)
    j = rng.integers(0, pop.n_part, 256)
    ng = pop.awa.n_class
    k_gpu = st.eval_kernel(kt, ENV, pop.vol[i], 1, pop.vol[j], 1, 1)
    k_cpu = np.array([orc.weighted_kernel(kt, pop.vol[a], 1, pop.vol[b], 1, 1, ENV.temp, ENV.pressure,
                                          ENV.additive_kernel_coefficient) for a, b in zip(i, j)])
    assert ng == 1
    ok = k_cpu != 0
    rel = np.abs(k_gpu[ok] - k_cpu[ok]) / np.abs(k_cpu[ok])
    assert rel.max() < 1e-12, rel.max()
    st.set_mode(pm.MODE_MIXED)
    k32 = st.eval_kernel(kt, ENV, pop.vol[i], 1, pop.vol[j], 1, 1)
    rel32 = np.abs(k32[ok] - k_cpu[ok]) / np.abs(k_cpu[ok])
    assert rel32.max() < 2e-5, rel32.max()


@pytest.mark.parametrize("name", ["additive_flat", "brown_power", "brown_20spec_nummass"])
def test_bins_bit_exact(gpu_lib, name):
    pop = populations()[name]
    st = pm.AeroState(pop.aero_data, pop.awa)
    st.add_particles(pop.vol, pop.group)
    edges, counts, bins = st.sort()
    orc = oracle_for(pop)
    orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
    orc.sort()
    assert np.array_equal(edges, orc.bin_edges())
    assert np.array_equal(counts, orc.bin_counts())
    assert np.array_equal(bins, orc.particle_bins())


@pytest.mark.parametrize("kt", KERNELS)
def test_kmax_table(gpu_lib, kt):
    pop = aero_dist.brown_20spec(3000, seed=9) if kt != pm.COAG_KERNEL_TYPE_SEDI else aero_dist.additive_exp(3000)
    st = pm.AeroState(pop.aero_data, pop.awa)
    st.add_particles(pop.vol, pop.group)
    edges, _, _ = st.sort()
    nb = len(edges) - 1
    kt_gpu = st.kmax_table(kt, ENV)[: nb * nb].reshape(nb, nb, order="F")
    orc = oracle_for(pop)
    orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
    orc.sort()
    _, kt_cpu = orc.kmax_table(kt, ENV.temp, ENV.pressure, ENV.additive_kernel_coefficient)
    rel = np.abs(kt_gpu - kt_cpu) / np.abs(kt_cpu)
    assert rel.max() < 1e-12, rel.max()


def test_upload_download_round_trip(gpu_lib):
    pop = aero_dist.brown_20spec(5000, seed=1)
    st = pm.AeroState(pop.aero_data, pop.awa)
    ids = np.arange(100, 100 + pop.n_part)
    st.add_particles(pop.vol, pop.group, ids=ids, n_primary_parts=3)
    p = st.particles()
    assert np.array_equal(p["vol"], pop.vol)
    assert np.array_equal(p["weight_group"], pop.group)
    assert np.array_equal(p["id"], ids)
    assert (p["n_primary_parts"] == 3).all()
    assert st.next_id() == 100 + pop.n_part
