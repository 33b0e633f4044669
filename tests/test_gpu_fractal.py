"""Fractal (non-spherical) particles on the device, through the C ABI.

1. Static parity with the oracle under three particle shapes: the kernel
   values of every kernel (FP64, 1e-12 relative; the Brownian and
   sedimentation kernels through the fractal mobility radius of
   fractal.F90:315-362), every particle's bin and the bin counts (exact,
   radii from fractal_vol2rad; the grid edges to 1e-14), and the k_max
   table (1e-12).
2. The reference's own test/fractal cases (test_fractal_2.sh, _3.sh): the
   device runs both through the package API and must meet the reference's
   criterion against the reference's golden vectors, numeric_diff --by col
   --rel-tol 0.1, in FP64 and in MIXED mode, for every seed tried.
"""
import os

import numpy as np
import pytest

import fractal_case as fc
import partmc_b200 as pm
from partmc_b200 import aero_dist
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REF = np.load(os.path.join(os.path.dirname(__file__), "golden", "fractal_ref.npz"))
SHAPES = {
    "free_df2.4": (2.4, 5e-10, 1.0),  # test/fractal's free molecular case
    "cont_df1.8": (1.8, 2.5e-7, 1.0),  # test/fractal's continuum case
    "df2.0_fill1.43": (2.0, 1e-8, 1.43),  # a filling factor as in test_fractal_radii_conversion
}
KERNELS = [pm.COAG_KERNEL_TYPE_ADDITIVE, pm.COAG_KERNEL_TYPE_CONSTANT, pm.COAG_KERNEL_TYPE_BROWN,
           pm.COAG_KERNEL_TYPE_SEDI, pm.COAG_KERNEL_TYPE_BROWN_FREE, pm.COAG_KERNEL_TYPE_BROWN_CONT]
ENV = pm.EnvState(300.0, 1e5, 1000.0)


def shaped(pop, shape):
    """pop with aero_data of the given fractal shape (same volumes)."""
    df, r0, f = SHAPES[shape]
    data = pm.AeroData(pop.aero_data.density, fractal=pm.Fractal(df, r0, f))
    return data


def oracle_for(pop, shape):
    o = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent))
    o.set_fractal(*SHAPES[shape])
    return o


def population(kt):
    if kt == pm.COAG_KERNEL_TYPE_SEDI:
        return aero_dist.additive_exp(3000, seed=5, radius_at_mean_vol=1e-5)
    return aero_dist.brown_bimodal(3000, seed=3)


@pytest.mark.parametrize("shape", list(SHAPES))
@pytest.mark.parametrize("kt", KERNELS)
def test_fractal_kernel_values_fp64(gpu_lib, shape, kt):
    pop = population(kt)
    st = pm.AeroState(shaped(pop, shape), pop.awa)
    orc = oracle_for(pop, shape)
    rng = np.random.default_rng(kt)
    i = rng.integers(0, pop.n_part, 256)
    j = rng.integers(0, pop.n_part, 256)
    k_gpu = st.eval_kernel(kt, ENV, pop.vol[i], 1, pop.vol[j], 1, 1)
    k_cpu = np.array([orc.weighted_kernel(kt, pop.vol[a], 1, pop.vol[b], 1, 1, ENV.temp, ENV.pressure,
                                          ENV.additive_kernel_coefficient) for a, b in zip(i, j)])
    ok = k_cpu != 0
    assert ok.sum() > 200
    rel = np.abs(k_gpu[ok] - k_cpu[ok]) / np.abs(k_cpu[ok])
    assert rel.max() < 1e-12, rel.max()


@pytest.mark.parametrize("shape", list(SHAPES))
def test_fractal_bins_bit_exact(gpu_lib, shape):
    pop = aero_dist.brown_20spec(4000, seed=4)
    st = pm.AeroState(shaped(pop, shape), pop.awa)
    st.add_particles(pop.vol, pop.group)
    edges, counts, bins = st.sort()
    orc = oracle_for(pop, shape)
    orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
    orc.sort()
    # the grid comes from the extreme radii, which the device computes with
    # CUDA's pow and the oracle with the C library's: the edges may differ in
    # the last bit; counts and bins are exact
    assert np.allclose(edges, orc.bin_edges(), rtol=1e-14, atol=0.0)
    assert np.array_equal(counts, orc.bin_counts())
    assert np.array_equal(bins, orc.particle_bins())
    # the grid spans the fractal radii, not the spheres' (d_f < 3 spreads them)
    sph = pm.AeroState(pop.aero_data, pop.awa)
    sph.add_particles(pop.vol, pop.group)
    assert not np.array_equal(sph.sort()[0], edges)


@pytest.mark.parametrize("shape", list(SHAPES))
@pytest.mark.parametrize("kt", [pm.COAG_KERNEL_TYPE_BROWN, pm.COAG_KERNEL_TYPE_BROWN_FREE,
                                pm.COAG_KERNEL_TYPE_BROWN_CONT, pm.COAG_KERNEL_TYPE_SEDI])
def test_fractal_kmax_table(gpu_lib, shape, kt):
    pop = population(kt)
    st = pm.AeroState(shaped(pop, shape), pop.awa)
    st.add_particles(pop.vol, pop.group)
    edges, _, _ = st.sort()
    nb = len(edges) - 1
    k_gpu = st.kmax_table(kt, ENV)[: nb * nb].reshape(nb, nb, order="F")
    orc = oracle_for(pop, shape)
    orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
    orc.sort()
    _, k_cpu = orc.kmax_table(kt, ENV.temp, ENV.pressure, ENV.additive_kernel_coefficient)
    # clusters whose mobility radius exceeds 3.5 mm all fall at the capped
    # terminal speed (fall_g), so their sedimentation kernel is 0 in both
    nz = k_cpu != 0
    assert np.array_equal(k_gpu[~nz], k_cpu[~nz])
    # the sedimentation kernel's |w1 - w2| cancels where both speeds are near
    # the cap: there the error is measured against a thousandth of the
    # table's largest value instead of the entry.  The fractal mobility
    # radius is the root of a sum of nearly cancelling terms (Newton,
    # fractal.F90:315-362), so the device's fused multiply-adds and the C
    # library's separate roundings differ by more than in the spherical
    # kernels: 1e-10 where the radius enters (Brownian, sedimentation)
    scale = np.maximum(np.abs(k_cpu[nz]), 1e-3 * np.abs(k_cpu).max())
    rel = np.abs(k_gpu[nz] - k_cpu[nz]) / scale
    tol = 1e-10 if kt in (pm.COAG_KERNEL_TYPE_BROWN, pm.COAG_KERNEL_TYPE_SEDI) else 1e-12
    assert rel.max() < tol, rel.max()


def test_set_fractal_rejects_the_reference_stops(gpu_lib):
    pop = aero_dist.brown_bimodal(100, seed=1)
    st = pm.AeroState(pop.aero_data, pop.awa)
    for bad in ((3.2, 1e-8, 1.0), (2.0, 0.0, 1.0), (2.0, 1e-8, -1.0)):
        with pytest.raises(pm.PmcError):
            st.set_fractal(pm.Fractal(*bad))


@pytest.mark.parametrize("case", ["free", "cont"])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_device_passes_reference_fractal_case(gpu_lib, case, mode):
    """test_fractal_2.sh / test_fractal_3.sh on the device: 750 steps of
    10,000 particles with rebalancing, against the reference's golden
    vectors at the reference's tolerance, for three seeds."""
    m = pm.MODE_FP64 if mode == "fp64" else pm.MODE_MIXED
    for seed in (1, 2, 3):
        rows = fc.run(case, fc.device_stepper(case, seed, m))
        err = fc.rel_err_by_col(REF[case], rows)
        print(case, mode, seed, err)
        assert (err < fc.REL_TOL).all(), (seed, err)
