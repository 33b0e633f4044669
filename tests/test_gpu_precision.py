"""MIXED precision against FP64 on the device, through the C ABI.

MIXED mode evaluates the pair tests' kernels in FP32 and decides a test in
FP64 whenever the FP32 acceptance probability lies within a margin (2^-12)
of the uniform, or near or above k_max.  The margin bounds the FP32 rounding
error, so every accept decision is the FP64 mode's for the same draws, and
with k_max, the merges and the sums in FP64 in both modes, a MIXED run must
reproduce the FP64 run particle for particle.  These tests check that on the
benchmark's workload classes and record the FP32 kernel error per workload:
  - 20 species with nummass weights, Brownian, 60 s steps (the 1e6-particle
    benchmark workload, in miniature);
  - the bimodal Brownian population with power weights (alpha = -1), 600 s
    steps (enough tests at 1e5 particles for the FP64 fallback to occur);
  - the additive kernel with flat weights at test/additive's 1 s steps;
  - the sedimentation kernel with flat weights at test/sedi's 5 s steps."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist

pytestmark = pytest.mark.gpu

MARGIN = 2.0 ** -12


def workloads():
    sedi = aero_dist.additive_exp(6000, seed=15, radius_at_mean_vol=1e-5)
    return {
        "brown_20spec_nummass": (aero_dist.brown_20spec(20000, seed=11), pm.COAG_KERNEL_TYPE_BROWN,
                                 pm.EnvState(288.0, 1e5), 60.0, 6),
        "brown_bimodal_power": (aero_dist.brown_bimodal(100000, seed=12), pm.COAG_KERNEL_TYPE_BROWN,
                                pm.EnvState(288.0, 1e5), 600.0, 10),
        "additive_flat": (aero_dist.additive_exp(10000, seed=13), pm.COAG_KERNEL_TYPE_ADDITIVE,
                          pm.EnvState(288.0, 1e5, 1000.0), 1.0, 20),
        "sedi_flat": (sedi, pm.COAG_KERNEL_TYPE_SEDI, pm.EnvState(288.0, 1e5), 5.0, 12),
    }


def run(pop, kt, env, del_t, n_steps, mode):
    st = pm.AeroState(pop.aero_data, pop.awa, seed=77, mode=mode)
    st.add_particles(pop.vol, pop.group)
    counts = [pm.mc_coag(kt, env, pop.aero_data, st, del_t) for _ in range(n_steps)]
    return st, counts, st.particles()


@pytest.mark.parametrize("name", list(workloads()))
def test_mixed_reproduces_fp64_particle_for_particle(gpu_lib, name):
    pop, kt, env, del_t, n_steps = workloads()[name]
    _, c64, p64 = run(pop, kt, env, del_t, n_steps, pm.MODE_FP64)
    st32, c32, p32 = run(pop, kt, env, del_t, n_steps, pm.MODE_MIXED)
    assert c32 == c64
    assert sum(c for _, c in c64) > 0
    for key in ("vol", "id", "weight_group", "n_primary_parts"):
        assert np.array_equal(p32[key], p64[key]), key
    # the FP64 fallback was exercised and stayed rare (about 2 * margin of
    # the tests, plus tests near k_max)
    n_tests = sum(s for s, _ in c32)
    n_exact = st32.exact_tests()
    print(f"{name}: {n_tests} tests, {n_exact} decided in FP64 ({n_exact / max(n_tests, 1):.2e})")
    assert n_exact < 0.05 * n_tests
    if n_tests > 20000:  # expected about 10 or more: the fallback must have run
        assert n_exact > 0


@pytest.mark.parametrize("name", list(workloads()))
def test_fp32_kernel_error_far_inside_the_margin(gpu_lib, name):
    """The FP32 weighted kernel against the FP64 one over random pairs of the
    workload's particles: the largest error on the acceptance scale is stated
    and must stay below a quarter of the margin.  The scale is the kernel
    itself where every term is positive (Brownian, additive); for the
    sedimentation kernel, whose |w1 - w2| cancels for drops of one size, it
    is the bin pair's k_max, which is what the acceptance divides by."""
    pop, kt, env, _, _ = workloads()[name]
    st = pm.AeroState(pop.aero_data, pop.awa, mode=pm.MODE_FP64)
    rng = np.random.default_rng(3)
    i = rng.integers(0, pop.n_part, 20000)
    j = rng.integers(0, pop.n_part, 20000)
    k64 = st.eval_kernel(kt, env, pop.vol[i], 1, pop.vol[j], 1, 1)
    st.set_mode(pm.MODE_MIXED)
    k32 = st.eval_kernel(kt, env, pop.vol[i], 1, pop.vol[j], 1, 1)
    if kt == pm.COAG_KERNEL_TYPE_SEDI:
        st.add_particles(pop.vol, pop.group)
        edges, _, bins = st.sort()
        nb = len(edges) - 1
        tab = st.kmax_table(kt, env)[: nb * nb].reshape(nb, nb, order="F")
        b1, b2 = np.minimum(bins[i], bins[j]) - 1, np.maximum(bins[i], bins[j]) - 1
        scale = tab[b1, b2] * float(pop.awa.magnitude[0, 0])  # flat weights: k times the number concentration
    else:
        scale = k64
    ok = scale > 0
    err = np.abs(k32[ok] - k64[ok]) / scale[ok]
    print(f"{name}: FP32 kernel max error {err.max():.3e} of its scale over {ok.sum()} pairs")
    assert err.max() < MARGIN / 4
