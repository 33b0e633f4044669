"""The launch-shape autotuner (pmc_coag_gpu_autotune): the search runs on the
caller's own steps, so a context that tunes must give the particles of one
that does not, bit for bit; the search ends with one of each site's
candidates and a score for every candidate."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist

pytestmark = pytest.mark.gpu

N_SEARCH = 5 * 3 * 3  # sites x candidates x steps per candidate
CANDS = {"test": (64, 128, 256), "resolve": (64, 128, 256), "items": (64, 128, 256), "chain": (32, 64, 128),
         "apply": (64, 128, 256)}


def same(a, b):
    for key in ("vol", "id", "weight_group", "weight_class", "n_primary_parts"):
        assert np.array_equal(a[key], b[key]), key


@pytest.mark.parametrize("mode", [pm.MODE_FP64, pm.MODE_MIXED])
def test_tuning_steps_give_the_untuned_particles(gpu_lib, mode):
    pop = aero_dist.brown_20spec(20000, seed=12)
    env = pm.EnvState(288.0, 1e5)
    out = []
    for tune in (False, True):
        st = pm.AeroState(pop.aero_data, pop.awa, seed=33, mode=mode)
        st.add_particles(pop.vol, pop.group)
        if tune:
            st.autotune()
        counts = [pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, 60.0) for _ in range(N_SEARCH + 2)]
        out.append((counts, st.particles(), st.tune_state()))
    (c0, p0, s0), (c1, p1, s1) = out
    assert c0 == c1 and sum(c for _, c in c0) > 0
    same(p0, p1)
    tuning, threads, ms = s1
    assert not tuning
    for site, t in threads.items():
        assert t in CANDS[site]
        assert all(m >= 0 for m in ms[site]), site
        assert ms[site][CANDS[site].index(t)] == min(ms[site])
    assert all(m > 0 for m in ms["test"] + ms["items"])
    assert s0[1] == {"test": 256, "resolve": 256, "items": 256, "chain": 128, "apply": 256}


def test_batched_tuning_and_set_tune(gpu_lib):
    pops = [aero_dist.brown_bimodal(n, seed=40 + k) for k, n in enumerate((3000, 8000, 1000, 5000))]
    out = []
    for how in ("default", "tuned", "set"):
        st = pm.AeroState(pops[0].aero_data, pops[0].awa, mode=pm.MODE_FP64, n_pop=4,
                          seeds=np.arange(70, 74, dtype=np.uint64))
        for k, p in enumerate(pops):
            st.set_weight_pop(k, p.awa)
            st.add_particles(p.vol, p.group, pop=k)
        if how == "tuned":
            st.autotune()
        if how == "set":
            st.set_tune({"test": 64, "resolve": 128, "items": 64, "chain": 32, "apply": 128})
            with pytest.raises(pm.PmcError):
                st.set_tune({"chain": 256})
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, 288.0, 1e5, 0.0, st, 600.0, n_steps=N_SEARCH + 1)
        out.append([st.particles(pop=k) for k in range(4)])
    for k in range(4):
        same(out[0][k], out[1][k])
        same(out[0][k], out[2][k])
