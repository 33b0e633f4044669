"""Device replay mode: one GPU thread runs mc_coag in the reference's order on
the stored uniform stream and must reproduce the oracle's particle list bit
for bit (volumes, order, ids, groups, components) and its counters."""
import glob
import os

import numpy as np
import pytest

import partmc_b200 as pm

pytestmark = pytest.mark.gpu

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "replay_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[7:-4] for p in GOLD])
def test_gpu_replay_bit_exact(gpu_lib, path):
    g = np.load(path)
    ad = pm.AeroData(g["density"])
    awa = pm.AeroWeightArray(g["w_type"], g["w_mag"], g["w_exp"])
    st = pm.AeroState(ad, awa, mode=pm.MODE_REPLAY)
    st.add_particles(g["vol0"], g["group0"], ids=g["id0"])
    st.set_next_id(len(g["vol0"]) + 1)
    st.set_replay(g["uniforms"])
    env = pm.EnvState(float(g["temp"]), float(g["pressure"]), float(g["coeff"]))
    counters = [pm.mc_coag(int(g["kernel"]), env, ad, st, float(g["del_t"])) for _ in range(int(g["steps"]))]
    assert np.array_equal(np.array(counters), g["counters"]), counters
    assert st.replay_used() == len(g["uniforms"])
    p = st.particles(components=True)
    assert np.array_equal(p["vol"], g["vol"])
    for k in ("weight_group", "weight_class", "id", "n_primary_parts", "n_comp"):
        assert np.array_equal(p[k], g[k]), k
    nc = g["n_comp"]
    for i in range(len(nc)):
        assert np.array_equal(p["comp_source"][i, :nc[i]], g["comp_source"][i, :nc[i]])
    assert st.next_id() == int(g["next_id"])


def test_replay_stream_exhaustion_is_an_error(gpu_lib):
    g = np.load(GOLD[0])
    ad = pm.AeroData(g["density"])
    st = pm.AeroState(ad, pm.AeroWeightArray(g["w_type"], g["w_mag"], g["w_exp"]), mode=pm.MODE_REPLAY)
    st.add_particles(g["vol0"], g["group0"], ids=g["id0"])
    st.set_replay(g["uniforms"][:10])
    env = pm.EnvState(float(g["temp"]), float(g["pressure"]), float(g["coeff"]))
    with pytest.raises(pm.PmcError) as e:
        for _ in range(int(g["steps"])):
            pm.mc_coag(int(g["kernel"]), env, ad, st, float(g["del_t"]))
    assert e.value.code == 6  # PMC_ERR_RNG_EXHAUSTED
