"""The redraw rounds run as one device-driven CUDA graph or from a host loop;
both launch the same kernels on the same device state, so the particles must
agree bit for bit after several steps with many conflicts."""
import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import aero_dist

pytestmark = pytest.mark.gpu


def run(pop, mode, graphs, n_steps, del_t):
    st = pm.AeroState(pop.aero_data, pop.awa, seed=21, mode=mode)
    st.set_graphs(graphs)
    st.add_particles(pop.vol, pop.group)
    env = pm.EnvState(288.0, 1e5)
    rounds, tot = [], 0
    for _ in range(n_steps):
        s, k = pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, del_t)
        tot += k
        rounds.append(st.stats()["rounds"])
    return st.particles(components=True), rounds, tot


@pytest.mark.parametrize("mode", [pm.MODE_FP64, pm.MODE_MIXED])
def test_graph_matches_host_loop(gpu_lib, mode):
    # the benchmark's 20-species population at a tenth of its size: several
    # redraw rounds per step
    pop = aero_dist.brown_20spec(100000, seed=12)
    a, ra, ka = run(pop, mode, True, 5, 60.0)
    b, rb, kb = run(pop, mode, False, 5, 60.0)
    assert ra == rb and ka == kb, (ra, rb)
    assert max(ra) >= 3, ra  # the graph ran more than one redraw round
    for key in a:
        assert np.array_equal(a[key], b[key]), key


def test_graph_matches_host_loop_batched(gpu_lib):
    pops, temps, press = aero_dist.batched_bimodal(n_pop=3, seed=5, n_min=5e3, n_max=2e4)
    out = []
    for graphs in (True, False):
        st = pm.AeroState(pops[0].aero_data, pops[0].awa, n_pop=3, seeds=np.array([3, 4, 5], dtype=np.uint64))
        st.set_graphs(graphs)
        for k, p in enumerate(pops):
            st.set_weight_pop(k, p.awa)
            st.add_particles(p.vol, p.group, pop=k)
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, st, 600.0, n_steps=4)
        out.append([st.particles(pop=k) for k in range(3)])
    for k in range(3):
        for key in out[0][k]:
            assert np.array_equal(out[0][k][key], out[1][k][key]), (k, key)
