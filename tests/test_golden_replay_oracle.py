"""The oracle, driven by the stored uniform streams, reproduces the stored
replay fixtures exactly (tests/golden/make_replay_golden.py made them)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "replay_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[7:-4] for p in GOLD])
def test_oracle_reproduces_fixture(path):
    g = np.load(path)
    n = len(g["vol0"])
    orc = O.Oracle(g["density"], (g["w_type"], g["w_mag"], g["w_exp"]))
    orc.add_particles(g["vol0"], O.make_meta(n, group=g["group0"], ids=g["id0"]))
    orc.set_next_id(n + 1)
    orc.set_replay(g["uniforms"])
    counters = [orc.mc_coag(int(g["kernel"]), float(g["temp"]), float(g["pressure"]), float(g["coeff"]),
                            float(g["del_t"])) for _ in range(int(g["steps"]))]
    assert np.array_equal(np.array(counters), g["counters"])
    assert orc.uniforms_used() == len(g["uniforms"])
    vol, meta = orc.particles()
    assert np.array_equal(vol, g["vol"])
    for k in ("weight_group", "weight_class", "id", "n_primary_parts", "n_comp"):
        assert np.array_equal(meta[k], g[k]), k
    assert np.array_equal(meta["comp_source"], g["comp_source"])
    assert orc.check() == 0
