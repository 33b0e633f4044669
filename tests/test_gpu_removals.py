"""Removal records (aero_info_array) from the device, through the C ABI.

1. Replay mode against the oracle on the golden replay fixtures: the same
   uniform stream gives the same records in the same order (ID, action,
   other ID), record for record.
2. The parallel step: every particle ID present before a step, or handed
   out during it, is present after it or removed with exactly one record,
   and every record's other_id names a particle (removal_check.py), for flat
   weights (additive), power weights with the per-particle path, nummass
   weights with 20 species, the sedimentation kernel's chains, and a
   halving (aero_state_halve records its removals)."""
import glob
import os

import numpy as np
import pytest

import partmc_b200 as pm
import removal_check as RCK
from partmc_b200 import aero_dist
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "replay_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[7:-4] for p in GOLD])
def test_replay_removal_records_match_the_oracle(gpu_lib, path):
    g = np.load(path)
    ad = pm.AeroData(g["density"])
    awa = pm.AeroWeightArray(g["w_type"], g["w_mag"], g["w_exp"])
    st = pm.AeroState(ad, awa, mode=pm.MODE_REPLAY)
    st.add_particles(g["vol0"], g["group0"], ids=g["id0"])
    st.set_next_id(len(g["vol0"]) + 1)
    st.set_replay(g["uniforms"])
    st.set_record_removals(True)
    o = O.Oracle(g["density"], (g["w_type"], g["w_mag"], g["w_exp"]))
    o.add_particles(g["vol0"], O.make_meta(len(g["vol0"]), group=g["group0"], ids=g["id0"]))
    o.set_next_id(len(g["vol0"]) + 1)
    o.set_replay(g["uniforms"])
    o.set_record_removals(True)
    env = pm.EnvState(float(g["temp"]), float(g["pressure"]), float(g["coeff"]))
    n_rec = 0
    for _ in range(int(g["steps"])):
        pm.mc_coag(int(g["kernel"]), env, ad, st, float(g["del_t"]))
        o.mc_coag(int(g["kernel"]), float(g["temp"]), float(g["pressure"]), float(g["coeff"]), float(g["del_t"]))
        dev, orc = st.removals(), o.removals()
        n_rec += len(orc["id"])
        for k in ("id", "action", "other_id"):
            assert np.array_equal(dev[k], orc[k]), k
    assert n_rec > 0


def workloads():
    pp = aero_dist.brown_bimodal(20000, seed=4, modes=[(1e11, 0.005e-6, np.log10(1.5)), (1e8, 0.25e-6, np.log10(1.5))])
    sedi = aero_dist.additive_exp(5000, seed=24, num_conc=1e8, radius_at_mean_vol=2e-5)
    return {
        "additive_flat": (aero_dist.additive_exp(20000, seed=3), pm.COAG_KERNEL_TYPE_ADDITIVE, 60.0),
        "brown_power_per_particle": (pp, pm.COAG_KERNEL_TYPE_BROWN, 600.0),
        "brown_20spec_nummass": (aero_dist.brown_20spec(20000, seed=5), pm.COAG_KERNEL_TYPE_BROWN, 600.0),
        "sedi_flat_chains": (sedi, pm.COAG_KERNEL_TYPE_SEDI, 5.0),
    }


@pytest.mark.parametrize("name", list(workloads()))
def test_removal_records_account_for_every_id(gpu_lib, name):
    pop, kt, dt = workloads()[name]
    st = pm.AeroState(pop.aero_data, pop.awa, seed=12, mode=pm.MODE_MIXED)
    st.add_particles(pop.vol, pop.group, ids=np.arange(1, pop.n_part + 1))
    st.set_next_id(pop.n_part + 1)
    st.set_record_removals(True)
    env = pm.EnvState(288.0, 1e5, 1000.0)
    n_rec = 0
    for _ in range(4):
        ids0, nid0 = st.particles()["id"].copy(), st.next_id()
        pm.mc_coag(kt, env, pop.aero_data, st, dt)
        rec = st.removals()
        RCK.check_id_accounting(ids0, nid0, st.next_id(), st.particles()["id"], rec)
        n_rec += len(rec["id"])
    assert n_rec > 0
    # halving: every removal recorded as HALVED
    ids0, nid0 = st.particles()["id"].copy(), st.next_id()
    st.rebalance(st.n_part() / 8.0, allow_doubling=False)
    rec = st.removals()
    assert len(rec["id"]) > 0 and (rec["action"] == RCK.INFO_HALVED).all()
    RCK.check_id_accounting(ids0, nid0, st.next_id(), st.particles()["id"], rec)


def test_removals_off_by_default_and_buffer_too_small(gpu_lib):
    pop = aero_dist.additive_exp(5000, seed=8)
    st = pm.AeroState(pop.aero_data, pop.awa, seed=3)
    st.add_particles(pop.vol, pop.group)
    env = pm.EnvState(288.0, 1e5, 1000.0)
    pm.mc_coag(pm.COAG_KERNEL_TYPE_ADDITIVE, env, pop.aero_data, st, 60.0)
    assert len(st.removals()["id"]) == 0
    st.set_record_removals(True)
    pm.mc_coag(pm.COAG_KERNEL_TYPE_ADDITIVE, env, pop.aero_data, st, 60.0)
    with pytest.raises(pm.PmcError):
        st.removals(max_n=1)  # too small: nothing copied or cleared
    assert len(st.removals()["id"]) > 1
