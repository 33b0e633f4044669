"""Generate the replay fixtures: small populations run through the CPU
oracle with its uniform stream dumped, so that the device replay mode can be
checked bit for bit (particles in the reference's swap-last order, ids,
counters, uniforms consumed).

    python tests/golden/make_replay_golden.py

Writes tests/golden/replay_<case>.npz.  The populations come from
partmc_b200.aero_dist; the uniform stream is the oracle's xoshiro256**
stream (the reference's own generator cannot run here).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from partmc_b200 import aero_dist  # noqa: E402

CASES = {
    # name: (population, kernel, temp, pressure, coeff, del_t, steps, seed)
    "additive_flat": (lambda: aero_dist.additive_exp(300, seed=21), O.KERNEL_ADDITIVE, 288.0, 1e5, 1000.0, 5.0, 6, 101),
    "brown_power": (lambda: aero_dist.brown_bimodal(500, seed=22), O.KERNEL_BROWN, 288.0, 1e5, 0.0, 3600.0, 5, 102),
    "brown_nummass_20spec": (lambda: aero_dist.brown_20spec(300, seed=23, num_concs=(2e11, 2e10, 2e9)),
                             O.KERNEL_BROWN, 280.0, 9e4, 0.0, 300.0, 2, 103),
    "sedi_flat": (lambda: aero_dist.additive_exp(300, seed=24, num_conc=1e8, radius_at_mean_vol=2e-5),
                  O.KERNEL_SEDI, 288.0, 1e5, 0.0, 5.0, 5, 104),
    "constant_power": (lambda: aero_dist.brown_bimodal(300, seed=25), O.KERNEL_CONSTANT, 288.0, 1e5, 0.0, 1.0, 5,
                       105),
}


def run_case(name):
    mk, kt, temp, press, coeff, del_t, steps, seed = CASES[name]
    pop = mk()
    n = pop.n_part
    ids = np.arange(1, n + 1, dtype=np.int64)
    orc = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=seed)
    orc.add_particles(pop.vol, O.make_meta(n, group=pop.group, ids=ids))
    orc.set_next_id(n + 1)
    orc.enable_dump(1 << 20)
    counters = []
    for _ in range(steps):
        counters.append(orc.mc_coag(kt, temp, press, coeff, del_t))
    vol, meta = orc.particles()
    return dict(
        density=pop.aero_data.density, w_type=pop.awa.type, w_mag=pop.awa.magnitude, w_exp=pop.awa.exponent,
        vol0=pop.vol, group0=pop.group, id0=ids, kernel=kt, temp=temp, pressure=press, coeff=coeff, del_t=del_t,
        steps=steps, uniforms=orc.dump(), counters=np.array(counters, dtype=np.int64), vol=vol,
        weight_group=meta["weight_group"], weight_class=meta["weight_class"], id=meta["id"],
        n_primary_parts=meta["n_primary_parts"], n_comp=meta["n_comp"], comp_source=meta["comp_source"],
        comp_create_time=meta["comp_create_time"], next_id=orc.next_id())


def main():
    for name in CASES:
        d = run_case(name)
        path = os.path.join(HERE, f"replay_{name}.npz")
        np.savez_compressed(path, **d)
        print(name, "particles", len(d["vol0"]), "->", len(d["vol"]), "uniforms", len(d["uniforms"]),
              "counters", d["counters"].tolist(), os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
