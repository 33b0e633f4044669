"""The oracle against the reference's sectional solver (oracle/sectional.py,
run_sect.F90) on the reference's test/brownian: one log-normal mode
(1e11 m^-3, geometric mean diameter 50 nm, log10 of the geometric standard
deviation 0.24, water density), the Brownian kernel at 288 K and 1e5 Pa,
24 hours.  Particle runs: 1000 particles under number-and-mass weighting
(AERO_STATE_WEIGHT_NUMMASS_SOURCE, run_part's choice when the spec file
selects none, run_part.F90:561-562), 600 s steps,
rebalanced after every step as run_part does (run_part.F90:982); sectional
run: 220 bins of diameter
from 1e-10 to 1e-4 m, 60 s steps (test/brownian/run_part.spec, run_sect.spec).
test_brownian_1.sh and _2.sh accept a relative 2-norm error of 0.4 for the
number and the mass distributions at every output hour (numeric_diff --by
col --rel-tol 0.4); every run here stays within it, and the mean of 8 runs
within 0.15.  CPU only."""
import math

import numpy as np

from oracle import exact as E
from oracle import ic_sampler as S
from oracle import oracle as O
from oracle import sectional as SC

RHO, N_TOTAL, R_GEOM, LOG10_SIGMA = 1000.0, 1e11, 2.5e-8, 0.24
N_BIN, D_MIN, D_MAX = 220, 1e-10, 1e-4


def sectional():
    times, centers, num = SC.run(O.KERNEL_BROWN, RHO, N_TOTAL, R_GEOM, LOG10_SIGMA, N_BIN, D_MIN, D_MAX, 60.0,
                                 86400.0, 3600.0)
    return num, num * E.rad2vol(centers) * RHO


ALPHAS = (0.0, -3.0)  # number and mass weighting: two groups, exponents 0 and -3


def particle_run(k, n_part=1000):
    """One particle run, half the particles in each weight group; each
    particle counts at the groups' harmonic number concentration at its
    radius (aero_weight_array_num_conc_at_radius)."""
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=R_GEOM, log10_std=LOG10_SIGMA, num_conc=N_TOTAL)
    ws = [S.Weight(S.WEIGHT_POWER, S.mode_number(mode, S.Weight(S.WEIGHT_POWER, 1.0, a)) / (n_part / 2), a)
          for a in ALPHAS]
    vols, grp, _ = S.add_dist_sample(np.random.default_rng(100 + k), [mode], ws, 1.0)
    orc = O.Oracle([RHO], ([[O.WEIGHT_POWER], [O.WEIGHT_POWER]], [[ws[0].magnitude], [ws[1].magnitude]],
                           [[ALPHAS[0]], [ALPHAS[1]]]), seed=7 + k)
    orc.add_particles(vols, O.make_meta(len(vols), group=grp + 1))
    orc.set_next_id(len(vols) + 1)
    num, mass = [], []
    for step in range(0, 145):
        if step > 0:
            orc.mc_coag(O.KERNEL_BROWN, 288.0, 1e5, 0.0, 600.0)
            orc.rebalance(n_part / 2)
        if step % 6 == 0:
            v = orc.particles()[0].sum(1)
            mags = orc.weight_magnitudes()[:, 0]
            r = E.vol2rad(v)
            nc = 1.0 / sum(1.0 / (mags[g] * r ** ALPHAS[g]) for g in range(len(ALPHAS)))
            num.append(E.size_histogram(2.0 * r, nc, N_BIN, D_MIN, D_MAX)[0])
            mass.append(E.size_histogram(2.0 * r, nc * v * RHO, N_BIN, D_MIN, D_MAX)[0])
    return np.array(num), np.array(mass)


def test_sectional_solver_keeps_the_mass():
    """Bott's flux step moves mass between bins without creating or losing
    any while no coagulated particle leaves the grid."""
    num, mass = sectional()
    width = math.log(D_MAX / D_MIN) / N_BIN
    total = mass.sum(axis=1) * width
    assert np.allclose(total, total[0], rtol=1e-9)
    assert num[-1].sum() < 0.2 * num[0].sum()  # the number falls to about 11% in 24 h


def test_brownian_matches_the_sectional_solution():
    sect_num, sect_mass = sectional()
    runs = [particle_run(k) for k in range(8)]
    for num, mass in runs:
        assert max(E.rel_err_by_col(sect_num[t], num[t])[0] for t in range(25)) < 0.4
        assert max(E.rel_err_by_col(sect_mass[t], mass[t])[0] for t in range(25)) < 0.4
    mean_num = np.mean([r[0] for r in runs], axis=0)
    mean_mass = np.mean([r[1] for r in runs], axis=0)
    assert max(E.rel_err_by_col(sect_num[t], mean_num[t])[0] for t in range(25)) < 0.15
    assert max(E.rel_err_by_col(sect_mass[t], mean_mass[t])[0] for t in range(25)) < 0.15
