"""The oracle against the reference's sectional solver (oracle/sectional.py,
run_sect.F90) on the reference's test/brownian and test/sedi.  Particle
runs: 1000 particles under number-and-mass weighting
(AERO_STATE_WEIGHT_NUMMASS_SOURCE, run_part's choice when the spec file
selects none, run_part.F90:561-562), rebalanced after every step as run_part
does (run_part.F90:982).  The settings of each test are its run_part.spec,
run_sect.spec and initial distribution:
  * test/brownian: one log-normal mode (1e11 m^-3, geometric mean diameter
    50 nm, log10 of the geometric standard deviation 0.24), Brownian kernel
    at 288 K and 1e5 Pa, 24 h; particles at 600 s steps, sections (220 bins
    of diameter 1e-10 to 1e-4 m) at 60 s; the test accepts a relative 2-norm
    error of 0.4 for the number and mass distributions at every hour;
  * test/sedi: one log-normal mode (1e9 m^-3, 20 um, 0.2), sedimentation
    kernel, 600 s; particles at 5 s steps, sections (100 bins of 1e-7 to
    1 m) at 1 s; the test accepts 0.7 at 0, 300 and 600 s.
Every run here stays within the test's tolerance, and the mean of 8 runs
within a tighter one.  CPU only."""
import math

import numpy as np

from oracle import exact as E
from oracle import ic_sampler as S
from oracle import oracle as O
from oracle import sectional as SC

RHO = 1000.0
ALPHAS = (0.0, -3.0)  # number and mass weighting: two groups, exponents 0 and -3

# test/brownian and test/sedi: run_part.spec, run_sect.spec, aero_init_dist*.dat
BROWN = dict(kernel=O.KERNEL_BROWN, num_conc=1e11, r_geom=2.5e-8, log10_sigma=0.24, n_bin=220, d_min=1e-10,
             d_max=1e-4, sect_dt=60.0, part_dt=600.0, t_max=86400.0, t_out=3600.0)
SEDI = dict(kernel=O.KERNEL_SEDI, num_conc=1e9, r_geom=1e-5, log10_sigma=0.2, n_bin=100, d_min=1e-7, d_max=1.0,
            sect_dt=1.0, part_dt=5.0, t_max=600.0, t_out=300.0)


def sectional(sc):
    times, centers, num = SC.run(sc["kernel"], RHO, sc["num_conc"], sc["r_geom"], sc["log10_sigma"], sc["n_bin"],
                                 sc["d_min"], sc["d_max"], sc["sect_dt"], sc["t_max"], sc["t_out"])
    return num, num * E.rad2vol(centers) * RHO


def particle_run(sc, k, n_part=1000):
    """One particle run, half the particles in each weight group; each
    particle counts at the groups' harmonic number concentration at its
    radius (aero_weight_array_num_conc_at_radius)."""
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=sc["r_geom"], log10_std=sc["log10_sigma"], num_conc=sc["num_conc"])
    ws = [S.Weight(S.WEIGHT_POWER, S.mode_number(mode, S.Weight(S.WEIGHT_POWER, 1.0, a)) / (n_part / 2), a)
          for a in ALPHAS]
    vols, grp, _ = S.add_dist_sample(np.random.default_rng(100 + k), [mode], ws, 1.0)
    orc = O.Oracle([RHO], ([[O.WEIGHT_POWER], [O.WEIGHT_POWER]], [[ws[0].magnitude], [ws[1].magnitude]],
                           [[ALPHAS[0]], [ALPHAS[1]]]), seed=7 + k)
    orc.add_particles(vols, O.make_meta(len(vols), group=grp + 1))
    orc.set_next_id(len(vols) + 1)
    n_steps = int(round(sc["t_max"] / sc["part_dt"]))
    every = int(round(sc["t_out"] / sc["part_dt"]))
    num, mass = [], []
    for step in range(0, n_steps + 1):
        if step > 0:
            orc.mc_coag(sc["kernel"], 288.0, 1e5, 0.0, sc["part_dt"])
            orc.rebalance(n_part / 2)
        if step % every == 0:
            v = orc.particles()[0].sum(1)
            mags = orc.weight_magnitudes()[:, 0]
            r = E.vol2rad(v)
            nc = 1.0 / sum(1.0 / (mags[g] * r ** ALPHAS[g]) for g in range(len(ALPHAS)))
            h = lambda wt: E.size_histogram(2.0 * r, wt, sc["n_bin"], sc["d_min"], sc["d_max"])[0]
            num.append(h(nc))
            mass.append(h(nc * v * RHO))
    return np.array(num), np.array(mass)


def max_err(ref, approx):
    return max(E.rel_err_by_col(ref[t], approx[t])[0] for t in range(len(ref)))


def test_sectional_solver_keeps_the_mass():
    """Bott's flux step moves mass between bins without creating or losing
    any while no coagulated particle leaves the grid."""
    num, mass = sectional(BROWN)
    width = math.log(BROWN["d_max"] / BROWN["d_min"]) / BROWN["n_bin"]
    total = mass.sum(axis=1) * width
    assert np.allclose(total, total[0], rtol=1e-9)
    assert num[-1].sum() < 0.2 * num[0].sum()  # the number falls to about 11% in 24 h


def check(sc, tol, tol_mean, n_runs=8):
    sect_num, sect_mass = sectional(sc)
    runs = [particle_run(sc, k) for k in range(n_runs)]
    for num, mass in runs:
        assert max_err(sect_num, num) < tol
        assert max_err(sect_mass, mass) < tol
    assert max_err(sect_num, np.mean([r[0] for r in runs], axis=0)) < tol_mean
    assert max_err(sect_mass, np.mean([r[1] for r in runs], axis=0)) < tol_mean


def test_brownian_matches_the_sectional_solution():
    """test_brownian_1.sh and _2.sh: 0.4 for number and mass, every hour."""
    check(BROWN, 0.4, 0.15)


def test_sedi_matches_the_sectional_solution():
    """test_sedi_1.sh and _2.sh: 0.7 for number and mass at 0, 300 and 600 s."""
    check(SEDI, 0.7, 0.4)
