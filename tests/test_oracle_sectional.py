"""The oracle against the reference's sectional solver (oracle/sectional.py,
run_sect.F90) on the reference's test/brownian and test/sedi (the settings
are in reference_cases.py).  Every run here stays within the test's
tolerance, and the mean of 8 runs within a tighter one.  CPU only."""
import math

import numpy as np

import reference_cases as RC


def test_sectional_solver_keeps_the_mass():
    """Bott's flux step moves mass between bins without creating or losing
    any while no coagulated particle leaves the grid."""
    num, mass = RC.sectional(RC.BROWN)
    width = math.log(RC.BROWN["d_max"] / RC.BROWN["d_min"]) / RC.BROWN["n_bin"]
    total = mass.sum(axis=1) * width
    assert np.allclose(total, total[0], rtol=1e-9)
    assert num[-1].sum() < 0.2 * num[0].sum()  # the number falls to about 11% in 24 h


def check(sc, tol, tol_mean):
    per_run, mean = RC.sectional_errors(sc)
    for e_num, e_mass in per_run:
        assert e_num < tol and e_mass < tol
    assert mean[0] < tol_mean and mean[1] < tol_mean


def test_brownian_matches_the_sectional_solution():
    """test_brownian_1.sh and _2.sh: 0.4 for number and mass, every hour."""
    check(RC.BROWN, 0.4, 0.15)


def test_sedi_matches_the_sectional_solution():
    """test_sedi_1.sh and _2.sh: 0.7 for number and mass at 0, 300 and 600 s."""
    check(RC.SEDI, 0.7, 0.4)
