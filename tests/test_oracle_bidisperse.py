"""The oracle against the reference's test/bidisperse (settings in
reference_cases.py): the reference's test accepts a relative 2-norm error
of 0.3 per series (numeric_diff --by col --rel-tol 0.3); every run here
stays within it, and the mean of 8 runs within 0.03.  CPU only."""
import numpy as np

import reference_cases as RC
from oracle import exact as E


def test_bidisperse_matches_the_ode():
    ode_n, ode_m = RC.bidisperse_ode()
    runs = [RC.bidisperse_run(31 + k) for k in range(8)]
    for n, m in runs:
        assert E.rel_err_by_col(ode_n, n)[0] < 0.3
        assert E.rel_err_by_col(ode_m, m)[0] < 0.3
    mean_n = np.mean([n for n, _ in runs], axis=0)
    mean_m = np.mean([m for _, m in runs], axis=0)
    assert E.rel_err_by_col(ode_n, mean_n)[0] < 0.03
    assert E.rel_err_by_col(ode_m, mean_m)[0] < 0.03
