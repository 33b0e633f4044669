"""The device on the reference's own validation cases at the reference's own
step lengths (reference_cases.py): test/brownian (600 s steps, against the
sectional solver, 0.4) and test/bidisperse (1 s steps, the ODE, 0.3).  Every device run must meet the
reference test's tolerance, as each run of the reference does, and the mean
of 8 runs the tighter bound the oracle meets (test_oracle_sectional.py,
test_oracle_bidisperse.py), in FP64 and in MIXED mode."""
import numpy as np
import pytest

import partmc_b200 as pm
import reference_cases as RC
from oracle import exact as E

pytestmark = pytest.mark.gpu
MODES = {"fp64": pm.MODE_FP64, "mixed": pm.MODE_MIXED}


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("case,tol,tol_mean", [("brownian", 0.4, 0.15)])
def test_device_matches_the_sectional_solution(gpu_lib, case, tol, tol_mean, mode):
    sc = RC.BROWN if case == "brownian" else RC.SEDI
    per_run, mean = RC.sectional_errors(sc, RC.DeviceEngine, mode=MODES[mode])
    print(case, mode, "worst run", np.max(per_run, axis=0), "mean", mean)
    for e_num, e_mass in per_run:
        assert e_num < tol and e_mass < tol
    assert mean[0] < tol_mean and mean[1] < tol_mean


@pytest.mark.parametrize("mode", list(MODES))
def test_device_bidisperse_matches_the_ode(gpu_lib, mode):
    ode_n, ode_m = RC.bidisperse_ode()
    runs = [RC.bidisperse_run(31 + k, RC.DeviceEngine, mode=MODES[mode]) for k in range(8)]
    errs = [(E.rel_err_by_col(ode_n, n)[0], E.rel_err_by_col(ode_m, m)[0]) for n, m in runs]
    mean_n = np.mean([n for n, _ in runs], axis=0)
    mean_m = np.mean([m for _, m in runs], axis=0)
    mean = (E.rel_err_by_col(ode_n, mean_n)[0], E.rel_err_by_col(ode_m, mean_m)[0])
    print("bidisperse", mode, "worst run", np.max(errs, axis=0), "mean", mean)
    for e_n, e_m in errs:
        assert e_n < 0.3 and e_m < 0.3
    assert mean[0] < 0.03 and mean[1] < 0.03
