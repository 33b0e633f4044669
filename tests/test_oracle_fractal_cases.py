"""The oracle on the reference's own test/fractal cases, against the
reference's golden vectors (tests/golden/fractal_ref.npz, copied from
test/fractal/ref_*_dimless_time_regrid.txt by make_fractal_golden.py), with
the reference's own criterion: numeric_diff --by col --rel-tol 0.1 on the
dimensionless time and N / N0 columns (test_fractal_2.sh:18,
test_fractal_3.sh:18).  One run per seed, like the reference's test.  CPU."""
import os

import numpy as np
import pytest

import fractal_case as fc

REF = np.load(os.path.join(os.path.dirname(__file__), "golden", "fractal_ref.npz"))


@pytest.mark.parametrize("case", ["free", "cont"])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_passes_reference_fractal_case(case, seed):
    rows = fc.run(case, fc.oracle_stepper(case, seed))
    err = fc.rel_err_by_col(REF[case], rows)
    print(case, seed, err)
    assert (err < fc.REL_TOL).all(), err
