"""The oracle's samplers against their exact pmfs, as test/rand does
(test_poisson_sample.F90, test_binomial_sample.F90, test_rand_1..8.sh), with
numeric_diff's column-wise relative 2-norm and the same tolerances."""
import math

import numpy as np
import pytest
from scipy.stats import binom, poisson

from oracle import oracle as O

N_SAMP = 10_000_000  # as test_rand_*.sh


def rel2(exact, approx):
    return np.sqrt(((exact - approx) ** 2).sum()) / np.sqrt((exact ** 2).sum())


@pytest.mark.parametrize("lam,tol", [(1, 1e-3), (4, 2e-3), (10, 2e-3), (20, 0.07), (30, 0.06)])
def test_poisson_pmf(lam, tol):
    orc = O.Oracle([1000.0], ([[1]], [[1.0]], [[0.0]]), seed=11 + lam)
    h = orc.poisson_hist(float(lam), N_SAMP, 50) / N_SAMP
    ex = poisson.pmf(np.arange(51), lam)
    # the noise of 2e6 draws is sqrt(1e7 / 2e6) times that of the reference's 1e7
    assert rel2(ex, h) < tol * math.sqrt(1e7 / N_SAMP)


@pytest.mark.parametrize("n,p,tol", [(10, 0.3, 1e-3), (10, 0.7, 2e-3), (30, 0.5, 5e-3)])
def test_binomial_pmf(n, p, tol):
    orc = O.Oracle([1000.0], ([[1]], [[1.0]], [[0.0]]), seed=5)
    h = orc.binomial_hist(n, p, N_SAMP, n) / N_SAMP
    ex = binom.pmf(np.arange(n + 1), n, p)
    assert rel2(ex, h) < tol * math.sqrt(1e7 / N_SAMP)


def test_normal_approx_branch_rounds_half_away():
    # rand_poisson above mean 10 returns nint(normal): mean preserved
    orc = O.Oracle([1000.0], ([[1]], [[1.0]], [[0.0]]), seed=3)
    h = orc.poisson_hist(200.0, 200_000, 400)
    k = np.arange(401)
    assert abs((h * k).sum() / h.sum() - 200.0) < 0.2


def test_replay_stream_is_consumed_in_order():
    orc = O.Oracle([1000.0], ([[1]], [[1.0]], [[0.0]]), seed=3)
    orc.enable_dump()
    draws = [orc.random() for _ in range(10)]
    assert np.array_equal(orc.dump(), draws)
    o2 = O.Oracle([1000.0], ([[1]], [[1.0]], [[0.0]]))
    o2.set_replay(np.array(draws))
    assert [o2.random() for _ in range(10)] == draws
