"""Exact solutions and histogram metrics used to pin the oracle and the GPU path.

TEST INFRASTRUCTURE ONLY.

* ``soln_additive_exp``: coag_kernel_additive.F90:99-165 (Golovin kernel,
  exponential initial volume distribution).  I_1 is evaluated as
  scipy.special.i1e(x) * exp(x), folded into the exponent, which is exact for
  every x; the reference switches to the large-x asymptote above x = 500.
* ``soln_constant_exp``: coag_kernel_constant.F90:92-143, including the
  reference's lambda = 1 terms; ``soln_constant_coag`` is the same solution
  without them (pure coagulation), which is what a coagulation-only run
  follows.
* ``size_histogram``: extract_aero_size.F90:132-138 with
  bin_grid_histogram_1d (bin_grid.F90:225-248): number (or mass) per unit
  ln(D), weighted by each particle's number concentration.
* ``rel_err_by_col``: numeric_diff.F90:170-205 ``--by col`` with the 2-norm.
"""
import numpy as np
from scipy.special import i1e

PI = 3.14159265358979323846
BETA_0 = 0.25 / (60.0 * 2e8)


def rad2vol(r):
    return 4.0 * PI * np.asarray(r, dtype=np.float64) ** 3 / 3.0


def vol2rad(v):
    return (3.0 * np.asarray(v, dtype=np.float64) / 4.0 / PI) ** (1.0 / 3.0)


def log_grid(n_bin, dmin, dmax):
    """bin_grid_make (log): edges and centers (bin_grid.F90:83-134)."""
    edges = np.exp(np.linspace(np.log(dmin), np.log(dmax), n_bin + 1))
    edges[0], edges[-1] = dmin, dmax
    ln = np.linspace(np.log(dmin), np.log(dmax), 2 * n_bin + 1)
    centers = np.exp(ln[1::2])
    width = (np.log(dmax) - np.log(dmin)) / n_bin
    return edges, centers, width


def soln_additive_exp(centers_r, time, num_conc, radius_at_mean_vol, beta1):
    """Number distribution n(D) dlnD at radii ``centers_r`` (m^-3)."""
    mean_vol = rad2vol(radius_at_mean_vol)
    v = rad2vol(centers_r)
    d3 = (2.0 * np.asarray(centers_r)) ** 3
    if time == 0.0:
        return PI / 2.0 * d3 * num_conc / mean_vol * np.exp(-(v / mean_vol))
    tau = num_conc * mean_vol * beta1 * time
    T = 1.0 - np.exp(-tau)
    rat_v = v / mean_vol
    x = 2.0 * rat_v * np.sqrt(T)
    nn = num_conc / v * (1.0 - T) / np.sqrt(T) * np.exp(-((1.0 + T) * rat_v) + x) * i1e(x)
    return PI / 2.0 * d3 * nn


def soln_constant_exp(centers_r, time, num_conc, radius_at_mean_vol):
    mean_vol = rad2vol(radius_at_mean_vol)
    v = rad2vol(centers_r)
    d3 = (2.0 * np.asarray(centers_r)) ** 3
    if time == 0.0:
        return PI / 2.0 * d3 * num_conc / mean_vol * np.exp(-(v / mean_vol))
    lam = 1.0
    tau = num_conc * BETA_0 * time
    rat_v = v / mean_vol
    nn = 4.0 * num_conc / (mean_vol * (tau + 2.0) ** 2.0) * np.exp(
        -2.0 * rat_v / (tau + 2.0) * np.exp(-lam * tau) - lam * tau)
    return PI / 2.0 * d3 ** 1.0 * nn


def soln_constant_coag(centers_r, time, num_conc, radius_at_mean_vol):
    """Pure constant-kernel coagulation from an exponential initial volume
    distribution: n(v, t) = N0 / v_mu * 4 / (tau + 2)^2 * exp(-2 v / (v_mu (tau + 2)))
    with tau = N0 beta_0 t (Smoluchowski's solution; the reference's
    soln_constant_exp adds lambda = 1 loss terms to it)."""
    mean_vol = rad2vol(radius_at_mean_vol)
    v = rad2vol(centers_r)
    d3 = (2.0 * np.asarray(centers_r)) ** 3
    tau = num_conc * BETA_0 * time
    nn = 4.0 * num_conc / (mean_vol * (tau + 2.0) ** 2) * np.exp(-2.0 * (v / mean_vol) / (tau + 2.0))
    return PI / 2.0 * d3 * nn


def size_histogram(diameters, weights, n_bin=160, dmin=1e-8, dmax=1e-3):
    """Histogram per unit ln D over a log diameter grid."""
    edges, centers, width = log_grid(n_bin, dmin, dmax)
    d = np.asarray(diameters, dtype=np.float64)
    lo, hi = np.log(dmin), np.log(dmax)
    with np.errstate(divide="ignore"):
        x = np.log(d)
    idx = np.floor((x - lo) / (hi - lo) * n_bin).astype(np.int64) + 1
    idx = np.where(x == hi, n_bin, idx)
    ok = (idx >= 1) & (idx <= n_bin)
    h = np.bincount(idx[ok] - 1, weights=np.asarray(weights)[ok], minlength=n_bin) / width
    return h, centers


def rel_err_by_col(exact, approx):
    exact = np.atleast_2d(np.asarray(exact, dtype=np.float64))
    approx = np.atleast_2d(np.asarray(approx, dtype=np.float64))
    diff = exact - approx
    return np.sqrt((diff ** 2).sum(axis=-1)) / np.sqrt((exact ** 2).sum(axis=-1))
