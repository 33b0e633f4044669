"""The reference's sectional coagulation solver, restated for the CPU.

TEST INFRASTRUCTURE ONLY: a second, independent solution of the coagulation
equation, which the reference's own tests (test/brownian, test/sedi) compare
particle runs with.

Follows run_sect.F90: one species on a log radius grid
(bin_grid_make, bin_grid.F90:83-134), the initial log-normal mode binned at
the bin centres (num_conc_log_normal and vol_conc_log_normal,
aero_mode.F90:131-188), the kernel at the bin centres (bin_kernel,
coag_kernel.F90:216-246) smoothed with half the self-rate
(smooth_bin_kernel, run_sect.F90:414-444), the Courant numbers and
destination bins (courant, run_sect.F90:364-409), and Bott's exponential flux
step (coad, run_sect.F90:283-359, in C as orc_sect_coad), with the
reference's unit conversions (radii in um, masses in mg, the kernel in
cm^3/s times del_t and the bin width).
"""
import ctypes
import math

import numpy as np

from . import exact as E
from . import oracle as O


def _coad():
    f = O.lib().orc_sect_coad
    f.restype = None
    f.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5
    return f


def courant(e, log_width):
    """courant, run_sect.F90:364-409, 0-based (ima -1: the sum goes nowhere).
    The reference tests c(i,j) before setting it, when it is still 0, so the
    lower of the two neighbouring bins is always taken."""
    n = len(e)
    c = np.zeros((n, n))
    ima = np.full((n, n), -1, dtype=np.int32)
    for i in range(n):
        for j in range(i, n):
            x0 = e[i] + e[j]
            p = int(np.searchsorted(e, x0, side="right"))  # find_1d: e[p-1] <= x0 < e[p], 1-based p
            if p < n:
                c[i, j] = math.log(x0 / e[p - 1]) / (3.0 * log_width)
                ima[i, j] = min(n - 2, p - 1)
            c[j, i] = c[i, j]
            ima[j, i] = ima[i, j]
    return c, ima


def smooth_kernel(k):
    """smooth_bin_kernel, run_sect.F90:414-444"""
    n = k.shape[0]
    out = np.empty_like(k)
    for i in range(n):
        im, ip = max(i - 1, 0), min(i + 1, n - 1)
        for j in range(n):
            jm, jp = max(j - 1, 0), min(j + 1, n - 1)
            out[i, j] = 0.125 * (k[i, jm] + k[im, j] + k[ip, j] + k[i, jp]) + 0.5 * k[i, j]
            if i == j:
                out[i, j] = 0.5 * out[i, j]
    return out


def run(kernel_type, density, num_conc, geom_mean_radius, log10_sigma, n_bin, d_min, d_max, del_t, t_max,
        t_output, temp=288.0, pressure=1e5):
    """run_sect for a single log-normal mode: returns (output times, bin
    centre radii, number concentration per unit ln r at each output time)."""
    _, centers, width = E.log_grid(n_bin, d_min / 2.0, d_max / 2.0)
    vol = E.rad2vol(centers)
    e = vol * density * 1e6  # kg to mg
    num = num_conc / (math.sqrt(2.0 * math.pi) * log10_sigma) * np.exp(
        -(np.log10(centers) - math.log10(geom_mean_radius)) ** 2 / (2.0 * log10_sigma ** 2)) / math.log(10.0)
    g = np.ascontiguousarray(num * vol * density)
    c, ima = courant(e, width)
    k = np.array([[O.kernel_value(kernel_type, vol[i], density, vol[j], density, temp, pressure)
                   for j in range(n_bin)] for i in range(n_bin)])
    ck = smooth_kernel(k) * 1e6  # m^3/s to cm^3/s
    ck = ck * del_t * width  # the reference scales row i by its bin width (all equal here)
    c = np.ascontiguousarray(c)
    ima = np.ascontiguousarray(ima)
    ck = np.ascontiguousarray(ck)
    e = np.ascontiguousarray(e)
    coad = _coad()
    n_steps = int(round(t_max / del_t))
    every = int(round(t_output / del_t))
    times, out = [0.0], [g / density / vol]
    for step in range(1, n_steps + 1):
        coad(n_bin, c.ctypes.data, ima.ctypes.data, g.ctypes.data, e.ctypes.data, ck.ctypes.data)
        if step % every == 0:
            times.append(step * del_t)
            out.append(g / density / vol)
    return np.array(times), centers, np.array(out)
