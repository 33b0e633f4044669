"""The oracle against the reference's test/bidisperse: one large droplet
(radius 100 um) collecting 1000 small ones (10 um) under the sedimentation
kernel, flat weights at 1e9 small droplets per m^3, 1 s steps for 600 s
(test/bidisperse/run_part.spec), compared with the reference's ODE for the
number of small droplets (test/bidisperse/test_bidisperse_ode.F90:
dn/dt = -K(v_small, v_big) n / V with v_big = v_big0 + (n0 - n) v_small),
solved here with scipy instead of RK4 at 1 ms.  The reference's test accepts
a relative 2-norm error of 0.3 per series (numeric_diff --by col
--rel-tol 0.3); every run here stays within it, and the mean of 8 runs within
0.03.  CPU only."""
import numpy as np
from scipy.integrate import solve_ivp

from oracle import exact as E
from oracle import oracle as O

R_SMALL, R_BIG, RHO, N0 = 1e-5, 1e-4, 1000.0, 1000
TIMES = np.arange(0.0, 601.0, 10.0)


def ode():
    vs, vb0 = float(E.rad2vol(R_SMALL)), float(E.rad2vol(R_BIG))
    comp_vol = N0 / 1e9

    def rhs(t, y):
        vb = vb0 + (N0 - y[0]) * vs
        return [-O.kernel_value(O.KERNEL_SEDI, vs, RHO, vb, RHO) / comp_vol * y[0]]

    n = solve_ivp(rhs, (0.0, 600.0), [float(N0)], t_eval=TIMES, rtol=1e-10, atol=1e-8).y[0]
    return n / comp_vol, (vb0 + (N0 - n) * vs) * RHO / comp_vol


def particle_run(seed):
    vs, vb0 = float(E.rad2vol(R_SMALL)), float(E.rad2vol(R_BIG))
    comp_vol = N0 / 1e9
    orc = O.Oracle([RHO], ([[1]], [[1.0 / comp_vol]], [[0.0]]), seed=seed)
    vols = np.full(N0 + 1, vs)
    vols[-1] = vb0
    orc.add_particles(vols[:, None], O.make_meta(N0 + 1))
    orc.set_next_id(N0 + 2)
    n, m = [N0 / comp_vol], [vb0 * RHO / comp_vol]
    for step in range(1, 601):
        orc.mc_coag(O.KERNEL_SEDI, 288.0, 1e5, 0.0, 1.0)
        if step % 10 == 0:
            v = orc.particles()[0].sum(1)
            n.append((len(v) - 1) / comp_vol)
            m.append(v.max() * RHO / comp_vol)
            assert abs(v.sum() - (N0 * vs + vb0)) <= 1e-12 * v.sum()  # volume conserved
    return np.array(n), np.array(m)


def test_bidisperse_matches_the_ode():
    ode_n, ode_m = ode()
    runs = [particle_run(31 + k) for k in range(8)]
    for n, m in runs:
        assert E.rel_err_by_col(ode_n, n)[0] < 0.3
        assert E.rel_err_by_col(ode_m, m)[0] < 0.3
    mean_n = np.mean([n for n, _ in runs], axis=0)
    mean_m = np.mean([m for _, m in runs], axis=0)
    assert E.rel_err_by_col(ode_n, mean_n)[0] < 0.03
    assert E.rel_err_by_col(ode_m, mean_m)[0] < 0.03
