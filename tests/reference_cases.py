"""The reference's own validation cases, as protocols any engine can run:
the CPU oracle or the device (through the package's public API).

  test/brownian   one log-normal mode (1e11 m^-3, geometric mean diameter
                  50 nm, log10 sigma 0.24), Brownian kernel at 288 K and
                  1e5 Pa, 24 h of 600 s steps, against the reference's
                  sectional solver (run_sect.F90, restated in
                  oracle/sectional.py) at 60 s steps on 220 bins of 1e-10 to
                  1e-4 m; the test accepts a relative 2-norm error of 0.4
                  for number and mass at every hour (test_brownian_1.sh, _2.sh)
  test/sedi       one log-normal mode (1e9 m^-3, 20 um, 0.2), sedimentation
                  kernel, 600 s of 5 s steps, against the sectional solver at
                  1 s on 100 bins of 1e-7 to 1 m; 0.7 at 0, 300 and 600 s
                  (test_sedi_1.sh, _2.sh)
  test/bidisperse one 100 um droplet collecting 1000 droplets of 10 um under
                  the sedimentation kernel, flat weights, 600 s of 1 s steps,
                  against the reference's ODE (test_bidisperse_ode.F90); 0.3
                  (test_bidisperse_1.sh)

The particle runs follow run_part: 1000 particles under number-and-mass
weighting (run_part.F90:561-562) for the first two, rebalanced after every
step (run_part.F90:982).
"""
import math

import numpy as np
from scipy.integrate import solve_ivp

from oracle import exact as E
from oracle import ic_sampler as S
from oracle import oracle as O
from oracle import sectional as SC

RHO = 1000.0
ALPHAS = (0.0, -3.0)  # number and mass weighting: two groups, exponents 0 and -3
KERNEL_SEDI, KERNEL_BROWN = 1, 4

BROWN = dict(kernel=KERNEL_BROWN, num_conc=1e11, r_geom=2.5e-8, log10_sigma=0.24, n_bin=220, d_min=1e-10,
             d_max=1e-4, sect_dt=60.0, part_dt=600.0, t_max=86400.0, t_out=3600.0)
SEDI = dict(kernel=KERNEL_SEDI, num_conc=1e9, r_geom=1e-5, log10_sigma=0.2, n_bin=100, d_min=1e-7, d_max=1.0,
            sect_dt=1.0, part_dt=5.0, t_max=600.0, t_out=300.0)


class OracleEngine:
    """One population on the CPU oracle (test infrastructure)."""

    def __init__(self, weights, vols, group, seed):
        w_type, w_mag, w_exp = weights
        self.o = O.Oracle([RHO], (w_type, w_mag, w_exp), seed=seed)
        self.o.add_particles(vols, O.make_meta(len(vols), group=group))
        self.o.set_next_id(len(vols) + 1)

    def step(self, kernel, del_t):
        self.o.mc_coag(kernel, 288.0, 1e5, 0.0, del_t)

    def rebalance(self, ideal):
        self.o.rebalance(ideal)

    def vols(self):
        return self.o.particles()[0]

    def magnitudes(self):
        return self.o.weight_magnitudes()[:, 0]


class DeviceEngine:
    """One population on the device through partmc_b200's API."""

    def __init__(self, weights, vols, group, seed, mode=None):
        import partmc_b200 as pm
        self.pm = pm
        w_type, w_mag, w_exp = (np.asarray(x) for x in weights)
        self.data = pm.AeroData([RHO])
        self.st = pm.AeroState(self.data, pm.AeroWeightArray(w_type, w_mag, w_exp), seed=seed,
                               mode=pm.MODE_FP64 if mode is None else mode)
        self.st.add_particles(vols, group)
        self.env = pm.EnvState(288.0, 1e5)

    def step(self, kernel, del_t):
        self.pm.mc_coag(kernel, self.env, self.data, self.st, del_t)

    def rebalance(self, ideal):
        self.st.rebalance(ideal)

    def vols(self):
        return self.st.particles()["vol"]

    def magnitudes(self):
        return self.st.weight_magnitudes()[:, 0]


def sectional(sc):
    times, centers, num = SC.run(sc["kernel"], RHO, sc["num_conc"], sc["r_geom"], sc["log10_sigma"], sc["n_bin"],
                                 sc["d_min"], sc["d_max"], sc["sect_dt"], sc["t_max"], sc["t_out"])
    return num, num * E.rad2vol(centers) * RHO


def particle_run(sc, k, engine=OracleEngine, n_part=1000, del_t=None, **kw):
    """One particle run, half the particles in each weight group; each
    particle counts at the groups' harmonic number concentration at its
    radius (aero_weight_array_num_conc_at_radius).  Returns the number and
    mass distributions at the output times."""
    mode = S.Mode(S.MODE_LOG_NORMAL, char_radius=sc["r_geom"], log10_std=sc["log10_sigma"], num_conc=sc["num_conc"])
    ws = [S.Weight(S.WEIGHT_POWER, S.mode_number(mode, S.Weight(S.WEIGHT_POWER, 1.0, a)) / (n_part / 2), a)
          for a in ALPHAS]
    vols, grp, _ = S.add_dist_sample(np.random.default_rng(100 + k), [mode], ws, 1.0)
    weights = ([[O.WEIGHT_POWER], [O.WEIGHT_POWER]], [[ws[0].magnitude], [ws[1].magnitude]],
               [[ALPHAS[0]], [ALPHAS[1]]])
    eng = engine(weights, vols, grp + 1, 7 + k, **kw)
    dt = sc["part_dt"] if del_t is None else del_t
    n_steps = int(round(sc["t_max"] / dt))
    every = int(round(sc["t_out"] / dt))
    num, mass = [], []
    for step in range(0, n_steps + 1):
        if step > 0:
            eng.step(sc["kernel"], dt)
            eng.rebalance(n_part / 2)
        if step % every == 0:
            v = eng.vols().sum(1)
            mags = eng.magnitudes()
            r = E.vol2rad(v)
            nc = 1.0 / sum(1.0 / (mags[g] * r ** ALPHAS[g]) for g in range(len(ALPHAS)))
            h = lambda wt: E.size_histogram(2.0 * r, wt, sc["n_bin"], sc["d_min"], sc["d_max"])[0]
            num.append(h(nc))
            mass.append(h(nc * v * RHO))
    return np.array(num), np.array(mass)


def max_err(ref, approx):
    return max(E.rel_err_by_col(ref[t], approx[t])[0] for t in range(len(ref)))


def sectional_errors(sc, engine=OracleEngine, n_runs=8, **kw):
    """Largest error over the output times of every run and of the runs'
    mean, for number and for mass, against the sectional solution."""
    sect_num, sect_mass = sectional(sc)
    runs = [particle_run(sc, k, engine, **kw) for k in range(n_runs)]
    per_run = [(max_err(sect_num, n), max_err(sect_mass, m)) for n, m in runs]
    mean = (max_err(sect_num, np.mean([r[0] for r in runs], axis=0)),
            max_err(sect_mass, np.mean([r[1] for r in runs], axis=0)))
    return per_run, mean


# test/bidisperse
R_SMALL, R_BIG, N0 = 1e-5, 1e-4, 1000
BIDI_TIMES = np.arange(0.0, 601.0, 10.0)


def bidisperse_ode():
    """test_bidisperse_ode.F90: dn/dt = -K(v_small, v_big) n / V with
    v_big = v_big0 + (n0 - n) v_small, solved with scipy instead of RK4."""
    vs, vb0 = float(E.rad2vol(R_SMALL)), float(E.rad2vol(R_BIG))
    comp_vol = N0 / 1e9

    def rhs(t, y):
        vb = vb0 + (N0 - y[0]) * vs
        return [-O.kernel_value(O.KERNEL_SEDI, vs, RHO, vb, RHO) / comp_vol * y[0]]

    n = solve_ivp(rhs, (0.0, 600.0), [float(N0)], t_eval=BIDI_TIMES, rtol=1e-10, atol=1e-8).y[0]
    return n / comp_vol, (vb0 + (N0 - n) * vs) * RHO / comp_vol


def bidisperse_run(seed, engine=OracleEngine, **kw):
    """Small-droplet number and big-droplet mass every 10 s; checks that
    volume is conserved (flat weights)."""
    vs, vb0 = float(E.rad2vol(R_SMALL)), float(E.rad2vol(R_BIG))
    comp_vol = N0 / 1e9
    vols = np.full(N0 + 1, vs)
    vols[-1] = vb0
    eng = engine(([[1]], [[1.0 / comp_vol]], [[0.0]]), vols[:, None], np.ones(N0 + 1, np.int32), seed, **kw)
    n, m = [N0 / comp_vol], [vb0 * RHO / comp_vol]
    for step in range(1, 601):
        eng.step(KERNEL_SEDI, 1.0)
        if step % 10 == 0:
            v = eng.vols().sum(1)
            n.append((len(v) - 1) / comp_vol)
            m.append(v.max() * RHO / comp_vol)
            assert abs(v.sum() - (N0 * vs + vb0)) <= 1e-12 * v.sum()
    return np.array(n), np.array(m)
