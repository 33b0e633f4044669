"""The oracle against the reference's known answers: the additive kernel's
exact solution (test/additive, soln_additive_exp) and the constant kernel's
(soln_constant_exp), on an ensemble of runs so the check stays within seconds."""
import numpy as np

from oracle import exact as E
from oracle import oracle as O

N0, R = 1e9, 1e-5


def run_ensemble(kernel, n_part, n_runs, t_end, del_t, times, coeff=1000.0):
    hs = {t: [] for t in times}
    ms = {t: [] for t in times}
    for k in range(n_runs):
        rng = np.random.default_rng(1000 + k)
        vols = -E.rad2vol(R) * np.log(rng.random(n_part))
        orc = O.Oracle([1000.0], ([[1]], [[N0 / n_part]], [[0.0]]), seed=77 + k)
        orc.add_particles(vols[:, None], O.make_meta(n_part))
        orc.set_next_id(n_part + 1)
        step = 0
        for step in range(1, int(round(t_end / del_t)) + 1):
            orc.mc_coag(kernel, 288.0, 1e5, coeff, del_t)
            # run_part_timestep rebalances after every step (run_part.F90:982)
            orc.rebalance(n_part)
            t = step * del_t
            if t in hs:
                vol, _ = orc.particles()
                nc = orc.weight_magnitudes()[0, 0]
                d = 2 * E.vol2rad(vol.sum(1))
                h, dc = E.size_histogram(d, np.full(len(d), nc))
                hm, _ = E.size_histogram(d, np.full(len(d), nc) * vol.sum(1) * 1000.0)
                hs[t].append(h)
                ms[t].append(hm)
    return hs, ms, dc


def test_additive_exact_solution():
    times = [60.0, 180.0, 300.0, 600.0]
    hs, ms, dc = run_ensemble(O.KERNEL_ADDITIVE, 10000, 10, 600.0, 1.0, times)
    for t in times:
        ex = E.soln_additive_exp(dc / 2, t, N0, R, 1000.0)
        exm = ex * E.rad2vol(dc / 2) * 1000.0
        num_err = E.rel_err_by_col(ex, np.mean(hs[t], axis=0))[0]
        mass_err = E.rel_err_by_col(exm, np.mean(ms[t], axis=0))[0]
        # test_additive_1.sh / _2.sh: 0.05 (number), 0.2 (mass); the ensemble of
        # 10 x 1e4 particles (doubled back to 1e4 each step, as with
        # allow_doubling yes) has the statistical power of one 1e5 run
        assert num_err < 0.05, (t, num_err)
        assert mass_err < 0.2, (t, mass_err)


def test_constant_exact_solution():
    # tau = N0 beta_0 t reaches 2 at t = 96 s for N0 = 1e9
    times = [24.0, 96.0]
    hs, ms, dc = run_ensemble(O.KERNEL_CONSTANT, 10000, 8, 96.0, 1.0, times)
    for t in times:
        ex = E.soln_constant_coag(dc / 2, t, N0, R)
        err = E.rel_err_by_col(ex, np.mean(hs[t], axis=0))[0]
        assert err < 0.1, (t, err)
