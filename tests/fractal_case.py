"""The reference's test/fractal cases (test_fractal_2.sh, test_fractal_3.sh)
as a protocol any stepper can run: the oracle on the CPU or the device.

Each case is PartMC's run_part with one species (density 4200 kg m^-3,
test/fractal/aero_data.dat), 10,000 particles of one monomer each (mode
"mono", number concentration 1e14 m^-3, test/fractal/aero_init_dist_*.dat),
flat weights, coagulation only, doubling and halving after every step
(run_part.F90:982), and the fractal parameters of the spec files:
  free  brown_free kernel, d_f 2.4, R0 0.5 nm, 1800 K (temp_free.dat)
  cont  brown_cont kernel, d_f 1.8, R0 0.25 um, 300 K (temp_cont.dat)
both at 1e5 Pa with a volume filling factor of 1.  The run is the spec
files' two legs: 1000 s of 10 s steps with output every 50 s, then (the
restart run) 65,000 s of 100 s steps with output every 5000 s.  At each
output test_fractal_dimless_time.F90 writes the dimensionless time
(free: sqrt(6 k T R0 / rho) N0 t; cont: 2 k T / (3 mu) N0 t, with mu the
reference's constant air viscosity) and N / N0; the shell scripts then
compare both columns with the reference solution by numeric_diff --by col
--rel-tol 0.1: per column, ||a - b||_2 / ||a||_2 < 0.1 (numeric_diff.F90).
"""
import math

import numpy as np

KERNEL_BROWN_FREE, KERNEL_BROWN_CONT = 6, 7
N_PART, NUM_CONC, DENSITY, PRESSURE = 10000, 1e14, 4200.0, 1e5
BOLTZMANN, AIR_DYN_VISC = 1.3806505e-23, 1.78e-5  # constants.F90
REL_TOL = 0.1  # test_fractal_2.sh:18, test_fractal_3.sh:18

CASES = {
    "free": dict(kernel=KERNEL_BROWN_FREE, frac_dim=2.4, prime_radius=5e-10, temp=1800.0),
    "cont": dict(kernel=KERNEL_BROWN_CONT, frac_dim=1.8, prime_radius=2.5e-7, temp=300.0),
}
# (step length s, steps, steps between outputs): the spec files' two legs
LEGS = ((10.0, 100, 5), (100.0, 650, 50))


def monomer_volume(case):
    """Mode diameter 2 R0 (diam_type geometric): fractal_rad2vol of R0 is the
    sphere of radius R0, one monomer."""
    r0 = CASES[case]["prime_radius"]
    return 4.0 * math.pi * r0 ** 3 / 3.0


def dimless_time(case, t):
    c = CASES[case]
    if case == "free":
        return math.sqrt(6.0 * BOLTZMANN * c["temp"] * c["prime_radius"] / DENSITY) * NUM_CONC * t
    return 2.0 * BOLTZMANN * c["temp"] / 3.0 / AIR_DYN_VISC * NUM_CONC * t


def run(case, stepper):
    """stepper(del_t) advances one step (coagulation, then rebalance) and
    returns the number concentration (m^-3); stepper(None) returns it
    without stepping.  Returns the rows (dimensionless time, N / N0) at the
    outputs, 34 of them like the reference solution."""
    rows = [(0.0, stepper(None) / NUM_CONC)]
    t = 0.0
    for del_t, n_steps, every in LEGS:
        for k in range(1, n_steps + 1):
            n = stepper(del_t)
            t += del_t
            if k % every == 0:
                rows.append((dimless_time(case, t), n / NUM_CONC))
    return np.array(rows)


def rel_err_by_col(ref, got):
    """numeric_diff --by col with the default two-norm: per column the norm
    of the difference over the norm of the first file's column."""
    ref, got = np.asarray(ref, dtype=np.float64), np.asarray(got, dtype=np.float64)
    assert ref.shape == got.shape, (ref.shape, got.shape)
    return np.sqrt(((ref - got) ** 2).sum(0)) / np.sqrt((ref ** 2).sum(0))


def oracle_stepper(case, seed):
    """The case on the CPU oracle (test infrastructure)."""
    from oracle import oracle as O
    c = CASES[case]
    o = O.Oracle([DENSITY], ([[1]], [[NUM_CONC / N_PART]], [[0.0]]), seed=seed)
    o.set_fractal(c["frac_dim"], c["prime_radius"], 1.0)
    o.add_particles(np.full((N_PART, 1), monomer_volume(case)), O.make_meta(N_PART))
    o.set_next_id(N_PART + 1)

    def step(del_t):
        if del_t is not None:
            o.mc_coag(c["kernel"], c["temp"], PRESSURE, 0.0, del_t)
            o.rebalance(N_PART)
        return o.n_part * float(o.weight_magnitudes().ravel()[0])
    return step


def device_stepper(case, seed, mode=None):
    """The case on the device through the package's public API."""
    import partmc_b200 as pm
    c = CASES[case]
    data = pm.AeroData([DENSITY], fractal=pm.Fractal(c["frac_dim"], c["prime_radius"], 1.0))
    st = pm.AeroState(data, pm.AeroWeightArray.flat(magnitude=NUM_CONC / N_PART), seed=seed,
                      mode=pm.MODE_FP64 if mode is None else mode)
    st.add_particles(np.full((N_PART, 1), monomer_volume(case)), 1)
    env = pm.EnvState(c["temp"], PRESSURE)

    def step(del_t):
        if del_t is not None:
            pm.mc_coag(c["kernel"], env, data, st, del_t)
            st.rebalance(N_PART)
        return st.n_part() * float(st.weight_magnitudes().ravel()[0])
    return step
