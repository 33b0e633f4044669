"""Unit checks of the oracle's restated functions (hand-checkable values)."""
import numpy as np

from oracle import exact as E
from oracle import oracle as O


def test_vol_rad_round_trip():
    for r in [1e-9, 3.3e-7, 2e-5]:
        # pow(x, fl(1/3)) carries |ln x| * (1/3 - fl(1/3)) ~ 1e-15 relative
        assert abs(O.vol2rad(O.rad2vol(r)) / r - 1) < 2e-15


def test_additive_and_constant_values():
    v1, v2 = 1e-15, 3e-16
    assert O.kernel_value(O.KERNEL_ADDITIVE, v1, 1000, v2, 1000, coeff=1000.0) == 1000.0 * (v1 + v2)
    assert O.kernel_value(O.KERNEL_CONSTANT, v1, 1000, v2, 1000) == 0.25 / (60.0 * 2e8)


def brown_numpy(v1, d1, v2, d2, T, p):
    """Jacobson (2005) eq. 15.33 in numpy, independent of the C code."""
    kb, NA, R, M, pi = 1.3806505e-23, 6.02214179e23, 8.314472, 2.89644e-2, np.pi
    rhoair = p * M / (R * T)
    mu = 1.8325e-5 * (416.16 / (T + 120.0)) * (T / 296.16) ** 1.5
    lam = 2.0 * (mu / rhoair) / np.sqrt(8.0 * kb * T * NA / (pi * M))
    out = []
    for v, d in [(v1, d1), (v2, d2)]:
        r = (3.0 * v / (4.0 * pi)) ** (1.0 / 3.0)
        kn = lam / r
        D = kb * T * (1.0 + kn * (1.249 + 0.42 * np.exp(-0.87 / kn))) / (6.0 * pi * r * mu)
        c2 = 8.0 * kb * T / (pi * d * v)
        l = 8.0 * D / (pi * np.sqrt(c2))
        delta = ((2 * r + l) ** 3 - (4 * r * r + l * l) ** 1.5) / (6 * r * l) - 2 * r
        out.append((r, D, c2, delta ** 2))
    (r1, D1, c1, s1), (r2, D2, c2, s2) = out
    rs, Ds = r1 + r2, D1 + D2
    return 4 * pi * rs * Ds / (rs / (rs + np.sqrt(s1 + s2)) + 4 * Ds / (rs * np.sqrt(c1 + c2)))


def test_brownian_matches_independent_formula():
    rng = np.random.default_rng(1)
    for _ in range(50):
        r1, r2 = 10 ** rng.uniform(-9, -5, 2)
        d1, d2 = rng.uniform(1000, 2000, 2)
        v1, v2 = O.rad2vol(r1), O.rad2vol(r2)
        k = O.kernel_value(O.KERNEL_BROWN, v1, d1, v2, d2, temp=288.0, pressure=1e5)
        assert abs(k / brown_numpy(v1, d1, v2, d2, 288.0, 1e5) - 1) < 1e-10


def test_sedi_kernel_positive_and_symmetric():
    for r1, r2 in [(1e-5, 2e-5), (5e-6, 1e-4), (2e-4, 3e-4)]:
        v1, v2 = O.rad2vol(r1), O.rad2vol(r2)
        a = O.kernel_value(O.KERNEL_SEDI, v1, 1000, v2, 1000)
        b = O.kernel_value(O.KERNEL_SEDI, v2, 1000, v1, 1000)
        assert a > 0 and a == b


def test_bin_grid_and_find():
    e, c = O.bin_grid_make(40, 1e-9, 1e-5)
    assert e[0] == 1e-9 and e[-1] == 1e-5 and len(c) == 40
    assert np.allclose(np.diff(np.log(e)), np.log(1e4) / 40)
    for b in range(1, 41):
        r = np.sqrt(e[b - 1] * e[b])
        assert O.bin_find(40, e[0], e[-1], r) == b
    assert O.bin_find(40, e[0], e[-1], 1e-10) == 0
    assert O.bin_find(40, e[0], e[-1], 1e-4) == 41
    assert O.bin_find(40, e[0], e[-1], e[-1]) == 40


def test_student_t_table():
    from scipy.stats import t
    for n in range(2, 60):
        assert abs(O.student_t_95(n) / t.ppf(0.975, n - 1) - 1) < 1e-3


def test_weight_harmonic_combination():
    orc = O.Oracle([1000.0], ([[1], [2]], [[2.0], [3.0]], [[0.0], [-3.0]]))
    r = 1e-7
    want = 1.0 / (1.0 / 2.0 + 1.0 / (3.0 * r ** -3))
    assert abs(orc.num_conc_at_radius(1, r) / want - 1) < 1e-15


def test_sort_bookkeeping_consistent_after_steps():
    rng = np.random.default_rng(2)
    n = 3000
    vol = E.rad2vol(10 ** rng.normal(np.log10(5e-8), 0.2, n))[:, None]
    orc = O.Oracle([1800.0], ([[2]], [[1e5]], [[-1.0]]), seed=4)
    orc.add_particles(vol, O.make_meta(n))
    orc.set_next_id(n + 1)
    for _ in range(20):
        orc.mc_coag(O.KERNEL_BROWN, 288.0, 1e5, 0.0, 600.0)
        assert orc.check() == 0
    vol2, meta = orc.particles()
    assert len(np.unique(meta["id"])) == len(meta)


def test_oracle_removal_records_account_for_every_id():
    """The oracle's aero_info log over coagulation steps of three weightings
    (flat additive; power weights with the per-particle path; nummass with 20
    species) and a halving: every ID that existed is present afterwards or
    removed with exactly one record (removal_check.py)."""
    import removal_check as RCK
    from partmc_b200 import aero_dist
    cases = [(aero_dist.additive_exp(3000, seed=3), O.KERNEL_ADDITIVE, 60.0),
             (aero_dist.brown_bimodal(3000, seed=4, modes=[(1e11, 0.005e-6, np.log10(1.5)),
                                                           (1e8, 0.25e-6, np.log10(1.5))]), O.KERNEL_BROWN, 600.0),
             (aero_dist.brown_20spec(3000, seed=5), O.KERNEL_BROWN, 600.0)]
    for pop, kt, dt in cases:
        o = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=9)
        o.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group, ids=np.arange(1, pop.n_part + 1)))
        o.set_next_id(pop.n_part + 1)
        o.set_record_removals(True)
        for _ in range(3):
            ids0, nid0 = o.particles()[1]["id"].copy(), o.next_id()
            o.mc_coag(kt, 288.0, 1e5, 1000.0, dt)
            rec = o.removals()
            RCK.check_id_accounting(ids0, nid0, o.next_id(), o.particles()[1]["id"], rec)
            assert len(rec["id"]) > 0
        ids0, nid0 = o.particles()[1]["id"].copy(), o.next_id()
        o.rebalance(np.full((o.n_group, o.n_class), o.n_part / 8.0), allow_doubling=False)
        rec = o.removals()
        assert (rec["action"] == RCK.INFO_HALVED).all() and len(rec["id"]) > 0
        RCK.check_id_accounting(ids0, nid0, o.next_id(), o.particles()[1]["id"], rec)
