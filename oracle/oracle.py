"""ctypes wrapper of the CPU oracle (oracle/pmc_oracle.c).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and bench.py's CPU
baseline leg use this module as the checker.  The product library in
partmc_b200/ never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

KERNEL_SEDI, KERNEL_ADDITIVE, KERNEL_CONSTANT, KERNEL_BROWN, KERNEL_ZERO = 1, 2, 3, 4, 5
KERNEL_BROWN_FREE, KERNEL_BROWN_CONT = 6, 7
WEIGHT_NONE, WEIGHT_POWER, WEIGHT_MFA = 1, 2, 3
INFO_NONE, INFO_DILUTION, INFO_COAG, INFO_HALVED, INFO_WEIGHT = 0, 1, 2, 3, 4  # aero_info.F90:19-28
MAX_COMPONENT = 20

# layout of orc_particle_meta (pmc_oracle.h)
META_DTYPE = np.dtype(
    [
        ("weight_group", np.int32),
        ("weight_class", np.int32),
        ("id", np.int64),
        ("n_primary_parts", np.int32),
        ("n_comp", np.int32),
        ("comp_source", np.int32, (MAX_COMPONENT,)),
        ("comp_create_time", np.float64, (MAX_COMPONENT,)),
        ("least_create_time", np.float64),
        ("greatest_create_time", np.float64),
        ("water_hyst_leg", np.int32),
        ("frozen", np.int32),
        ("imf_temperature", np.float64),
        ("den_ice", np.float64),
        ("ice_shape_phi", np.float64),
    ],
    align=True,
)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, dp, dp]
        L.orc_destroy.argtypes = [P]
        L.orc_set_weight.argtypes = [P, ip, dp, dp]
        L.orc_set_seed.argtypes = [P, ctypes.c_uint64]
        L.orc_set_replay.argtypes = [P, dp, ctypes.c_int64]
        L.orc_enable_dump.argtypes = [P, ctypes.c_int64]
        L.orc_dump_count.restype = ctypes.c_int64
        L.orc_dump_count.argtypes = [P]
        L.orc_dump_copy.restype = ctypes.c_int64
        L.orc_dump_copy.argtypes = [P, dp, ctypes.c_int64]
        L.orc_uniforms_used.restype = ctypes.c_int64
        L.orc_uniforms_used.argtypes = [P]
        L.orc_random.restype = ctypes.c_double
        L.orc_random.argtypes = [P]
        L.orc_set_next_id.argtypes = [P, ctypes.c_int64]
        L.orc_get_next_id.restype = ctypes.c_int64
        L.orc_get_next_id.argtypes = [P]
        L.orc_add_particles.argtypes = [P, ctypes.c_int, dp, P]
        L.orc_n_part.argtypes = [P]
        L.orc_get_particles.argtypes = [P, dp, P]
        L.orc_mc_coag.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ip, ip]
        L.orc_kmax_warnings.restype = ctypes.c_int64
        L.orc_kmax_warnings.argtypes = [P]
        L.orc_pp_targets.restype = ctypes.c_int64
        L.orc_pp_targets.argtypes = [P]
        L.orc_sort.argtypes = [P]
        L.orc_n_bin.argtypes = [P]
        L.orc_bin_edges.argtypes = [P, dp]
        L.orc_bin_counts.argtypes = [P, ip]
        L.orc_particle_bins.argtypes = [P, ip]
        L.orc_check.argtypes = [P]
        L.orc_kmax_table.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_vol2rad.restype = ctypes.c_double
        L.orc_vol2rad.argtypes = [ctypes.c_double]
        L.orc_rad2vol.restype = ctypes.c_double
        L.orc_rad2vol.argtypes = [ctypes.c_double]
        L.orc_kernel_value.restype = ctypes.c_double
        L.orc_kernel_value.argtypes = [ctypes.c_int] + [ctypes.c_double] * 7
        L.orc_kernel_minmax.argtypes = [P, ctypes.c_int] + [ctypes.c_double] * 5 + [dp, dp]
        L.orc_weighted_kernel.restype = ctypes.c_double
        L.orc_weighted_kernel.argtypes = [P, ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_num_conc_at_radius.restype = ctypes.c_double
        L.orc_num_conc_at_radius.argtypes = [P, ctypes.c_int, ctypes.c_double]
        L.orc_bin_find.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_bin_grid_make.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_coag_dest_class.argtypes = [P, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_max_num_conc_factor.restype = ctypes.c_double
        L.orc_max_num_conc_factor.argtypes = [P, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int]
        L.orc_student_t_95.restype = ctypes.c_double
        L.orc_student_t_95.argtypes = [ctypes.c_int]
        L.orc_rand_poisson.argtypes = [P, ctypes.c_double]
        L.orc_rand_binomial.argtypes = [P, ctypes.c_int, ctypes.c_double]
        L.orc_rand_normal.restype = ctypes.c_double
        L.orc_rand_normal.argtypes = [P, ctypes.c_double, ctypes.c_double]
        L.orc_rand_int.argtypes = [P, ctypes.c_int]
        L.orc_prob_round.argtypes = [P, ctypes.c_double]
        L.orc_step_many.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        L.orc_poisson_hist.argtypes = [P, ctypes.c_double, ctypes.c_int64, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int64)]
        L.orc_binomial_hist.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int64)]
        L.orc_set_fractal.argtypes = [P, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_set_record_removals.argtypes = [P, ctypes.c_int]
        L.orc_removals.restype = ctypes.c_int64
        L.orc_removals.argtypes = [P, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ip,
                                   ctypes.POINTER(ctypes.c_int64)]
        L.orc_fractal_radius.restype = ctypes.c_double
        L.orc_fractal_radius.argtypes = [ctypes.c_double] * 6 + [dp]
        L.orc_kernel_value_fractal.restype = ctypes.c_double
        L.orc_kernel_value_fractal.argtypes = [ctypes.c_int] + [ctypes.c_double] * 10
        L.orc_rebalance.argtypes = [P, dp, ctypes.c_int, ctypes.c_int]
        L.orc_get_weight.argtypes = [P, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_meta(n, group=None, cls=None, ids=None, n_primary=None, source=None, create_time=0.0):
    """Particle metadata the way aero_state_add_aero_dist_sample makes it
    (aero_state.F90:812-822): one component, n_primary_parts = 1."""
    m = np.zeros(n, dtype=META_DTYPE)
    m["weight_group"] = 1 if group is None else group
    m["weight_class"] = 1 if cls is None else cls
    m["id"] = np.arange(1, n + 1) if ids is None else ids
    m["n_primary_parts"] = 1 if n_primary is None else n_primary
    m["n_comp"] = 1
    m["comp_source"][:, 0] = 1 if source is None else source
    m["comp_create_time"][:, 0] = create_time
    m["least_create_time"] = create_time
    m["greatest_create_time"] = create_time
    m["den_ice"] = np.nan
    m["ice_shape_phi"] = np.nan
    return m


class Oracle:
    """One population held by the C oracle."""

    def __init__(self, density, weights, i_water=0, seed=1):
        L = lib()
        density = np.ascontiguousarray(density, dtype=np.float64)
        w_type, w_mag, w_exp = weights
        w_type = np.asfortranarray(np.atleast_2d(w_type), dtype=np.int32)
        w_mag = np.asfortranarray(np.atleast_2d(w_mag), dtype=np.float64)
        w_exp = np.asfortranarray(np.atleast_2d(w_exp), dtype=np.float64)
        self.n_group, self.n_class = w_type.shape
        self.n_spec = density.size
        self._keep = [density, w_type, w_mag, w_exp]
        self.ptr = L.orc_create(self.n_spec, _dp(density), i_water, self.n_group, self.n_class,
                                _ip(w_type.ravel(order="F")), _dp(w_mag.ravel(order="F")),
                                _dp(w_exp.ravel(order="F")))
        if not self.ptr:
            raise ValueError("orc_create failed")
        L.orc_set_seed(self.ptr, seed)
        self._replay = None

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_destroy(self.ptr)
            self.ptr = None

    def set_weight(self, weights):
        w_type, w_mag, w_exp = weights
        w_type = np.asfortranarray(np.atleast_2d(w_type), dtype=np.int32).ravel(order="F")
        w_mag = np.asfortranarray(np.atleast_2d(w_mag), dtype=np.float64).ravel(order="F")
        w_exp = np.asfortranarray(np.atleast_2d(w_exp), dtype=np.float64).ravel(order="F")
        self._keep_w = [w_type, w_mag, w_exp]
        lib().orc_set_weight(self.ptr, _ip(w_type), _dp(w_mag), _dp(w_exp))

    def set_fractal(self, frac_dim, prime_radius, vol_fill_factor=1.0):
        """Particle shape (fractal_t); d_f = 3, f = 1 are spheres."""
        rc = lib().orc_set_fractal(self.ptr, frac_dim, prime_radius, vol_fill_factor)
        if rc:
            raise ValueError(f"orc_set_fractal failed: {rc}")

    def set_record_removals(self, on=True):
        lib().orc_set_record_removals(self.ptr, int(bool(on)))

    def removals(self, max_n=1 << 22):
        """Removal records since the last call, in removal order: dict of id,
        action (aero_info.F90 codes) and other_id arrays; cleared."""
        i64 = ctypes.POINTER(ctypes.c_int64)
        ids = np.zeros(max_n, np.int64)
        act = np.zeros(max_n, np.int32)
        oth = np.zeros(max_n, np.int64)
        n = lib().orc_removals(self.ptr, max_n, ids.ctypes.data_as(i64), _ip(act), oth.ctypes.data_as(i64))
        if n < 0:
            raise ValueError(f"{-n} removal records exceed max_n")
        return {"id": ids[:n], "action": act[:n], "other_id": oth[:n]}

    def seed(self, s):
        lib().orc_set_seed(self.ptr, s)

    def set_replay(self, u):
        self._replay = np.ascontiguousarray(u, dtype=np.float64)
        lib().orc_set_replay(self.ptr, _dp(self._replay), self._replay.size)

    def enable_dump(self, cap=1 << 16):
        lib().orc_enable_dump(self.ptr, cap)

    def dump(self):
        n = lib().orc_dump_count(self.ptr)
        out = np.empty(n, dtype=np.float64)
        lib().orc_dump_copy(self.ptr, _dp(out), n)
        return out

    def uniforms_used(self):
        return lib().orc_uniforms_used(self.ptr)

    def set_next_id(self, i):
        lib().orc_set_next_id(self.ptr, i)

    def next_id(self):
        return lib().orc_get_next_id(self.ptr)

    def add_particles(self, vol, meta):
        vol = np.ascontiguousarray(vol, dtype=np.float64)  # (n, n_spec)
        assert vol.ndim == 2 and vol.shape[1] == self.n_spec
        meta = np.ascontiguousarray(meta, dtype=META_DTYPE)
        rc = lib().orc_add_particles(self.ptr, vol.shape[0], _dp(vol), meta.ctypes.data_as(ctypes.c_void_p))
        if rc:
            raise RuntimeError(f"orc_add_particles failed: {rc}")

    @property
    def n_part(self):
        return lib().orc_n_part(self.ptr)

    def particles(self):
        n = self.n_part
        vol = np.empty((n, self.n_spec), dtype=np.float64)
        meta = np.empty(n, dtype=META_DTYPE)
        lib().orc_get_particles(self.ptr, _dp(vol), meta.ctypes.data_as(ctypes.c_void_p))
        return vol, meta

    def mc_coag(self, kernel_type, temp, pressure, additive_coeff, del_t):
        a = ctypes.c_int()
        b = ctypes.c_int()
        rc = lib().orc_mc_coag(self.ptr, kernel_type, temp, pressure, additive_coeff, del_t,
                               ctypes.byref(a), ctypes.byref(b))
        if rc:
            raise RuntimeError(f"orc_mc_coag failed with status {rc}")
        return a.value, b.value

    def kmax_warnings(self):
        return lib().orc_kmax_warnings(self.ptr)

    def pp_targets(self):
        """Targets the per-particle (accelerated) path has handled."""
        return lib().orc_pp_targets(self.ptr)

    def sort(self):
        rc = lib().orc_sort(self.ptr)
        if rc:
            raise RuntimeError(f"orc_sort failed: {rc}")

    def n_bin(self):
        return lib().orc_n_bin(self.ptr)

    def bin_edges(self):
        n = self.n_bin()
        e = np.empty(n + 1, dtype=np.float64)
        if n > 0:
            lib().orc_bin_edges(self.ptr, _dp(e))
        return e

    def bin_counts(self):
        n = self.n_bin()
        c = np.zeros(n * self.n_class, dtype=np.int32)
        if n > 0:
            lib().orc_bin_counts(self.ptr, _ip(c))
        return c.reshape(self.n_class, n).T  # (n_bin, n_class)

    def particle_bins(self):
        b = np.empty(self.n_part, dtype=np.int32)
        rc = lib().orc_particle_bins(self.ptr, _ip(b))
        if rc:
            raise RuntimeError("not sorted")
        return b

    def check(self):
        return lib().orc_check(self.ptr)

    def kmax_table(self, kernel_type, temp, pressure, coeff):
        n = self.n_bin()
        kmin = np.empty(n * n)
        kmax = np.empty(n * n)
        rc = lib().orc_kmax_table(self.ptr, kernel_type, temp, pressure, coeff, _dp(kmin), _dp(kmax))
        if rc:
            raise RuntimeError(rc)
        return kmin.reshape(n, n, order="F"), kmax.reshape(n, n, order="F")

    def weighted_kernel(self, kernel_type, vol1, c1, vol2, c2, cij, temp, pressure, coeff):
        v1 = np.ascontiguousarray(vol1, dtype=np.float64)
        v2 = np.ascontiguousarray(vol2, dtype=np.float64)
        return lib().orc_weighted_kernel(self.ptr, kernel_type, _dp(v1), c1, _dp(v2), c2, cij, temp, pressure,
                                         coeff)

    def num_conc_at_radius(self, c, r):
        return lib().orc_num_conc_at_radius(self.ptr, c, r)

    def rand_poisson(self, mean):
        return lib().orc_rand_poisson(self.ptr, mean)

    def rand_binomial(self, n, p):
        return lib().orc_rand_binomial(self.ptr, n, p)

    def random(self):
        return lib().orc_random(self.ptr)

    def rebalance(self, n_part_ideal, allow_doubling=True, allow_halving=True):
        ideal = np.asfortranarray(np.broadcast_to(np.atleast_2d(n_part_ideal), (self.n_group, self.n_class)),
                                  dtype=np.float64).ravel(order="F")
        rc = lib().orc_rebalance(self.ptr, _dp(ideal), int(allow_doubling), int(allow_halving))
        if rc:
            raise RuntimeError(f"orc_rebalance failed {rc}")

    def weight_magnitudes(self):
        out = np.empty(self.n_group * self.n_class)
        lib().orc_get_weight(self.ptr, _dp(out))
        return out.reshape(self.n_class, self.n_group).T

    def poisson_hist(self, mean, n, k_max):
        out = np.zeros(k_max + 1, dtype=np.int64)
        lib().orc_poisson_hist(self.ptr, mean, n, k_max, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        return out

    def binomial_hist(self, nn, p, n, k_max):
        out = np.zeros(k_max + 1, dtype=np.int64)
        lib().orc_binomial_hist(self.ptr, nn, p, n, k_max, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        return out


def kernel_value(kernel_type, v1, d1, v2, d2, temp=288.0, pressure=1e5, coeff=1000.0):
    return lib().orc_kernel_value(kernel_type, v1, d1, v2, d2, temp, pressure, coeff)


def vol2rad(v):
    return lib().orc_vol2rad(v)


def rad2vol(r):
    return lib().orc_rad2vol(r)


def fractal_radius(v, frac_dim, prime_radius, vol_fill_factor=1.0, temp=288.0, pressure=1e5):
    """(fractal_vol2rad, fractal_vol_to_mobility_rad) of volume v."""
    m = ctypes.c_double()
    r = lib().orc_fractal_radius(v, frac_dim, prime_radius, vol_fill_factor, temp, pressure, ctypes.byref(m))
    return r, m.value


def kernel_value_fractal(kernel_type, v1, d1, v2, d2, frac_dim, prime_radius, vol_fill_factor=1.0, temp=288.0,
                         pressure=1e5, coeff=1000.0):
    return lib().orc_kernel_value_fractal(kernel_type, v1, d1, v2, d2, temp, pressure, coeff, frac_dim,
                                          prime_radius, vol_fill_factor)


def bin_find(n_bin, emin, emax, r):
    return lib().orc_bin_find(n_bin, emin, emax, r)


def bin_grid_make(n_bin, rmin, rmax):
    e = np.empty(n_bin + 1)
    c = np.empty(n_bin)
    lib().orc_bin_grid_make(n_bin, rmin, rmax, _dp(e), _dp(c))
    return e, c


def student_t_95(n):
    return lib().orc_student_t_95(n)


def step_many(oracles, n_threads, kernel_type, temps, pressures, coeff, del_t, n_steps):
    arr = (ctypes.c_void_p * len(oracles))(*[o.ptr for o in oracles])
    t = np.ascontiguousarray(temps, dtype=np.float64)
    p = np.ascontiguousarray(pressures, dtype=np.float64)
    a = ctypes.c_int64()
    b = ctypes.c_int64()
    rc = lib().orc_step_many(arr, len(oracles), n_threads, kernel_type, _dp(t), _dp(p), coeff, del_t, n_steps,
                             ctypes.byref(a), ctypes.byref(b))
    if rc:
        raise RuntimeError(f"orc_step_many failed {rc}")
    return a.value, b.value
