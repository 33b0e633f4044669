"""Host-side mirror of the reference's coagulation interface over the C ABI.

The names follow the reference: ``mc_coag(coag_kernel_type, env_state,
aero_data, aero_state, del_t) -> (tot_n_samp, tot_n_coag)``
(coagulation.F90:43-59), with ``AeroData``, ``AeroWeightArray``,
``EnvState`` and ``AeroState`` standing for aero_data_t, aero_weight_array_t,
env_state_t and aero_state_t.  An ``AeroState`` keeps its particles on the
GPU between calls; ``particles()`` copies them back.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import MODE_FP64, MODE_MIXED, MODE_REPLAY, check, dp, ip, lp

# coag_kernel.F90:29-45
COAG_KERNEL_TYPE_SEDI = 1
COAG_KERNEL_TYPE_ADDITIVE = 2
COAG_KERNEL_TYPE_CONSTANT = 3
COAG_KERNEL_TYPE_BROWN = 4
COAG_KERNEL_TYPE_ZERO = 5
COAG_KERNEL_TYPE_BROWN_FREE = 6
COAG_KERNEL_TYPE_BROWN_CONT = 7
KERNEL_NAMES = {"sedi": 1, "additive": 2, "constant": 3, "brown": 4, "zero": 5, "brown_free": 6, "brown_cont": 7}

# aero_weight.F90:24-30
AERO_WEIGHT_TYPE_NONE = 1
AERO_WEIGHT_TYPE_POWER = 2
AERO_WEIGHT_TYPE_MFA = 3

MAX_AERO_COMPONENT_SIZE = 20

# aero_mode.F90:31-37
AERO_MODE_TYPE_LOG_NORMAL = 1
AERO_MODE_TYPE_EXP = 2
AERO_MODE_TYPE_MONO = 3
AERO_MODE_TYPE_SAMPLED = 4


class Fractal:
    """Particle shape (fractal_t, fractal.F90:59-66): volume fractal dimension,
    primary-particle radius (m) and volume filling factor.  The defaults are
    spherical particles (fractal_set_spherical, fractal.F90:73-82)."""

    def __init__(self, frac_dim=3.0, prime_radius=1e-8, vol_fill_factor=1.0):
        self.frac_dim = float(frac_dim)
        self.prime_radius = float(prime_radius)
        self.vol_fill_factor = float(vol_fill_factor)

    @property
    def spherical(self):
        return self.frac_dim == 3.0 and self.vol_fill_factor == 1.0


class AeroData:
    """Species densities (kg/m^3), the water species index (1-based, 0 = none)
    and the particle shape (aero_data%fractal)."""

    def __init__(self, density, i_water=0, names=None, fractal=None):
        self.density = np.ascontiguousarray(np.atleast_1d(density), dtype=np.float64)
        self.i_water = int(i_water)
        self.names = names
        self.fractal = Fractal() if fractal is None else fractal

    @property
    def n_spec(self):
        return self.density.size


class AeroWeightArray:
    """weight(n_group, n_class) of (type, magnitude, exponent)
    (aero_weight_array.F90:35-39)."""

    def __init__(self, w_type, magnitude, exponent):
        self.type = np.asfortranarray(np.atleast_2d(w_type), dtype=np.int32)
        self.magnitude = np.asfortranarray(np.atleast_2d(magnitude), dtype=np.float64)
        self.exponent = np.asfortranarray(np.atleast_2d(exponent), dtype=np.float64)

    @property
    def n_group(self):
        return self.type.shape[0]

    @property
    def n_class(self):
        return self.type.shape[1]

    # aero_weight_array_set_flat / _set_power / _set_nummass, aero_weight_array.F90:66-118
    @classmethod
    def flat(cls, n_class=1, magnitude=1.0):
        return cls(np.full((1, n_class), AERO_WEIGHT_TYPE_NONE), np.full((1, n_class), magnitude),
                   np.zeros((1, n_class)))

    @classmethod
    def power(cls, exponent, n_class=1, magnitude=1.0):
        return cls(np.full((1, n_class), AERO_WEIGHT_TYPE_POWER), np.full((1, n_class), magnitude),
                   np.full((1, n_class), float(exponent)))

    @classmethod
    def nummass(cls, n_class=1, magnitudes=(1.0, 1.0)):
        t = np.array([[AERO_WEIGHT_TYPE_NONE] * n_class, [AERO_WEIGHT_TYPE_POWER] * n_class])
        m = np.array([[magnitudes[0]] * n_class, [magnitudes[1]] * n_class], dtype=np.float64)
        e = np.array([[0.0] * n_class, [-3.0] * n_class])
        return cls(t, m, e)

    def flat_arrays(self):
        return (np.ascontiguousarray(self.type.ravel(order="F")),
                np.ascontiguousarray(self.magnitude.ravel(order="F")),
                np.ascontiguousarray(self.exponent.ravel(order="F")))

    def num_conc_at_radius(self, i_class, radius):
        """aero_weight_array_num_conc_at_radius (aero_weight_array.F90:232-252),
        i_class 1-based, vectorised over radius."""
        r = np.asarray(radius, dtype=np.float64)
        inv = np.zeros_like(r)
        for g in range(self.n_group):
            t, m, e = self.type[g, i_class - 1], self.magnitude[g, i_class - 1], self.exponent[g, i_class - 1]
            nc = np.full_like(r, m) if t == AERO_WEIGHT_TYPE_NONE else m * r ** e
            inv = inv + 1.0 / nc
        return 1.0 / inv


class AeroMode:
    """aero_mode_t (aero_mode.F90:40-66): type, characteristic radius (m),
    log10 of the geometric standard deviation, number concentration
    (m^-3), species volume fractions and their standard deviations, the
    source, and for sampled modes the radius edges (m) and the number
    concentration (m^-3) of each interval."""

    def __init__(self, type, char_radius=0.0, log10_std_dev_radius=0.0, num_conc=0.0, vol_frac=(1.0,),
                 vol_frac_std=None, source=None, sample_radius=None, sample_num_conc=None):
        self.type = int(type)
        self.char_radius = float(char_radius)
        self.log10_std_dev_radius = float(log10_std_dev_radius)
        self.num_conc = float(num_conc)
        self.vol_frac = np.asarray(vol_frac, dtype=np.float64)
        self.vol_frac_std = (np.zeros_like(self.vol_frac) if vol_frac_std is None
                             else np.asarray(vol_frac_std, dtype=np.float64))
        self.source = source
        self.sample_radius = None if sample_radius is None else np.asarray(sample_radius, dtype=np.float64)
        self.sample_num_conc = None if sample_num_conc is None else np.asarray(sample_num_conc, dtype=np.float64)


class AeroDist:
    """aero_dist_t (aero_dist.F90:33-36): a list of modes."""

    def __init__(self, modes):
        self.mode = list(modes)


class EnvState:
    def __init__(self, temp=288.0, pressure=1e5, additive_kernel_coefficient=1000.0):
        self.temp = float(temp)
        self.pressure = float(pressure)
        self.additive_kernel_coefficient = float(additive_kernel_coefficient)


class AeroState:
    """Particle population(s) resident on the GPU (aero_state_t).

    ``n_pop > 1`` makes a batched state: independent populations with their
    own seeds that advance together in one step.
    """

    def __init__(self, aero_data, aero_weight_array, seed=1, mode=MODE_FP64, n_pop=1, seeds=None):
        self.aero_data = aero_data
        self.awa = aero_weight_array
        self.n_pop = int(n_pop)
        t, m, e = aero_weight_array.flat_arrays()
        L = _lib.lib()
        ctx = ctypes.c_void_p()
        if self.n_pop == 1 and seeds is None:
            rc = L.pmc_coag_gpu_init(aero_data.n_spec, dp(aero_data.density), aero_data.i_water,
                                     aero_weight_array.n_group, aero_weight_array.n_class, ip(t), dp(m), dp(e),
                                     int(seed), ctypes.byref(ctx))
        else:
            sd = np.ascontiguousarray(seeds if seeds is not None else np.arange(1, self.n_pop + 1) + int(seed) * 1000003,
                                      dtype=np.uint64)
            rc = L.pmc_coag_gpu_init_batch(self.n_pop, aero_data.n_spec, dp(aero_data.density), aero_data.i_water,
                                           aero_weight_array.n_group, aero_weight_array.n_class, ip(t), dp(m), dp(e),
                                           sd.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(ctx))
        check(rc, "pmc_coag_gpu_init")
        self.ctx = ctx
        self.set_mode(mode)
        if not aero_data.fractal.spherical:
            self.set_fractal(aero_data.fractal)

    def set_fractal(self, fractal):
        """Particle shape of every population (pmc_coag_gpu_set_fractal)."""
        check(_lib.lib().pmc_coag_gpu_set_fractal(self.ctx, fractal.frac_dim, fractal.prime_radius,
                                                  fractal.vol_fill_factor), "pmc_coag_gpu_set_fractal")

    def __del__(self):
        if getattr(self, "ctx", None):
            try:
                _lib.lib().pmc_coag_gpu_destroy(self.ctx)
            except (TypeError, AttributeError):
                pass  # interpreter shutdown: the module's globals are gone; the process's exit frees the device memory
            self.ctx = None

    def close(self):
        self.__del__()

    def set_mode(self, mode):
        check(_lib.lib().pmc_coag_gpu_set_mode(self.ctx, mode), "pmc_coag_gpu_set_mode")
        self.mode = mode

    def rebalance(self, n_part_ideal, allow_doubling=True, allow_halving=True, pop=0):
        """aero_state_rebalance (aero_state.F90:1797-1852) of population
        ``pop``; n_part_ideal per (group, class), or one number for all.
        Returns the population's weight magnitudes afterwards."""
        ideal = np.asfortranarray(np.broadcast_to(n_part_ideal, self.awa.magnitude.shape), dtype=np.float64)
        flat = np.ascontiguousarray(ideal.ravel(order="F"))
        check(_lib.lib().pmc_coag_gpu_rebalance(self.ctx, pop, dp(flat), int(bool(allow_doubling)),
                                                 int(bool(allow_halving))), "pmc_coag_gpu_rebalance")
        mag = self.weight_magnitudes(pop)
        if self.n_pop == 1:
            self.awa = AeroWeightArray(self.awa.type, mag, self.awa.exponent)
        return mag

    TUNE_SITES = ("test", "resolve", "items", "chain", "apply")

    def autotune(self, enable=True):
        """Make the next steps a search over the step's launch shapes
        (pmc_coag_gpu_autotune); tune_state() tells when it is done."""
        check(_lib.lib().pmc_coag_gpu_autotune(self.ctx, int(bool(enable))), "pmc_coag_gpu_autotune")

    def tune_state(self):
        """(tuning, {site: threads per block}, {site: [ms per candidate]})."""
        n = len(self.TUNE_SITES)
        tuning = ctypes.c_int()
        threads = np.zeros(n, dtype=np.int32)
        ms = np.zeros(3 * n, dtype=np.float32)
        check(_lib.lib().pmc_coag_gpu_tune_state(self.ctx, ctypes.byref(tuning), ip(threads),
                                                  ms.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
              "pmc_coag_gpu_tune_state")
        return (bool(tuning.value), dict(zip(self.TUNE_SITES, threads.tolist())),
                {k: ms[3 * i:3 * i + 3].tolist() for i, k in enumerate(self.TUNE_SITES)})

    def set_tune(self, threads):
        """Launch shapes found earlier: {site: threads per block}."""
        _, cur, _ = self.tune_state()
        cur.update(threads)
        a = np.array([cur[k] for k in self.TUNE_SITES], dtype=np.int32)
        check(_lib.lib().pmc_coag_gpu_set_tune(self.ctx, ip(a)), "pmc_coag_gpu_set_tune")

    def set_n_part_ideal(self, n_part):
        """aero_state_set_n_part_ideal (aero_state.F90:241-258): the ideal
        number of computational particles, split evenly over the weight
        groups and classes."""
        self.n_part_ideal = np.full(self.awa.magnitude.shape, float(n_part) / self.awa.magnitude.size)

    def add_aero_dist_sample(self, aero_dist, sample_prop=1.0, characteristic_factor=1.0, create_time=0.0,
                             allow_doubling=True, allow_halving=True, pop=0):
        """aero_state_add_aero_dist_sample (aero_state.F90:758-831) on the
        device (pmc_coag_gpu_add_dist_sample): a Poisson sample of the modes
        of ``aero_dist`` added to population ``pop``, the weights prepared
        for the ideal particle count when set_n_part_ideal was called.
        Returns the number of particles added."""
        modes = aero_dist.mode
        n_mode = len(modes)
        n_spec = self.aero_data.n_spec
        typ = np.array([m.type for m in modes], dtype=np.int32)
        rad = np.array([m.char_radius for m in modes], dtype=np.float64)
        std = np.array([m.log10_std_dev_radius for m in modes], dtype=np.float64)
        nc = np.array([m.num_conc for m in modes], dtype=np.float64)
        vf = np.zeros((max(n_mode, 1), n_spec))
        vfs = np.zeros((max(n_mode, 1), n_spec))
        for k, m in enumerate(modes):
            if m.vol_frac.size != n_spec or m.vol_frac_std.size != n_spec:
                raise ValueError("vol_frac and vol_frac_std need one entry per species")
            vf[k], vfs[k] = m.vol_frac, m.vol_frac_std
        src = np.array([k + 1 if m.source is None else int(m.source) for k, m in enumerate(modes)], dtype=np.int32)
        ns = np.array([0 if m.type != AERO_MODE_TYPE_SAMPLED else m.sample_num_conc.size for m in modes],
                      dtype=np.int32)
        sr = [m.sample_radius for m in modes if m.type == AERO_MODE_TYPE_SAMPLED]
        sn = [m.sample_num_conc for m in modes if m.type == AERO_MODE_TYPE_SAMPLED]
        sr = np.ascontiguousarray(np.concatenate(sr) if sr else np.zeros(1))
        sn = np.ascontiguousarray(np.concatenate(sn) if sn else np.zeros(1))
        ideal = getattr(self, "n_part_ideal", None)
        ideal_flat = None if ideal is None else np.ascontiguousarray(np.asarray(ideal).ravel(order="F"))
        n_add = ctypes.c_int64(0)
        check(_lib.lib().pmc_coag_gpu_add_dist_sample(
            self.ctx, pop, n_mode, ip(typ), dp(rad), dp(std), dp(nc), dp(np.ascontiguousarray(vf)),
            dp(np.ascontiguousarray(vfs)), ip(src), ip(ns), dp(sr), dp(sn), float(sample_prop),
            float(characteristic_factor), float(create_time), None if ideal_flat is None else dp(ideal_flat),
            int(bool(allow_doubling)), int(bool(allow_halving)), ctypes.byref(n_add)),
            "pmc_coag_gpu_add_dist_sample")
        if self.n_pop == 1:
            self.awa = AeroWeightArray(self.awa.type, self.weight_magnitudes(pop), self.awa.exponent)
        return int(n_add.value)

    def size_dist(self, n_bin, d_min, d_max, pop=0):
        """Number and per-species mass distributions on a log diameter grid
        (per unit ln D), computed on the device (pmc_coag_gpu_size_dist).
        Returns (num (n_bin,), mass (n_bin, n_spec))."""
        num = np.empty(n_bin)
        mass = np.empty((n_bin, self.aero_data.n_spec))
        check(_lib.lib().pmc_coag_gpu_size_dist(self.ctx, pop, int(n_bin), float(d_min), float(d_max), dp(num),
                                                 dp(mass)), "pmc_coag_gpu_size_dist")
        return num, mass

    def weight_magnitudes(self, pop=0):
        """Weight magnitudes (n_group, n_class) population ``pop`` uses now."""
        m = np.empty(self.awa.magnitude.size, dtype=np.float64)
        check(_lib.lib().pmc_coag_gpu_get_weight(self.ctx, pop, dp(m)), "pmc_coag_gpu_get_weight")
        return m.reshape(self.awa.magnitude.shape, order="F")

    def set_seed(self, seed, pop=0):
        """New seed for population ``pop``; its step counter restarts."""
        check(_lib.lib().pmc_coag_gpu_set_seed(self.ctx, pop, int(seed)), "pmc_coag_gpu_set_seed")

    def set_graphs(self, enable):
        """The later rounds of a step (retries, walks, chains) as one
        device-driven CUDA graph (default) or from a host loop; the particles
        are the same either way."""
        check(_lib.lib().pmc_coag_gpu_set_graphs(self.ctx, 1 if enable else 0), "pmc_coag_gpu_set_graphs")

    def set_weight(self, aero_weight_array):
        self.awa = aero_weight_array
        t, m, e = aero_weight_array.flat_arrays()
        check(_lib.lib().pmc_coag_gpu_set_weight(self.ctx, ip(t), dp(m), dp(e)), "pmc_coag_gpu_set_weight")

    def set_weight_pop(self, pop, aero_weight_array):
        """Weights of one population of a batched state."""
        t, m, e = aero_weight_array.flat_arrays()
        check(_lib.lib().pmc_coag_gpu_set_weight_pop(self.ctx, pop, ip(t), dp(m), dp(e)),
              "pmc_coag_gpu_set_weight_pop")

    def add_particles(self, vol, weight_group=None, weight_class=None, ids=None, n_primary_parts=None,
                      n_comp=None, comp_source=None, comp_create_time=None, pop=0):
        """Replace population ``pop`` by these particles.  vol: (n_part, n_spec)."""
        vol = np.ascontiguousarray(vol, dtype=np.float64)
        if vol.ndim == 1:
            vol = vol[:, None]
        n = vol.shape[0]
        as32 = lambda a: None if a is None else np.ascontiguousarray(np.broadcast_to(a, (n,)), dtype=np.int32)
        g, c, npp = as32(weight_group), as32(weight_class), as32(n_primary_parts)
        ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int64)
        rc = _lib.lib().pmc_coag_gpu_upload(self.ctx, pop, n, dp(vol), ip(g), ip(c), lp(ids), ip(npp))
        check(rc, "pmc_coag_gpu_upload")
        if n_comp is not None:
            nc = as32(n_comp)
            cs = np.ascontiguousarray(comp_source, dtype=np.int32).reshape(n, MAX_AERO_COMPONENT_SIZE)
            ct = np.ascontiguousarray(comp_create_time, dtype=np.float64).reshape(n, MAX_AERO_COMPONENT_SIZE)
            rc = _lib.lib().pmc_coag_gpu_upload_components(self.ctx, pop, n, ip(nc), ip(cs), dp(ct))
            check(rc, "pmc_coag_gpu_upload_components")

    def n_part(self, pop=0):
        n = ctypes.c_int()
        check(_lib.lib().pmc_coag_gpu_n_part(self.ctx, pop, ctypes.byref(n)), "pmc_coag_gpu_n_part")
        return n.value

    def particles(self, pop=0, components=False, out=None):
        """The particles of population ``pop`` (aero_state.F90 particle
        arrays, in slot order).  ``out``: optional dict of preallocated
        arrays (e.g. in pinned host memory) with room for every particle;
        the result then holds views of their first n_part rows."""
        n = self.n_part(pop)
        if out is None:
            out = {
                "vol": np.empty((n, self.aero_data.n_spec), dtype=np.float64),
                "weight_group": np.empty(n, dtype=np.int32),
                "weight_class": np.empty(n, dtype=np.int32),
                "id": np.empty(n, dtype=np.int64),
                "n_primary_parts": np.empty(n, dtype=np.int32),
            }
        else:
            for key, dt in (("vol", np.float64), ("weight_group", np.int32), ("weight_class", np.int32),
                            ("id", np.int64), ("n_primary_parts", np.int32)):
                a = out[key]
                if a.dtype != dt or not a.flags.c_contiguous or a.shape[0] < n:
                    raise ValueError(f"out[{key!r}] must be a C-contiguous {np.dtype(dt).name} array "
                                     f"with at least {n} rows")
            out = {k: v[:n] for k, v in out.items()}
        got = ctypes.c_int()
        rc = _lib.lib().pmc_coag_gpu_download(self.ctx, pop, n, dp(out["vol"]), ip(out["weight_group"]),
                                              ip(out["weight_class"]), lp(out["id"]), ip(out["n_primary_parts"]),
                                              ctypes.byref(got))
        check(rc, "pmc_coag_gpu_download")
        if components:
            out["n_comp"] = np.empty(n, dtype=np.int32)
            out["comp_source"] = np.empty((n, MAX_AERO_COMPONENT_SIZE), dtype=np.int32)
            out["comp_create_time"] = np.empty((n, MAX_AERO_COMPONENT_SIZE), dtype=np.float64)
            rc = _lib.lib().pmc_coag_gpu_download_components(self.ctx, pop, n, ip(out["n_comp"]),
                                                             ip(out["comp_source"]), dp(out["comp_create_time"]))
            check(rc, "pmc_coag_gpu_download_components")
        return out

    def set_next_id(self, next_id, pop=0):
        check(_lib.lib().pmc_coag_gpu_set_next_id(self.ctx, pop, int(next_id)), "pmc_coag_gpu_set_next_id")

    def next_id(self, pop=0):
        v = ctypes.c_int64()
        check(_lib.lib().pmc_coag_gpu_get_next_id(self.ctx, pop, ctypes.byref(v)), "pmc_coag_gpu_get_next_id")
        return v.value

    def set_replay(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        check(_lib.lib().pmc_coag_gpu_replay_set(self.ctx, dp(u), u.size), "pmc_coag_gpu_replay_set")

    def replay_used(self):
        v = ctypes.c_int64()
        check(_lib.lib().pmc_coag_gpu_replay_used(self.ctx, ctypes.byref(v)), "pmc_coag_gpu_replay_used")
        return v.value

    def stats(self):
        """Last step: k_max violations, events that lost a claim ("redraws":
        each was retried or dropped in the next round), rounds."""
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(_lib.lib().pmc_coag_gpu_stats(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
              "pmc_coag_gpu_stats")
        return {"kmax_violations": a.value, "redraws": b.value, "rounds": c.value}

    def set_record_removals(self, enable=True):
        """Keep removal records (aero_info_array) on the device from now on."""
        check(_lib.lib().pmc_coag_gpu_set_record_removals(self.ctx, int(bool(enable))),
              "pmc_coag_gpu_set_record_removals")

    def removals(self, pop=0, max_n=None):
        """Removal records of population ``pop`` since the last call (dict of
        id, action and other_id arrays; action codes of aero_info.F90:
        2 coagulation, 3 halved, 4 weight), cleared on the device."""
        n = ctypes.c_int64()
        cap = max(1024, 2 * self.n_part(pop)) if max_n is None else int(max_n)
        while True:
            ids = np.zeros(cap, np.int64)
            act = np.zeros(cap, np.int32)
            oth = np.zeros(cap, np.int64)
            rc = _lib.lib().pmc_coag_gpu_removals(self.ctx, pop, cap, lp(ids), ip(act), lp(oth), ctypes.byref(n))
            if rc == _lib.PMC_ERR_CAPACITY and n.value > cap and max_n is None:
                cap = n.value
                continue
            check(rc, "pmc_coag_gpu_removals")
            return {"id": ids[:n.value], "action": act[:n.value], "other_id": oth[:n.value]}

    def exact_tests(self):
        """Pair tests that MIXED mode decided in FP64 (near the uniform or
        near k_max), summed over the populations since their upload."""
        n = ctypes.c_int64()
        check(_lib.lib().pmc_coag_gpu_exact_tests(self.ctx, ctypes.byref(n)), "pmc_coag_gpu_exact_tests")
        return n.value

    def conflicts(self):
        v = [ctypes.c_int64() for _ in range(4)]
        check(_lib.lib().pmc_coag_gpu_conflicts(self.ctx, *[ctypes.byref(x) for x in v]), "pmc_coag_gpu_conflicts")
        return {"events": v[0].value, "event_losers": v[1].value, "target_ops": v[2].value,
                "target_op_losers": v[3].value}

    def sort(self, pop=0, max_bin=256):
        n = self.n_part(pop)
        nb = ctypes.c_int()
        edges = np.zeros(max_bin + 1)
        counts = np.zeros(max_bin * self.awa.n_class, dtype=np.int32)
        bins = np.zeros(max(n, 1), dtype=np.int32)
        rc = _lib.lib().pmc_coag_gpu_sort(self.ctx, pop, ctypes.byref(nb), dp(edges), max_bin, ip(counts), ip(bins))
        check(rc, "pmc_coag_gpu_sort")
        k = nb.value
        return edges[:k + 1], counts[:k * self.awa.n_class].reshape(self.awa.n_class, k).T, bins[:n]

    def kmax_table(self, coag_kernel_type, env_state, max_bin=256):
        out = np.zeros(max_bin * max_bin)
        rc = _lib.lib().pmc_coag_gpu_kmax_table(self.ctx, coag_kernel_type, env_state.temp, env_state.pressure,
                                                env_state.additive_kernel_coefficient, dp(out), max_bin)
        check(rc, "pmc_coag_gpu_kmax_table")
        return out

    def eval_kernel(self, coag_kernel_type, env_state, vol1, c1, vol2, c2, c_ij):
        vol1 = np.ascontiguousarray(vol1, dtype=np.float64)
        vol2 = np.ascontiguousarray(vol2, dtype=np.float64)
        n = vol1.shape[0]
        c1 = np.ascontiguousarray(np.broadcast_to(c1, (n,)), dtype=np.int32)
        c2 = np.ascontiguousarray(np.broadcast_to(c2, (n,)), dtype=np.int32)
        cij = np.ascontiguousarray(np.broadcast_to(c_ij, (n,)), dtype=np.int32)
        out = np.zeros(n)
        rc = _lib.lib().pmc_coag_gpu_eval_kernel(self.ctx, coag_kernel_type, env_state.temp, env_state.pressure,
                                                 env_state.additive_kernel_coefficient, n, dp(vol1), ip(c1),
                                                 dp(vol2), ip(c2), ip(cij), dp(out))
        check(rc, "pmc_coag_gpu_eval_kernel")
        return out


class HostMirror:
    """A host copy of one population kept slot by slot and brought up to date
    by copying only the slots written since the previous sync
    (pmc_coag_gpu_sync_host).  particles() gives the same arrays, in the same
    order, as AeroState.particles().  ``alloc`` makes the arrays (default
    numpy.empty; pass an allocator of page-locked memory to speed the first,
    full copy)."""

    def __init__(self, aero_state, pop=0, cap=None, alloc=None):
        self.st, self.pop = aero_state, pop
        self.alloc = alloc or (lambda shape, dtype: np.empty(shape, dtype=dtype))
        self.n_slots = 0
        self._make(cap if cap is not None else max(1024, 2 * aero_state.n_part(pop)))

    def _make(self, cap):
        ns = self.st.aero_data.n_spec
        self.cap = int(cap)
        self.vol = self.alloc((self.cap, ns), np.float64)
        self.group = self.alloc((self.cap,), np.int32)
        self.cls = self.alloc((self.cap,), np.int32)
        self.id = self.alloc((self.cap,), np.int64)
        self.n_primary = self.alloc((self.cap,), np.int32)
        self.alive = self.alloc((self.cap,), np.uint8)
        self.alive[:] = 0
        self._fresh = True

    def sync(self):
        """Bring the copy up to date; returns (slots copied, full copy?)."""
        ns, nc = ctypes.c_int(), ctypes.c_int()
        u8 = ctypes.POINTER(ctypes.c_uint8)
        while True:
            full = ctypes.c_int(1 if self._fresh else 0)
            rc = _lib.lib().pmc_coag_gpu_sync_host(
                self.st.ctx, self.pop, self.cap, dp(self.vol), ip(self.group), ip(self.cls), lp(self.id),
                ip(self.n_primary), self.alive.ctypes.data_as(u8), ctypes.byref(ns), ctypes.byref(nc),
                ctypes.byref(full))
            if rc == _lib.PMC_ERR_CAPACITY and ns.value > self.cap:
                self._make(2 * ns.value)  # regrown arrays: the next call copies every slot
                continue
            break
        check(rc, "pmc_coag_gpu_sync_host")
        self._fresh = False
        self.n_slots = ns.value
        return nc.value, bool(full.value)

    def particles(self):
        live = np.flatnonzero(self.alive[:self.n_slots])
        return {"vol": self.vol[live], "weight_group": self.group[live], "weight_class": self.cls[live],
                "id": self.id[live], "n_primary_parts": self.n_primary[live]}


def mc_coag(coag_kernel_type, env_state, aero_data, aero_state, del_t):
    """Do coagulation for time del_t (coagulation.F90:43-96).

    Returns (tot_n_samp, tot_n_coag), the reference's counters of samples
    tested and coagulation events.  Raises PmcError where the reference would
    stop (e.g. a coagulated particle outside the bin grid).
    """
    if aero_data is not aero_state.aero_data and aero_data.n_spec != aero_state.aero_data.n_spec:
        raise ValueError("aero_data does not match aero_state")
    a, b = ctypes.c_int(), ctypes.c_int()
    rc = _lib.lib().pmc_coag_gpu_step(aero_state.ctx, int(coag_kernel_type), env_state.temp, env_state.pressure,
                                      env_state.additive_kernel_coefficient, float(del_t), ctypes.byref(a),
                                      ctypes.byref(b))
    check(rc, "mc_coag")
    return a.value, b.value


def mc_coag_batch(coag_kernel_type, temps, pressures, additive_kernel_coefficient, aero_state, del_t, n_steps=1):
    """Advance every population of a batched AeroState by n_steps steps.
    Returns (tot_n_samp, tot_n_coag) summed over populations and steps."""
    t = np.ascontiguousarray(np.broadcast_to(temps, (aero_state.n_pop,)), dtype=np.float64)
    p = np.ascontiguousarray(np.broadcast_to(pressures, (aero_state.n_pop,)), dtype=np.float64)
    a, b = ctypes.c_int64(), ctypes.c_int64()
    rc = _lib.lib().pmc_coag_gpu_step_batch(aero_state.ctx, int(coag_kernel_type), dp(t), dp(p),
                                            float(additive_kernel_coefficient), float(del_t), int(n_steps),
                                            ctypes.byref(a), ctypes.byref(b))
    check(rc, "mc_coag_batch")
    return a.value, b.value
