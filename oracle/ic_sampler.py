"""Initial-condition sampler of the reference, restated for the CPU.

TEST INFRASTRUCTURE ONLY: the checker for a device sampler, never the product.

The reference fills an aerosol state from a distribution of modes with
``aero_state_add_aero_dist_sample`` (aero_state.F90:758-831): for every weight
group and mode, a Poisson number of particles with mean
``sample_prop * aero_mode_number`` (aero_mode.F90:495-546), each with a radius
from ``aero_mode_sample_radius`` (aero_mode.F90:550-630) and species volumes
from ``aero_mode_sample_vols`` (aero_mode.F90:633-665).  This module restates
those functions with draws from a numpy Generator, so it pins distributions,
not the reference's random stream.

Parity is pinned by known answers that follow from the mathematics, not by
reference fixtures (the reference has none for this path):
  * ``mode_number`` against direct quadrature of the mode's density divided by
    the weight;
  * the sampled radii against the weighted density (mean and spread of
    log10 r);
  * the truncation rule of ``rand_normal`` (rand.F90:410-487):
    1 - |erf(z / sqrt 2)| >= prob_threshold for every accepted draw;
  * volumes that sum to the particle's volume and are never negative.
"""
import math

import numpy as np

from .exact import rad2vol, vol2rad

MODE_LOG_NORMAL, MODE_EXP, MODE_MONO, MODE_SAMPLED = 1, 2, 3, 4  # aero_mode.F90:31-37
WEIGHT_NONE, WEIGHT_POWER, WEIGHT_MFA = 0, 1, 2
# rand_normal divides by 2.0**.5 (rand.F90:465, :478), a default-kind (single
# precision) constant
SQRT2_SINGLE = float(np.float32(math.sqrt(2.0)))
INFO_HALVED, INFO_WEIGHT = 3, 4  # aero_info.F90:19-28


class Weight:
    """aero_weight_t: type, magnitude (m^-3) and exponent."""

    def __init__(self, kind=WEIGHT_NONE, magnitude=1.0, exponent=0.0):
        self.kind, self.magnitude, self.exponent = kind, float(magnitude), float(exponent)

    def num_conc_at_radius(self, r):
        """aero_weight_num_conc_at_radius, aero_weight.F90:127-146."""
        if self.kind == WEIGHT_NONE:
            return self.magnitude * np.ones_like(np.asarray(r, dtype=np.float64))
        return self.magnitude * np.asarray(r, dtype=np.float64) ** self.exponent

    def radius_at_num_conc(self, nc):
        """aero_weight_radius_at_num_conc, aero_weight.F90:170-190."""
        if self.kind == WEIGHT_NONE or self.exponent == 0.0:
            raise ValueError("the weight cannot be inverted")
        return np.exp(np.log(nc / self.magnitude) / self.exponent)


class Mode:
    """aero_mode_t: type, characteristic radius (m), log10 of the geometric
    standard deviation, number concentration (m^-3), volume fractions and
    their standard deviations, and for sampled modes the radius edges and the
    number concentration of each interval."""

    def __init__(self, kind, char_radius=0.0, log10_std=0.0, num_conc=0.0, vol_frac=(1.0,), vol_frac_std=None,
                 sample_radius=None, sample_num_conc=None):
        self.kind = kind
        self.char_radius, self.log10_std, self.num_conc = float(char_radius), float(log10_std), float(num_conc)
        self.vol_frac = np.asarray(vol_frac, dtype=np.float64)
        self.vol_frac_std = (np.zeros_like(self.vol_frac) if vol_frac_std is None
                             else np.asarray(vol_frac_std, dtype=np.float64))
        self.sample_radius = None if sample_radius is None else np.asarray(sample_radius, dtype=np.float64)
        self.sample_num_conc = None if sample_num_conc is None else np.asarray(sample_num_conc, dtype=np.float64)


def weighted_sampled_num_conc(mode, w):
    """aero_mode_weighted_sampled_num_conc, aero_mode.F90:457-491.  The
    interval's number concentration, spread uniformly in ln r, divided by the
    weight and integrated.  At exponent 0 the reference's formula is 0/0; its
    limit, the unweighted concentration, is returned."""
    if w.kind == WEIGHT_NONE:
        return mode.sample_num_conc.copy()
    x0 = np.log(mode.sample_radius[:-1])
    x1 = np.log(mode.sample_radius[1:])
    if w.exponent == 0.0:
        return mode.sample_num_conc.copy()
    return mode.sample_num_conc / w.exponent * (np.exp(-w.exponent * x0) - np.exp(-w.exponent * x1)) / (x1 - x0)


def mode_number(mode, w):
    """aero_mode_number, aero_mode.F90:495-546: the expected number of
    computational particles of the mode per unit sample volume."""
    if mode.kind == MODE_LOG_NORMAL:
        if w.kind == WEIGHT_NONE:
            return mode.num_conc / w.magnitude
        x = math.log10(mode.char_radius)
        xp = x - w.exponent * mode.log10_std ** 2 * math.log(10.0)
        return mode.num_conc / w.magnitude * math.exp((xp ** 2 - x ** 2) / (2.0 * mode.log10_std ** 2))
    if mode.kind == MODE_EXP:
        if w.kind != WEIGHT_NONE:
            raise ValueError("cannot use exponential modes with weighting")
        return mode.num_conc / w.magnitude
    if mode.kind == MODE_MONO:
        return mode.num_conc / float(w.num_conc_at_radius(mode.char_radius))
    if mode.kind == MODE_SAMPLED:
        return float(weighted_sampled_num_conc(mode, w).sum()) / w.magnitude
    raise ValueError("unknown mode type")


def rand_normal(rng, mean, std, prob_threshold=None):
    """rand_normal, rand.F90:410-487 (Box-Muller form): redraw while
    1 - |erf(z0 / 2.0**.5)| < prob_threshold."""
    while True:
        u1, u2 = 1.0 - rng.random(), rng.random()  # u1 in (0, 1]
        z0 = math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)
        if prob_threshold is None or 1.0 - abs(math.erf(z0 / SQRT2_SINGLE)) >= prob_threshold:
            return std * z0 + mean


def sample_cts_pdf(rng, pdf):
    """sample_cts_pdf, rand.F90:550-576: accept-reject on an unnormalised
    density; returns a 0-based index."""
    pdf = np.asarray(pdf, dtype=np.float64)
    if pdf.min() < 0.0 or pdf.max() <= 0.0:
        raise ValueError("pdf must be non-negative with a positive entry")
    pmax = pdf.max()
    while True:
        k = int(rng.random() * len(pdf))
        if rng.random() < pdf[k] / pmax:
            return k


def sample_radius(rng, mode, w, prob_threshold):
    """aero_mode_sample_radius, aero_mode.F90:550-630."""
    if mode.kind == MODE_LOG_NORMAL:
        x = math.log10(mode.char_radius)
        xp = x if w.kind == WEIGHT_NONE else x - w.exponent * mode.log10_std ** 2 * math.log(10.0)
        return 10.0 ** rand_normal(rng, xp, mode.log10_std, prob_threshold)
    if mode.kind == MODE_SAMPLED:
        i = sample_cts_pdf(rng, weighted_sampled_num_conc(mode, w))
        if w.kind == WEIGHT_NONE or w.exponent == 0.0:
            x0, x1 = math.log(mode.sample_radius[i]), math.log(mode.sample_radius[i + 1])
            r = rng.random()
            return math.exp((1.0 - r) * x0 + r * x1)
        inv0 = 1.0 / float(w.num_conc_at_radius(mode.sample_radius[i]))
        inv1 = 1.0 / float(w.num_conc_at_radius(mode.sample_radius[i + 1]))
        r = rng.random()
        return float(w.radius_at_num_conc(1.0 / ((1.0 - r) * inv0 + r * inv1)))
    if mode.kind == MODE_EXP:
        if w.kind != WEIGHT_NONE:
            raise ValueError("cannot use exponential modes with weighting")
        return float(vol2rad(-rad2vol(mode.char_radius) * math.log(1.0 - rng.random())))
    if mode.kind == MODE_MONO:
        return mode.char_radius
    raise ValueError("unknown mode type")


def sample_vols(rng, mode, total_vol, max_loops=1000000):
    """aero_mode_sample_vols, aero_mode.F90:633-665: normal perturbations of
    the volume fractions projected back onto sum 1 along the mean fractions,
    redrawn until none is negative, then scaled to total_vol."""
    for _ in range(max_loops):
        v = np.array([rand_normal(rng, m, s) for m, s in zip(mode.vol_frac, mode.vol_frac_std)])
        v = v + (1.0 - v.sum()) * mode.vol_frac
        if v.min() >= 0.0:
            return v / v.sum() * total_vol
    raise RuntimeError("unable to sample non-negative volumes")


def add_dist_sample(rng, modes, weights, sample_prop, characteristic_factor=1.0):
    """aero_state_add_aero_dist_sample, aero_state.F90:758-831, for one
    weight class: for every group and mode, Poisson(sample_prop *
    mode_number) particles, the radius threshold min(1 / (characteristic
    factor * mean), 0.32).  Returns (vols (n, n_spec), group, mode index)."""
    vols, groups, mode_of = [], [], []
    for g, w in enumerate(weights):
        for m, mode in enumerate(modes):
            mean = sample_prop * mode_number(mode, w)
            if mean == 0.0:
                continue
            n = int(rng.poisson(mean))
            size_factor = min(1.0 / (characteristic_factor * mean), 0.32)
            for _ in range(n):
                r = sample_radius(rng, mode, w, size_factor)
                vols.append(sample_vols(rng, mode, float(rad2vol(r))))
                groups.append(g)
                mode_of.append(m)
    n_spec = len(modes[0].vol_frac) if modes else 1
    return (np.array(vols).reshape(-1, n_spec), np.array(groups, dtype=np.int32),
            np.array(mode_of, dtype=np.int32))


def prob_round(rng, val):
    """prob_round, rand.F90:214-227: floor or ceiling with mean val."""
    c = math.ceil(val)
    return int(math.floor(val)) if rng.random() < c - val else int(c)


class SampleState:
    """The parts of aero_state_t (aero_state.F90:69-84) the sampler touches:
    per particle the species volumes, 1-based weight group and class,
    component source, creation time and ID; the weights per (group, class)
    as a nested list weights[g-1][c-1]; n_part_ideal (n_group, n_class) or
    None; the removal records (id, action)."""

    def __init__(self, n_spec, weights, n_part_ideal=None, next_id=1):
        self.n_spec = n_spec
        self.weights = weights
        self.n_group, self.n_class = len(weights), len(weights[0])
        self.n_part_ideal = None if n_part_ideal is None else np.asarray(n_part_ideal, dtype=np.float64)
        self.vols, self.group, self.cls, self.source, self.ctime, self.id = [], [], [], [], [], []
        self.next_id = next_id
        self.removed = []

    def add(self, vols, g, c, source, create_time):
        self.vols.append(np.asarray(vols, dtype=np.float64))
        self.group.append(g)
        self.cls.append(c)
        self.source.append(source)
        self.ctime.append(create_time)
        self.id.append(self.next_id)
        self.next_id += 1

    def members(self, g, c):
        return [i for i in range(len(self.id)) if self.group[i] == g and self.cls[i] == c]

    def remove(self, idx, action):
        for i in sorted(idx, reverse=True):
            self.removed.append((self.id[i], action))
            for a in (self.vols, self.group, self.cls, self.source, self.ctime, self.id):
                del a[i]

    def arrays(self):
        return (np.array(self.vols).reshape(-1, self.n_spec), np.array(self.group, dtype=np.int32),
                np.array(self.cls, dtype=np.int32), np.array(self.source, dtype=np.int32),
                np.array(self.id, dtype=np.int64))


def scale_weight(rng, st, g, c, ratio, allow_doubling, allow_halving):
    """aero_state_scale_weight, aero_state.F90:1859-1922.  The halving branch
    removes prob_round(n (1 - 1/ratio)) members; the reference picks them
    one at a time uniformly from the shrinking list, which is a uniform
    subset of that size, drawn here at once.  The doubling branch ends each
    member as prob_round(1/ratio) particles (aero_state_dup_particle,
    :488-539)."""
    mem = st.members(g, c)
    n = len(mem)
    w = st.weights[g - 1][c - 1]
    if ratio > 1.0 and (allow_halving or n == 0):
        w.magnitude *= ratio
        n_remove = prob_round(rng, n * (1.0 - 1.0 / ratio))
        if n_remove > 0:
            st.remove(list(rng.choice(mem, n_remove, replace=False)), INFO_HALVED)
    elif ratio < 1.0 and (allow_doubling or n == 0):
        w.magnitude *= ratio
        gone = []
        for i in reversed(mem):
            k = prob_round(rng, 1.0 / ratio)
            if k == 0:
                gone.append(i)
            for _ in range(k - 1):
                st.add(st.vols[i], st.group[i], st.cls[i], st.source[i], st.ctime[i])
        st.remove(gone, INFO_WEIGHT)


def prepare_weight_for_add(rng, st, g, c, n_add, allow_doubling, allow_halving):
    """aero_state_prepare_weight_for_add, aero_state.F90:704-752 (one
    process)."""
    n_new = len(st.members(g, c)) + n_add
    if n_new == 0.0:
        return
    ideal = st.n_part_ideal[g - 1, c - 1]
    if n_new < ideal / 2.0 or n_new > ideal * 2.0:
        scale_weight(rng, st, g, c, n_new / ideal, allow_doubling, allow_halving)


def add_aero_dist_sample(rng, st, modes, sample_prop, characteristic_factor=1.0, create_time=0.0,
                         allow_doubling=True, allow_halving=True, sources=None, rad2vol_fn=rad2vol):
    """aero_state_add_aero_dist_sample, aero_state.F90:758-831, over a
    SampleState: for every group and mode, the weight prepared for the
    expected count (when n_part_ideal is set), then Poisson(sample_prop *
    aero_mode_number) particles.  The class is the mode's source when there
    is more than one class (aero_state_weight_class_for_source,
    aero_state.F90:263-282); sources default to mode index + 1.
    rad2vol_fn is aero_data_rad2vol (the particle shape).  Returns the
    number of particles added."""
    added = 0
    for g in range(1, st.n_group + 1):
        for m, mode in enumerate(modes):
            src = m + 1 if sources is None else sources[m]
            c = src if st.n_class > 1 else 1
            w = st.weights[g - 1][c - 1]
            n_avg = sample_prop * mode_number(mode, w)
            if st.n_part_ideal is not None:
                prepare_weight_for_add(rng, st, g, c, n_avg, allow_doubling, allow_halving)
            if n_avg == 0.0:
                continue
            w = st.weights[g - 1][c - 1]
            n_avg = sample_prop * mode_number(mode, w)
            n = int(rng.poisson(n_avg))
            size_factor = min(1.0 / (characteristic_factor * n_avg), 0.32)
            added += n
            for _ in range(n):
                r = sample_radius(rng, mode, w, size_factor)
                st.add(sample_vols(rng, mode, float(rad2vol_fn(r))), g, c, src, create_time)
    return added
