"""Benchmark of the coagulation step (mc_coag) on B200.

Workload: 1e6 computational particles, 20 species with per-particle
Dirichlet(1) mass fractions and densities U(1000, 2000) kg/m^3, three
log-normal modes (D_g 0.02 / 0.1 / 0.5 um), nummass weighting, Brownian
kernel at 288 K and 1e5 Pa, del_t = 60 s.  A step is one mc_coag call on that
population; the metric is pair tests per second (the reference's tot_n_samp
counter) and simulated seconds per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank advances its own population (weak scaling, no
data-path collective); rank 0 prints one JSON line.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

B_TEST = 56  # algorithmic bytes per pair test: two cell-list entries and two 24-byte records
B_SORT = 8  # per slot: its cell key read, its cell-list entry written
# DRAM traffic per unit (dram__bytes_read.sum + dram__bytes_write.sum) from
# ncu captures of one launch at this workload: k_test read 27.29 MB and wrote
# 1.5 kB for about 209,000 tests; k_sort_all read 4.04 MB and wrote none for
# 1e6 slots.  The roofline's traffic scales these by the units of a launch.
DRAM_TEST = (27.29e6 + 1.5e3) / 209000
DRAM_SORT = 4.04e6 / 1e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-part", type=int, default=1_000_000)
    ap.add_argument("--del-t", type=float, default=60.0)
    ap.add_argument("--mode", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes instead of searching them on a copy of each workload")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--batch-pops", type=int, default=256)
    ap.add_argument("--batch-same", type=int, default=16)
    ap.add_argument("--serve-jobs", type=int, default=200)
    ap.add_argument("--no-graphs", action="store_true",
                    help="later rounds from the host loop instead of the CUDA graph (for launch lists)")
    ap.add_argument("--headline-only", action="store_true",
                    help="measure the headline step only (no FP64, batched or end-to-end lines)")
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(n_part, seed):
    from partmc_b200 import aero_dist
    return aero_dist.brown_20spec(n_part, seed=seed)


def tune_shapes(make_state, step, max_steps=64):
    """The autotuner's launch shapes for a workload, searched on a copy of
    it (untimed), so that the timed state starts from the workload itself.
    Returns (shapes, scores in ms per candidate)."""
    st = make_state()
    st.autotune()
    for _ in range(max_steps):
        if not st.tune_state()[0]:
            break
        step(st)
    _, shapes, scores = st.tune_state()
    st.close()
    return shapes, scores


def run_batched(pm, n_pop, steps, warmup, del_t, mode, seed=5, autotune=True):
    """Batched form: n_pop independent populations (log-uniform 1e3..1e5
    particles, per-population T, p and mode parameters, power weighting) in
    one context; every launch covers all populations.  Returns aggregate
    pair tests per second and simulated seconds per second."""
    import torch
    from partmc_b200 import aero_dist
    pops, temps, press = aero_dist.batched_bimodal(n_pop=n_pop, seed=seed)
    ad = pops[0].aero_data

    def make():
        st = pm.AeroState(ad, pops[0].awa, mode=mode, n_pop=n_pop)
        for k, p in enumerate(pops):
            st.set_weight_pop(k, p.awa)
            st.add_particles(p.vol, p.group, pop=k)
        return st

    shapes = None
    if autotune:
        shapes, _ = tune_shapes(make, lambda s: pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, s,
                                                                  del_t))
    st = make()
    if shapes:
        st.set_tune(shapes)
    for _ in range(warmup):
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, st, del_t)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    samp, _ = pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, st, del_t, n_steps=steps)
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    n_part = int(sum(p.n_part for p in pops))
    return ({"unit": "pair-tests/s", "populations": n_pop, "particles": n_part,
             "ms_per_step": 1e3 * sec / steps, "sim_s_per_s": n_pop * steps * del_t / sec,
             "rounds_last_step": st.stats()["rounds"], "launch_shapes": shapes}, samp, sec)


def run_batched_same(pm, n_pop, n_part, steps, warmup, del_t, mode, autotune=True):
    """n_pop independent copies (different seeds and samples) of the 1e6
    particle workload advanced together in one batched context."""
    import torch
    pops = [workload(n_part, seed=200 + k) for k in range(n_pop)]
    temps, press = np.full(n_pop, 288.0), np.full(n_pop, 1e5)

    def make():
        st = pm.AeroState(pops[0].aero_data, pops[0].awa, mode=mode, n_pop=n_pop)
        for k, p in enumerate(pops):
            # same densities (seeded); the weights depend on the sample
            st.set_weight_pop(k, p.awa)
            st.add_particles(p.vol, p.group, pop=k)
        return st

    shapes = None
    if autotune:
        shapes, _ = tune_shapes(make, lambda s: pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, s,
                                                                  del_t))
    st = make()
    if shapes:
        st.set_tune(shapes)
    for _ in range(warmup):
        pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, st, del_t)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    samp, _ = pm.mc_coag_batch(pm.COAG_KERNEL_TYPE_BROWN, temps, press, 0.0, st, del_t, n_steps=steps)
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    return ({"unit": "pair-tests/s", "populations": n_pop, "particles_each": n_part,
             "ms_per_step": 1e3 * sec / steps, "sim_s_per_s": n_pop * steps * del_t / sec,
             "launch_shapes": shapes}, samp, sec)


def fp32_error(pm, pop, env, n_pairs=200000, seed=3):
    """Largest relative error of the FP32 weighted kernel against the FP64
    one over random particle pairs of the workload (the acceptance of MIXED
    mode falls back to FP64 within 2^-12 of the uniform, far above it)."""
    rng = np.random.default_rng(seed)
    i = rng.integers(0, pop.n_part, n_pairs)
    j = rng.integers(0, pop.n_part, n_pairs)
    st = pm.AeroState(pop.aero_data, pop.awa, mode=pm.MODE_FP64)
    k64 = st.eval_kernel(pm.COAG_KERNEL_TYPE_BROWN, env, pop.vol[i], 1, pop.vol[j], 1, 1)
    st.set_mode(pm.MODE_MIXED)
    k32 = st.eval_kernel(pm.COAG_KERNEL_TYPE_BROWN, env, pop.vol[i], 1, pop.vol[j], 1, 1)
    ok = k64 > 0
    return float((np.abs(k32[ok] - k64[ok]) / k64[ok]).max())


def cpu_baseline(n_part, del_t, budget_s=20.0):
    """The oracle (C restatement of the reference's mc_coag), one thread, on
    a bounded sample of the same workload: as many steps as fit in budget_s."""
    from oracle import oracle as O
    pop = workload(n_part, seed=11)
    orc = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=5)
    orc.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
    orc.set_next_id(pop.n_part + 1)
    orc.mc_coag(4, 288.0, 1e5, 0.0, del_t)  # first step builds the k_max table: untimed
    steps, samp, t0 = 0, 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and steps < 1000:
        a, _ = orc.mc_coag(4, 288.0, 1e5, 0.0, del_t)
        samp += a
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": samp / dt, "unit": "pair-tests/s", "cores": 1, "kind": "port",
            "sample": f"{steps} steps of the 1e6-particle workload after one untimed step ({dt:.1f} s)",
            "sim_s_per_s": steps * del_t / dt}


def run_reference(args, ws, rank):
    """--impl reference: the reference's CPU algorithm (the oracle port, since
    the Fortran reference cannot be built here) on all host threads, one
    independent population per thread, same workload and metric."""
    if rank != 0:
        return
    from oracle import oracle as O
    n_thr = min(os.cpu_count() or 1, 32)
    orcs = []
    for k in range(n_thr):
        pop = workload(args.n_part, seed=100 + k)
        o = O.Oracle(pop.aero_data.density, (pop.awa.type, pop.awa.magnitude, pop.awa.exponent), seed=7 + k)
        o.add_particles(pop.vol, O.make_meta(pop.n_part, group=pop.group))
        o.set_next_id(pop.n_part + 1)
        orcs.append(o)
    temps = np.full(n_thr, 288.0)
    press = np.full(n_thr, 1e5)
    O.step_many(orcs, n_thr, 4, temps, press, 0.0, args.del_t, max(1, args.warmup))
    per_step = []
    tot = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        a, _ = O.step_many(orcs, n_thr, 4, temps, press, 0.0, args.del_t, 1)
        per_step.append(time.perf_counter() - t0)
        tot += a
    dt = sum(per_step)
    v = tot / dt
    line = {"metric": "coag pair-tests/s at 1e6 particles", "value": v, "unit": "pair-tests/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "brown_20spec_1e6_nummass", "n_part": args.n_part, "n_spec": 20,
                       "kernel": "brown", "del_t": args.del_t, "populations": n_thr,
                       "l2": "populations larger than L2"},
            "cpu_baseline": {"value": v, "unit": "pair-tests/s", "cores": n_thr, "kind": "port",
                             "sample": f"{n_thr} independent 1e6-particle populations, one per thread"},
            "e2e": {"value": v, "unit": "pair-tests/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "sim_s_per_s": args.steps * args.del_t * n_thr / dt}
    print(json.dumps(line))


def step_phases(prof, steps):
    """Where a step's device time goes, from the CUDA events around the
    phases: round 0 (sort, pair set-up, tests, resolve, apply, host
    read-backs between them) and the later rounds (the conditional graph of
    retries, walks and chains).  The later rounds are bound by the
    dependent loads of their slowest walk or chain, not by HBM; their
    per-kernel shares come from the ncu launch list."""
    step_ms = prof["step"][0] / max(steps, 1)
    later_ms = prof["redraw_graph"][0] / max(steps, 1)
    return {"round0_ms": step_ms - later_ms, "later_rounds_ms": later_ms,
            "later_rounds_share": later_ms / step_ms if step_ms > 0 else 0.0,
            "later_rounds_bound": "latency (dependent loads of walks and chains)",
            "test_ms": prof["test"][0] / max(steps, 1), "sort_ms": prof["sort"][0] / max(steps, 1)}


def aggregate(d, samp, sec, ws):
    """Whole-job form of a per-rank measurement: summed work over the
    slowest rank's time."""
    t = allreduce_max(sec, ws)
    d["value"] = allreduce_sum(samp, ws) / t
    return d


def run_ic_sample(pm, pop, n_part, ws, reps=3):
    import torch
    from partmc_b200 import aero_dist
    rng = np.random.default_rng(3)
    sig = rng.uniform(1.5, 2.0, size=3)
    n_spec = pop.aero_data.n_spec
    frac = np.full(n_spec, 1.0 / n_spec)
    modes = [pm.AeroMode(pm.AERO_MODE_TYPE_LOG_NORMAL, d / 2.0, np.log10(sig[k]), nc, vol_frac=frac,
                         vol_frac_std=0.1 * frac)
             for k, (d, nc) in enumerate(((0.02e-6, 1e10), (0.1e-6, 1e9), (0.5e-6, 1e8)))]
    dev_s, host_s, n_dev, n_host = [], [], 0, 0
    for k in range(reps):
        st = pm.AeroState(pop.aero_data, pm.AeroWeightArray.nummass(), seed=40 + k)
        st.set_n_part_ideal(n_part)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n_dev = st.add_aero_dist_sample(pm.AeroDist(modes))
        torch.cuda.synchronize()
        dev_s.append(time.perf_counter() - t0)
        del st
        st = pm.AeroState(pop.aero_data, pop.awa, seed=40 + k)
        t0 = time.perf_counter()
        hp = aero_dist.brown_20spec(n_part, seed=40 + k)
        st.add_particles(hp.vol, hp.group)
        n_host = hp.n_part
        torch.cuda.synchronize()
        host_s.append(time.perf_counter() - t0)
        del st
    return {"particles": n_dev, "device_ms": 1e3 * float(np.median(dev_s)),
            "particles_per_s": n_dev / float(np.median(dev_s)),
            "host_particles": int(n_host), "host_numpy_and_upload_ms": 1e3 * float(np.median(host_s)),
            "host_particles_per_s": n_host / float(np.median(host_s)),
            "what": "pmc_coag_gpu_add_dist_sample of three log-normal modes, 20 species with fraction "
                    "deviations, nummass weights prepared for the ideal count, wall clock with a device "
                    "synchronize; against numpy sampling on the host plus upload"}


def run_extras(args, pm, torch, pop, env, new_state, timed_steps, mode, ws):
    """Secondary lines: the plain FP64 step, the batched forms and the two
    end-to-end measurements through the C ABI."""
    out = {}
    # plain FP64 form of the same step, for the precision comparison
    k64 = max(3, args.steps // 2)
    st64 = new_state(pm.MODE_FP64)
    ms64, samp64, _, _ = timed_steps(st64, k64, args.warmup)
    del st64
    out["fp64_plain"] = aggregate({"unit": "pair-tests/s", "ms_per_step": ms64 / k64}, samp64, ms64 / 1e3, ws)
    kb = max(3, args.steps // 2)
    b, samp_b, sec_b = run_batched(pm, args.batch_pops, kb, args.warmup, args.del_t, mode,
                                   autotune=not args.no_autotune)
    out["batched"] = aggregate(b, samp_b, sec_b, ws)
    b, samp_b, sec_b = run_batched_same(pm, args.batch_same, args.n_part, kb, args.warmup, args.del_t, mode,
                                        autotune=not args.no_autotune)
    out["batched_1e6"] = aggregate(b, samp_b, sec_b, ws)

    # end to end through the C ABI with host buffers, the way a drop-in
    # mc_coag sees them: the population lives in pinned host memory; every
    # step uploads it, steps it and downloads it into the same buffers.
    def pinned(shape, dt):
        return torch.empty(shape, dtype=dt, pin_memory=True).numpy()

    cap_h = pop.n_part + pop.n_part // 2
    hb = {"vol": pinned((cap_h, pop.aero_data.n_spec), torch.float64),
          "weight_group": pinned((cap_h,), torch.int32), "weight_class": pinned((cap_h,), torch.int32),
          "id": pinned((cap_h,), torch.int64), "n_primary_parts": pinned((cap_h,), torch.int32)}
    n_h = pop.n_part
    hb["vol"][:n_h] = pop.vol
    hb["weight_group"][:n_h] = pop.group
    hb["weight_class"][:n_h] = 1
    hb["id"][:n_h] = np.arange(1, n_h + 1)
    hb["n_primary_parts"][:n_h] = 1
    ste = new_state(mode)

    def e2e_step():
        nonlocal n_h
        ste.add_particles(hb["vol"][:n_h], hb["weight_group"][:n_h], hb["weight_class"][:n_h], ids=hb["id"][:n_h],
                          n_primary_parts=hb["n_primary_parts"][:n_h])
        a, _ = pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, ste, args.del_t)
        got = ste.particles(out=hb)
        n_in = n_h
        n_h = got["id"].shape[0]
        return a, n_in, n_h

    for _ in range(args.warmup):
        e2e_step()
    barrier(ws)
    torch.cuda.synchronize()
    e2e_samp, h2d, d2h = 0, 0, 0
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        a, n_in, n_out = e2e_step()
        e2e_samp += a
        h2d += n_in * (8 * pop.aero_data.n_spec + 4 + 4 + 8 + 4)
        d2h += n_out * (8 * pop.aero_data.n_spec + 4 + 4 + 8 + 4)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    del ste

    # the drop-in for a coagulation-only run: the population stays in HBM and
    # the host's copy of it (slot by slot, in pinned memory) is brought up to
    # date after every step with the slots that step wrote; per step the host
    # passes temperature and pressure in and reads the counters and the
    # changed particles back
    str_ = new_state(mode)
    mirror = pm.HostMirror(str_, alloc=lambda shape, dt: pinned(shape, torch.from_numpy(np.empty(0, dt)).dtype))
    mirror.sync()  # the first, full copy: before the timed region
    rec = 8 * pop.aero_data.n_spec + 4 + 4 + 8 + 4 + 4 + 4  # vol, group, class, id, n_primary, slot, alive
    for _ in range(args.warmup):
        pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, str_, args.del_t)
        mirror.sync()
    barrier(ws)
    torch.cuda.synchronize()
    res_samp, res_d2h = 0, 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        a, _ = pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, str_, args.del_t)
        n_changed, _ = mirror.sync()
        res_samp += a
        res_d2h += 8 + n_changed * rec
    torch.cuda.synchronize()
    res_s = time.perf_counter() - t0
    del mirror, str_

    # the same resident path in FP64 mode, for an end-to-end figure at
    # matched precision
    str64 = new_state(pm.MODE_FP64)
    mirror = pm.HostMirror(str64, alloc=lambda shape, dt: pinned(shape, torch.from_numpy(np.empty(0, dt)).dtype))
    mirror.sync()
    for _ in range(args.warmup):
        pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, str64, args.del_t)
        mirror.sync()
    barrier(ws)
    torch.cuda.synchronize()
    r64_samp, r64_d2h = 0, 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        a, _ = pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, str64, args.del_t)
        n_changed, _ = mirror.sync()
        r64_samp += a
        r64_d2h += 8 + n_changed * rec
    torch.cuda.synchronize()
    r64_s = time.perf_counter() - t0
    del mirror, str64
    out["e2e_fp64"] = aggregate({"unit": "pair-tests/s", "h2d_bytes_per_step": 16,
                                 "d2h_bytes_per_step": int(r64_d2h / max(args.steps, 1)),
                                 "path": "as e2e, FP64 mode",
                                 "ms_per_step": 1e3 * r64_s / max(args.steps, 1)}, r64_samp, r64_s, ws)

    # the initial condition on the device: the benchmark's three log-normal
    # modes (20 species, fraction deviations 0.1 of each fraction) sampled
    # into an empty nummass state with an ideal of n_part particles
    # (aero_state_add_aero_dist_sample), against drawing the population in
    # numpy on the host and uploading it
    out["ic_sample"] = run_ic_sample(pm, pop, args.n_part, ws)

    # serving (cfg 5): Poisson arrivals at 50 jobs/s, 1e3..1e6 particles,
    # additive / Brownian / sedimentation, 10..200 steps each of the step
    # length of the reference's test for the kernel (serve.DEL_T: 1 s, 600 s,
    # 5 s), continuous batching within a 150 GB HBM budget
    from partmc_b200 import serve
    jobs = serve.poisson_jobs(args.serve_jobs, rate=50.0, seed=5 + 1000 * (ws > 1))
    srv = serve.Server([pm.COAG_KERNEL_TYPE_ADDITIVE, pm.COAG_KERNEL_TYPE_BROWN, pm.COAG_KERNEL_TYPE_SEDI],
                       slots=48, hbm_budget=150e9, mode=mode)
    serve.warm_up(srv)
    sm = serve.run(jobs, srv)
    del srv
    # each kernel at the step length of the reference's own test for it: at
    # 60 s an additive job (total volume fraction 4.2e-6, beta1 = 1000 1/s:
    # number decays as exp(-t / 240 s)) would coagulate to a few particles
    # within its steps
    del_t_s = {"additive": serve.DEL_T[pm.COAG_KERNEL_TYPE_ADDITIVE],
               "brownian": serve.DEL_T[pm.COAG_KERNEL_TYPE_BROWN],
               "sedimentation": serve.DEL_T[pm.COAG_KERNEL_TYPE_SEDI]}
    out["serving"] = aggregate(dict(sm, unit="pair-tests/s", rate_jobs_per_s=50.0, del_t_s=del_t_s),
                               sm["pair_tests_per_s"] * sm["wall_s"], sm["wall_s"], ws)

    out["e2e"] = aggregate({"unit": "pair-tests/s", "h2d_bytes_per_step": 16,
                            "d2h_bytes_per_step": int(res_d2h / max(args.steps, 1)),
                            "path": "mc_coag through the C ABI with the population resident in HBM; after every "
                                    "step the host copy (pinned, slot-indexed) is brought up to date with the "
                                    "slots the step wrote (pmc_coag_gpu_sync_host)",
                            "ms_per_step": 1e3 * res_s / max(args.steps, 1)}, res_samp, res_s, ws)
    out["e2e_full_sync"] = aggregate({"unit": "pair-tests/s",
                                      "h2d_bytes_per_step": int(h2d / max(args.e2e_steps, 1)),
                                      "d2h_bytes_per_step": int(d2h / max(args.e2e_steps, 1)),
                                      "path": "upload (pinned host) + mc_coag + download (pinned host) of the "
                                              "whole population every step through the C ABI",
                                      "ms_per_step": 1e3 * e2e_s / max(args.e2e_steps, 1)}, e2e_samp, e2e_s, ws)
    return out


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            barrier(ws)
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    from partmc_b200 import build
    build.build()
    import partmc_b200 as pm
    from partmc_b200 import _lib

    L = _lib.lib()
    mode = pm.MODE_MIXED if args.mode == "mixed" else pm.MODE_FP64
    pop = workload(args.n_part, seed=1 + rank)
    env = pm.EnvState(288.0, 1e5)

    shapes = {}

    def new_state(m):
        st = pm.AeroState(pop.aero_data, pop.awa, seed=1000 + rank, mode=m)
        st.set_graphs(not args.no_graphs)
        st.add_particles(pop.vol, pop.group)
        if m in shapes:
            st.set_tune(shapes[m][0])
        return st

    # the autotuner's launch shapes for the workload in each mode, searched on
    # a copy of it before anything is timed
    if not args.no_autotune:
        for m in (mode, pm.MODE_FP64):
            if m not in shapes:
                shapes[m] = tune_shapes(lambda: new_state(m), lambda s: pm.mc_coag(
                    pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, s, args.del_t))

    # L2 flush buffer (larger than the 126 MB L2), written between timed steps
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def timed_steps(st, k, w):
        for _ in range(w):
            pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, args.del_t)
        L.pmc_coag_gpu_profile(st.ctx, 1)
        exact0 = st.exact_tests()
        n0 = ctypes.c_int64()
        L.pmc_coag_gpu_launch_count(ctypes.byref(n0))
        barrier(ws)
        torch.cuda.synchronize()
        samp = 0
        ms = 0.0
        rounds = redraws = 0
        conf = {"events": 0, "event_losers": 0, "target_ops": 0, "target_op_losers": 0}
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            a, _ = pm.mc_coag(pm.COAG_KERNEL_TYPE_BROWN, env, pop.aero_data, st, args.del_t)
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            samp += a
            stt = st.stats()
            rounds += stt["rounds"]
            redraws += stt["redraws"]
            for kk, vv in st.conflicts().items():
                conf[kk] += vv
        n1 = ctypes.c_int64()
        L.pmc_coag_gpu_launch_count(ctypes.byref(n1))
        exact1 = st.exact_tests()
        prof = {}
        for which, name in ((0, "test"), (1, "sort"), (2, "redraw_graph"), (3, "step")):
            t, nl, u = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
            L.pmc_coag_gpu_profile_read(st.ctx, which, ctypes.byref(t), ctypes.byref(nl), ctypes.byref(u))
            prof[name] = (t.value, nl.value, u.value)
        L.pmc_coag_gpu_profile(st.ctx, 0)
        prof["exact_tests_per_step"] = (exact1 - exact0) / max(k, 1)
        prof["rounds_per_step"] = rounds / max(k, 1)
        prof["redraws_per_step"] = redraws / max(k, 1)
        prof["conflicts_per_step"] = {kk: vv / max(k, 1) for kk, vv in conf.items()}
        return ms, samp, n1.value - n0.value, prof

    clocks = ClockSampler(local)
    st = new_state(mode)
    clocks.start()
    ms, samp, launches, prof = timed_steps(st, args.steps, args.warmup)
    clk = clocks.stop()
    del st
    # whole-job aggregates: max time over ranks, summed work
    t_max = allreduce_max(ms / 1e3, ws)
    samp_all = allreduce_sum(samp, ws)
    extra = {}
    if not args.headline_only:
        extra = run_extras(args, pm, torch, pop, env, new_state, timed_steps, mode, ws)

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        ttest, ntest, utest = prof["test"]
        tsc, nsc, usc = prof["sort"]
        # dominant kernel by measured time
        if tsc >= ttest:
            dom, t_tot, n_l, units, bpu, dpu = "k_sort_all (cell counting sort)", tsc, nsc, usc, B_SORT, DRAM_SORT
        else:
            dom, t_tot, n_l, units, bpu, dpu = "k_test (pair tests)", ttest, ntest, utest, B_TEST, DRAM_TEST
        avg_ms = t_tot / max(n_l, 1)
        bytes_per_launch = units / max(n_l, 1) * bpu
        achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(args.n_part, args.del_t)
        line = {
            "metric": "coag pair-tests/s at 1e6 particles",
            "value": samp_all / t_max,
            "unit": "pair-tests/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if args.mode == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": "brown_20spec_1e6_nummass", "n_part": args.n_part, "n_spec": 20,
                       "kernel": "brown", "weighting": "nummass", "del_t": args.del_t,
                       "precision": "FP32 kernel eval/accept, FP64 k_max/merge/sums" if args.mode == "mixed"
                       else "FP64", "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": f"replicas x{ws}"},
            "sim_s_per_s": args.steps * args.del_t * ws / t_max,
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": units / max(n_l, 1) * dpu, "traffic_unit": "bytes per launch (ncu, scaled)",
                         "avg_launch_ms": avg_ms, "launches": n_l,
                         "bytes_per_unit": bpu, "units_per_launch": units / max(n_l, 1)},
            "kernel_ms": {k: {"total_ms": v[0], "launches": v[1], "units": v[2]} for k, v in prof.items()
                          if isinstance(v, tuple)},
            "precision": {"kernel_eval": "FP32" if args.mode == "mixed" else "FP64",
                          "fp32_kernel_max_rel_err": fp32_error(pm, pop, env),
                          "accept_margin": 2.0 ** -12,
                          "tests_decided_in_fp64_per_step": prof["exact_tests_per_step"],
                          "decisions": "identical to FP64 mode (FP64 fallback within the margin)"},
            "step_phases": step_phases(prof, args.steps),
            "autotune": ({"launch_shapes": shapes[mode][0], "scores_ms": shapes[mode][1],
                          "how": "coordinate search over threads per block at five launch sites, 3 steps per "
                                 "candidate on a copy of the workload, untimed (pmc_coag_gpu_autotune)"}
                         if mode in shapes else None),
            "rounds_per_step": prof["rounds_per_step"],
            "redraws_per_step": prof["redraws_per_step"],
            "conflicts_per_step": prof["conflicts_per_step"],
            "clocks": clk,
        }
        line.update(extra)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if ws > 1:
        barrier(ws)
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
