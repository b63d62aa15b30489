#!/usr/bin/env python
"""Benchmark of the short-range MD step: LJ particle-steps/s on one B200.

Workload (the large LJ fluid): N = 160^3 = 4,096,000 particles on a simple-cubic
lattice at reduced density 0.8442 with uniform jitter +-0.05 sigma (seed 1),
Maxwell-Boltzmann velocities at T = 1 (seed 2, zero net momentum), LJ eps = sigma = 1,
rc = 2.5 (auto shift), Verlet skin 0.3, cell grid 60^3, velocity Verlet dt = 0.005, NVE,
mixed precision (FP32 pair forces on box-wrapped int32 coordinates, int64 2^-32
fixed-point force sums, FP64 positions / velocities / energies).  Particle data
(262 MB of positions, velocities and packed coordinates) exceeds the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one velocity-Verlet step (force, aftCalcF, integrate2 + integrate1, and the
re-sort + Verlet rebuild whenever the accumulated displacement exceeds skin/2).  As the
workload prescribes, 1,000 Langevin steps (gamma 1, T 1) first melt the lattice into the
fluid; then W untimed NVE steps; the K timed NVE steps are one espp_run call whose step
loop is timed by CUDA events on the library's stream (max over ranks).  Under torchrun
each rank steps its own independent copy of the system on its GPU (replicas, weak
scaling).

The accuracy block compares the mixed-precision forces with the all-FP64 kernel on the
same positions, measures NVE energy drift of both precisions on a fixed 2,000-step
segment, and (1 GPU) compares the pair set of a list built inside the captured step loop
and the forces with the FP64 CPU oracle at 4,096,000 particles.  other_configs carries
the Kremer-Grest melt, the 32k LJ fluid and the 64 parallel-tempering replicas (batched
against sequential).

``--impl reference`` times the CPU restatement of the reference algorithm (the FP64
oracle; the reference itself cannot be built on this image: it needs Boost, MPI, FFTW
and HDF5) on all host cores, one independent 32,768-particle sample system per core at
the same density, cutoff and skin.  It steps the oracle's twin of the reference's vec
path (SoA cell arrays, packed candidates, src/vec/*), the faster of the reference's two
CPU paths; the GPU arm's cpu_baseline reports both, the vec twin as its value.
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

RHO = 0.8442
RC = 2.5
SKIN = 0.3
DT = 0.005
# neighbours within rc + skin, counted once per pair (half list): (2/3) pi (rc+skin)^3 rho
N_HALF = 2.0 / 3.0 * math.pi * (RC + SKIN) ** 3 * RHO
# algorithmic bytes per particle and step, whole step (mixed precision):
# x r/w 48 + v r/w 48 + int64 F w/r 48 + FP32 packed x w/r 24 + 4 B per half-list pair
STEP_BYTES = 168.0 + 4.0 * N_HALF
# algorithmic FLOPs per particle-step: 24 per half-list pair (3 sub, 5 for r^2, 1 rcp,
# 2 for r^6, 4 for the force factor, 3 for F, 6 accumulate)
STEP_FLOPS = 24.0 * N_HALF
# force kernel: packed coordinates read 12 + 4 B per half-list pair + int64 F write 24
FORCE_BYTES = 12.0 + 4.0 * N_HALF + 24.0
# DRAM bytes (read + write) per particle of one force-kernel launch, measured by ncu on
# the 1,000,000-particle case (profiles/force_mixed_lj_1M_ncu.txt: 345.0 MB + 6.7 MB for
# the global-list kernel); traffic grows in proportion to the particle count at fixed
# density
FORCE_TRAFFIC_PER_PARTICLE = {"k_force_mixed": 347.4}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def lattice(n_side, rho, jitter, seed):
    N = n_side ** 3
    L = (N / rho) ** (1.0 / 3.0)
    a = L / n_side
    g = (np.arange(n_side) + 0.5) * a
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.Generator(np.random.PCG64(seed))
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    return pos, L


def mb_velocities(N, T, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    v = rng.normal(0.0, math.sqrt(T), size=(N, 3))
    v *= math.sqrt(T / (np.sum(v * v) / (3 * N)))
    v -= v.mean(axis=0)
    return v


def make_system(lib, n_side, precision, seed=12345):
    from espressopp_b200._abi import call, dptr, i32ptr, i64ptr
    pos, L = lattice(n_side, RHO, 0.05, 1)
    vel = mb_velocities(len(pos), 1.0, 2)
    ids = np.arange(len(pos), dtype=np.int64)
    box = np.array([L, L, L])
    ncell = int(L / (RC + SKIN))
    cg = np.array([ncell] * 3, np.int32)
    h = ctypes.c_void_p()
    call(lib, "espp_system_create", dptr(box), SKIN, i32ptr(cg), precision, seed, ctypes.byref(h))
    call(lib, "espp_add_particles", h, len(ids), i64ptr(ids), None, None,
         dptr(np.ascontiguousarray(pos.reshape(-1))), dptr(np.ascontiguousarray(vel.reshape(-1))))
    call(lib, "espp_decompose", h)
    call(lib, "espp_vl_create", h, RC, 0, None)
    shift = 4.0 * (RC ** -12 - RC ** -6)
    call(lib, "espp_lj_set", h, 0, 0, 1.0, 1.0, RC, shift, 0.0)
    call(lib, "espp_integrator_set", h, DT)
    return h, ids, pos, vel, box, cg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0}, "fallback"


def max_over_ranks(dist, value, device="cuda"):
    """The largest of the ranks' values (every multi-GPU time is the max over ranks);
    `value` itself without a process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- CPU baseline (the oracle: a restatement of the reference algorithm) ------------
def _oracle_sample(args):
    """Steps one 32^3 sample system with the FP64 CPU oracle, through `entry`
    (espp_run: the classic AoS step; espp_vec_run: the vec SoA twin); returns
    (particle_steps, seconds).  Runs in its own process."""
    n_side, steps, budget_s, entry = args
    sys.path.insert(0, REPO)
    from espressopp_b200 import _abi
    lib_path = os.path.join(REPO, "oracle", "_build", "liboracle_espp.so")
    if not os.path.exists(lib_path):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle")])
    lib = _abi.bind(ctypes.CDLL(lib_path),
                    extra={"espp_vec_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int64])})
    h, ids, pos, vel, box, cg = make_system(lib, n_side, _abi.PREC_FP64)
    _abi.call(lib, entry, h, 1)  # decompose + list build outside the timing
    done = 0
    t0 = time.perf_counter()
    while True:
        _abi.call(lib, entry, h, steps)
        done += steps
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    lib.espp_system_destroy(h)
    return done * n_side ** 3, el


def cpu_baseline(cores, budget_s=12.0, n_side=32, steps=4, entry="espp_vec_run"):
    import multiprocessing as mp
    if cores == 1:
        ps, el = _oracle_sample((n_side, steps, budget_s, entry))
        return ps / el, 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        t0 = time.perf_counter()
        res = pool.map(_oracle_sample, [(n_side, steps, budget_s, entry)] * cores)
        wall = time.perf_counter() - t0
    # aggregate rate over the longest worker's timed span
    return sum(r[0] for r in res) / max(r[1] for r in res), cores


def reference_arm(args, rank, world):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    rates = []
    for _ in range(max(1, args.steps_ref)):
        r, c = cpu_baseline(cores, budget_s=args.ref_budget)
        rates.append(r)
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": "LJ particle-steps/s", "value": value,
        "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "LJ fluid 160^3 (rho 0.8442, rc 2.5, skin 0.3, dt 0.005, NVE)",
                   "sample": "32^3 = 32768-particle systems at the same density, cutoff and skin, "
                             "one per host core"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores,
                         "kind": "port",
                         "sample": "%d cores x independent 32768-particle systems, %.0f s each, "
                                   "vec SoA twin of the oracle" % (cores, args.ref_budget)},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    emit(line)


# ---- GPU arm ---------------------------------------------------------------------
def gpu_arm(args, rank, world, local_rank):
    import espressopp_b200
    from espressopp_b200 import _abi
    from espressopp_b200._abi import call, dptr, i64ptr

    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(local_rank)
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = dist_mod

    lib = espressopp_b200.load_library()
    call(lib, "espp_select_device", local_rank)
    prec = _abi.PREC_MIXED if args.precision == "mixed" else _abi.PREC_FP64
    t_setup = time.perf_counter()
    h, ids, pos, vel, box, cg = make_system(lib, args.n_side, prec)
    N = len(ids)
    log("rank %d: setup %.1f s, N=%d, cells %s" % (rank, time.perf_counter() - t_setup, N,
                                                   tuple(cg)))

    def barrier():
        if dist is not None:
            import torch
            t = torch.zeros(1, device="cuda")
            dist.all_reduce(t)
            torch.cuda.synchronize()

    # the workload's protocol: 1,000 Langevin steps (gamma 1, T 1) melt the lattice into
    # the equilibrated fluid; the timed segment is NVE from that state
    t_eq = time.perf_counter()
    steps_per_build = 10.0
    if args.equil > 0:
        call(lib, "espp_langevin_set", h, 1, 1.0, 1.0, 0, None)
        call(lib, "espp_run", h, args.equil)
        call(lib, "espp_langevin_set", h, 0, 1.0, 1.0, 0, None)
        rs = ctypes.c_int64()
        call(lib, "espp_num_resorts", h, ctypes.byref(rs))
        steps_per_build = args.equil / max(1, rs.value)
    log("rank %d: %d Langevin steps in %.1f s" % (rank, args.equil, time.perf_counter() - t_eq))
    # warm-up (untimed), then the list layout: per-particle global lists (1, 2, 4, 8
    # threads per particle) or brick windows of several extents, each timed (one build,
    # three force launches) and scored by force time + build time / steps per build
    call(lib, "espp_run", h, args.warmup)
    layout, tune = autotune_layout(lib, h, args, steps_per_build)
    log("rank %d: layout %s (steps per build %.1f)" % (rank, layout, steps_per_build))

    def total_energy(hh):
        e = ctypes.c_double()
        call(lib, "espp_energy", hh, 0, ctypes.byref(e))
        v2 = ctypes.c_double()
        nn = ctypes.c_int64()
        call(lib, "espp_kinetic", hh, ctypes.byref(v2), ctypes.byref(nn))
        return e.value + 0.5 * v2.value

    log("rank %d: timed run" % rank)
    # timed region: one run of K steps on the captured step-loop graph; CUDA events on
    # the library's stream around the step loop
    call(lib, "espp_set_profiling", h, 0)
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    barrier()
    call(lib, "espp_run", h, args.steps)
    barrier()
    clocks = sampler.stop()
    ms = np.zeros(2)
    call(lib, "espp_last_run_ms", h, dptr(ms))
    ph_g = np.zeros(8)
    launches = np.zeros(8, np.int64)
    call(lib, "espp_profile", h, dptr(ph_g), i64ptr(launches))
    resorts = ctypes.c_int64()
    call(lib, "espp_num_resorts", h, ctypes.byref(resorts))
    loop_ms = max_over_ranks(dist, float(ms[1]))


    log("rank %d: profiled pass" % rank)
    # per-kernel device times: the same workload stepped K more steps with every launch
    # bracketed by CUDA events on the library's stream (host-driven loop)
    call(lib, "espp_set_profiling", h, 1)
    call(lib, "espp_run", h, args.steps)
    ph = np.zeros(8)
    launches_p = np.zeros(8, np.int64)
    call(lib, "espp_profile", h, dptr(ph), i64ptr(launches_p))
    call(lib, "espp_set_profiling", h, 0)

    log("rank %d: end-to-end pass" % rank)
    # end to end through the C ABI with pinned host buffers: state in, K steps, state out
    import torch
    pin_pos = torch.empty((N, 3), dtype=torch.float64, pin_memory=True).numpy()
    pin_vel = torch.empty((N, 3), dtype=torch.float64, pin_memory=True).numpy()
    pin_ids = torch.empty((N,), dtype=torch.int64, pin_memory=True).numpy()
    pin_ids[:] = ids
    call(lib, "espp_get_particles", h, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel), None,
         None)
    barrier()
    t0 = time.perf_counter()
    call(lib, "espp_set_particles", h, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel))
    call(lib, "espp_run", h, args.steps)
    call(lib, "espp_get_particles", h, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel), None,
         None)
    barrier()
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0)

    log("rank %d: FP64 comparison" % rank)
    # mixed vs all-FP64 GPU on the same positions: force error and step throughput
    cmp = {}
    if prec == _abi.PREC_MIXED and not args.no_fp64:
        h64 = make_system(lib, args.n_side, _abi.PREC_FP64)[0]
        call(lib, "espp_set_particles", h64, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel))
        call(lib, "espp_run", h64, 0)
        call(lib, "espp_run", h, 0)
        f32 = np.zeros((N, 3))
        f64 = np.zeros((N, 3))
        call(lib, "espp_get_particles", h, N, i64ptr(pin_ids), None, None, dptr(f32), None)
        call(lib, "espp_get_particles", h64, N, i64ptr(pin_ids), None, None, dptr(f64), None)
        df = f32 - f64
        rel_rms = float(np.sqrt(np.sum(df * df) / np.sum(f64 * f64)))
        rel_max = float(np.max(np.linalg.norm(df, axis=1)) /
                        np.sqrt(np.mean(np.sum(f64 * f64, axis=1))))
        call(lib, "espp_run", h64, args.warmup)
        layout64, tune64 = autotune_layout(lib, h64, args, steps_per_build)
        # throughput of the all-FP64 kernel: the same K NVE steps from the same state
        call(lib, "espp_set_particles", h64, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel))
        call(lib, "espp_run", h64, 0)
        barrier()
        call(lib, "espp_run", h64, args.steps)
        barrier()
        ms64 = np.zeros(2)
        call(lib, "espp_last_run_ms", h64, dptr(ms64))
        loop64 = max_over_ranks(dist, float(ms64[1]))
        # NVE drift on a fixed segment, both precisions from the same state
        call(lib, "espp_set_particles", h64, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel))
        call(lib, "espp_set_particles", h, N, i64ptr(pin_ids), dptr(pin_pos), dptr(pin_vel))
        call(lib, "espp_run", h64, 0)
        call(lib, "espp_run", h, 0)
        e64_before = total_energy(h64)
        e32_before = total_energy(h)
        call(lib, "espp_run", h64, args.drift_steps)
        call(lib, "espp_run", h, args.drift_steps)
        drift64 = (total_energy(h64) - e64_before) / N / (args.drift_steps * DT)
        drift32 = (total_energy(h) - e32_before) / N / (args.drift_steps * DT)
        lib.espp_system_destroy(h64)
        cmp = {"force_rel_rms_err": rel_rms, "force_rel_max_err": rel_max,
               "force_rel_max_err_definition": "max over particles of |F_mixed - F_fp64| "
                                                "divided by the RMS force",
               "fp64_value": world * N * args.steps / (loop64 * 1e-3),
               "fp64_ms_per_step": loop64 / args.steps,
               "mixed_over_fp64": loop64 / loop_ms,
               "fp64_layout": layout64,
               "nve_drift_per_particle_per_tau": {
                   "mixed": drift32, "fp64": drift64, "e0_per_particle": e64_before / N,
                   "segment_steps": args.drift_steps,
                   "definition": "(E_after - E_before) / N / (steps dt), both precisions "
                                 "stepping the same NVE segment from the same equilibrated "
                                 "state"}}
        if rank == 0 and world == 1 and not args.no_oracle:
            cmp.update(oracle_parity(lib, h, ids, box))

    lib.espp_system_destroy(h)
    if rank == 0:
        log("LJ: %.4g particle-steps/s, %.4f ms/step%s" % (
            world * N * args.steps / (loop_ms * 1e-3), loop_ms / args.steps,
            ", mixed/fp64 %.3f" % cmp["mixed_over_fp64"] if "mixed_over_fp64" in cmp else ""))
    configs = (small_configs(lib, args.replica_steps, args.cg_small)
               if (rank == 0 and world == 1 and not args.no_configs) else None)
    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    peaks, peak_kind = measured_peaks()
    hbm = float(peaks["hbm_gbs"])
    fp32 = ctypes.c_double()
    call(lib, "espp_fp32_peak", ctypes.byref(fp32))
    force_avg_ms = ph[0] / max(1, launches_p[0])
    achieved = FORCE_BYTES * N / (force_avg_ms * 1e-3) / 1e9
    step_s = loop_ms * 1e-3 / args.steps
    value = world * N * args.steps / (loop_ms * 1e-3)
    cpu_rate, cpu_cores = cpu_baseline(1, budget_s=args.cpu_budget) if world == 1 else (None, 1)
    cpu_classic = (cpu_baseline(1, budget_s=args.cpu_budget, entry="espp_run")[0]
                   if world == 1 else None)
    force_kernel = ("k_force_brick_" if layout["form"] == "brick" else "k_force_") + \
        ("mixed" if prec else "fp64")
    tr = FORCE_TRAFFIC_PER_PARTICLE.get(force_kernel)
    traffic = tr * N if tr else None
    line = {
        "metric": "LJ particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": loop_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if prec else "f64",
        "dtype_detail": "pair forces f32 on int32 box-wrapped coordinates, int64 2^-32 "
                        "fixed-point force sums, f64 positions/velocities/energies"
                        if prec else "all f64",
        "data": "synthetic",
        "config": {"workload": "LJ fluid, %d^3 = %d particles, rho %.4f, rc %.1f, skin %.1f, "
                               "dt %.3f, NVE, %s" % (args.n_side, N, RHO, RC, SKIN, DT,
                                                     args.precision),
                   "cell_grid": list(map(int, cg)), "l2": "inputs larger than L2 (262 MB)",
                   "parallelism": "replicas x%d" % world if world > 1 else "1 GPU",
                   "resorts_in_timed_steps": int(resorts.value),
                   "layout": layout, "steps_per_build": steps_per_build,
                   "autotune": tune},
        "roofline": {"kernel": force_kernel, "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "alg_bytes_per_particle": FORCE_BYTES, "traffic": traffic,
                     "avg_launch_ms": force_avg_ms},
        "step_roofline": {"alg_bytes_per_particle_step": STEP_BYTES,
                          "achieved_gbs": STEP_BYTES * N / step_s / 1e9,
                          "frac": STEP_BYTES * N / step_s / 1e9 / hbm},
        "step_flop_roofline": {"alg_flops_per_particle_step": STEP_FLOPS,
                               "achieved_tflops": STEP_FLOPS * N / step_s / 1e12,
                               "peak_tflops": fp32.value,
                               "frac": (STEP_FLOPS * N / step_s / 1e12 / fp32.value
                                        if fp32.value > 0 else None),
                               "peak_kind": "measured FP32 FMA throughput (probe kernel)"},
        "profiled_pass_ms": {"force": ph[0], "integrate": ph[1], "resort": ph[2],
                             "decide": ph[3], "verlet_build": ph[4],
                             "launches": [int(x) for x in launches_p[:5]]},
        "gpu_launches": int(launches.sum()),
        "accuracy": dict(cmp, note="forces of the mixed and the all-FP64 kernel on identical "
                                   "positions of the equilibrated fluid"),
        "clocks": clocks,
        "other_configs": configs,
        "e2e": {"value": world * N * args.steps / e2e_s, "unit": "particle-steps/s",
                "h2d_bytes_per_step": int(N * (48 + 8) / args.steps),
                "d2h_bytes_per_step": int(N * 48 / args.steps),
                "note": "pinned host state in (ids, x, v), K steps, state out (x, v) per call"},
    }
    if cpu_rate is not None:
        line["cpu_baseline"] = {"value": cpu_rate, "unit": "particle-steps/s", "cores": cpu_cores,
                                "kind": "port",
                                "sample": "one 32768-particle system (same density, rc, skin), "
                                          "%.0f s of stepping on 1 core, vec SoA twin of the "
                                          "oracle" % args.cpu_budget,
                                "classic_aos_value": cpu_classic}
    emit(line)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def autotune_layout(lib, h, args, steps_per_build):
    """espp_autotune_layout (or the layout forced by --layout): returns the layout in use
    {form, tpp, brick} and the timed candidates."""
    from espressopp_b200._abi import call, dptr, i32ptr
    best = np.zeros(5, np.int32)
    table = np.zeros((32, 8))
    n = ctypes.c_int32(0)
    if args.layout == "auto":
        call(lib, "espp_autotune_layout", h, steps_per_build, i32ptr(best), dptr(table), 32,
             ctypes.byref(n))
    else:
        form = {"global": 0, "brick": 1, "global-brick-build": 2}[args.layout]
        b = np.zeros(3, np.int32)
        call(lib, "espp_set_layout", h, form, max(1, args.tpp), i32ptr(b))
        call(lib, "espp_get_layout", h, i32ptr(best))
    names = {0: "global", 1: "brick", 2: "global-brick-build"}
    lay = {"form": names[int(best[0])], "threads_per_particle": int(best[1]),
           "brick": [int(x) for x in best[2:5]]}
    rows = [{"form": names[int(r[0])], "threads_per_particle": int(r[1]),
             "brick": [int(x) for x in r[2:5]], "force_ms": float(r[5]),
             "build_ms": float(r[6]), "score_ms": float(r[7])} for r in table[:n.value]]
    return lay, rows


def oracle_parity(lib, h, ids, box):
    """The running system's Verlet pair set and mixed-precision forces against the FP64
    oracle (the CPU restatement of VerletList.cpp:274-450 and the LJ loop) at the same
    positions.  The system is stepped until a re-sort happens inside the captured step
    loop, so the list in use was built at the positions the run ends on; the pair sets
    are compared through espp_vl_digest (each unordered pair once, by id)."""
    from espressopp_b200 import _abi
    from espressopp_b200._abi import call, dptr, i32ptr, i64ptr
    log("oracle parity: stepping to an in-graph re-sort")
    N = len(ids)
    r1 = ctypes.c_int64()
    steps = 0
    for steps in range(1, 41):
        call(lib, "espp_run", h, 1)
        call(lib, "espp_num_resorts", h, ctypes.byref(r1))  # re-sorts of this run
        if r1.value > 0:
            break
    x = np.zeros((N, 3))
    f = np.zeros((N, 3))
    call(lib, "espp_get_particles", h, N, i64ptr(ids), dptr(x), None, dptr(f), None)
    dg = (ctypes.c_uint64 * 4)()
    call(lib, "espp_vl_digest", h, dg)
    t0 = time.perf_counter()
    olib = _abi.bind(ctypes.CDLL(os.path.join(REPO, "oracle", "_build", "liboracle_espp.so")))
    ho = ctypes.c_void_p()
    cg = np.array([int(b / (RC + SKIN)) for b in box], np.int32)
    call(olib, "espp_system_create", dptr(np.asarray(box, np.float64)), SKIN, i32ptr(cg), 0, 1,
         ctypes.byref(ho))
    call(olib, "espp_add_particles", ho, N, i64ptr(ids), None, None,
         dptr(np.ascontiguousarray(x.reshape(-1))), None)
    call(olib, "espp_decompose", ho)
    call(olib, "espp_vl_create", ho, RC, 0, None)
    call(olib, "espp_lj_set", ho, 0, 0, 1.0, 1.0, RC, 4.0 * (RC ** -12 - RC ** -6), 0.0)
    call(olib, "espp_integrator_set", ho, DT)
    call(olib, "espp_run", ho, 0)
    do = (ctypes.c_uint64 * 4)()
    call(olib, "espp_vl_digest", ho, do)
    fo = np.zeros((N, 3))
    call(olib, "espp_get_particles", ho, N, i64ptr(ids), None, None, dptr(fo), None)
    olib.espp_system_destroy(ho)
    df = f - fo
    log("oracle parity: %d pairs, digests %s, %.1f s" %
        (do[0], "equal" if list(dg) == list(do) else "DIFFER", time.perf_counter() - t0))
    return {"pairs_bit_exact_vs_oracle": list(dg) == list(do) and r1.value > 0,
            "pairs_vs_oracle": {"pairs": int(do[0]), "steps_to_in_graph_resort": steps,
                                "compared": "espp_vl_digest (count, sum, xor, sum2 of 64-bit "
                                            "pair hashes)"},
            "force_rel_rms_err_vs_oracle": float(np.sqrt(np.sum(df * df) / np.sum(fo * fo))),
            "force_rel_max_err_vs_oracle": float(np.max(np.linalg.norm(df, axis=1)) /
                                                 np.sqrt(np.mean(np.sum(fo * fo, axis=1))))}


# ---- the smaller configurations: Kremer-Grest melt and 32k LJ fluid ----------------
def kg_melt_config(lib, prec, nchains=200, nbeads=200, cap_steps=1000, steps=9000):
    """Kremer-Grest melt: nchains x nbeads beads at density 0.85 (random walks, bond 0.97,
    overlaps < 0.8 rejected; tools.topology.polymer_melt, seed 3), WCA (rc 2^(1/6), auto
    shift) + FENE (K 30, R0 1.5), dt 0.01, Langevin gamma 0.5 T 1.  The first cap_steps
    steps cap the pair force (LennardJonesCapped, caprad 0.9) so that the growth overlaps
    relax while FENE keeps every bond below R0 (a cap on the total force would let bonds
    stretch past R0, where FENE turns repulsive); then `steps` more with plain WCA.
    The list layout is the autotuner's choice at the start (before the timed steps).
    Returns device-timed throughput and end-state observables."""
    from espressopp_b200._abi import call, dptr, i32ptr, i64ptr
    from espressopp_b200.tools import topology
    pos, bonds, L = topology.polymer_melt(nchains, nbeads, 0.85, seed=3)
    rc = 2.0 ** (1.0 / 6.0)
    box = np.array([L, L, L])
    cg = np.array([int(L / (rc + SKIN))] * 3, np.int32)
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    h = ctypes.c_void_p()
    call(lib, "espp_system_create", dptr(box), SKIN, i32ptr(cg), prec, 77, ctypes.byref(h))
    call(lib, "espp_add_particles", h, len(ids), i64ptr(ids), None, None,
         dptr(np.ascontiguousarray(pos.reshape(-1))), None)
    call(lib, "espp_decompose", h)
    call(lib, "espp_vl_create", h, rc, 0, None)
    shift = 4.0 * (rc ** -12 - rc ** -6)
    call(lib, "espp_lj_set", h, 0, 0, 1.0, 1.0, rc, shift, 0.9)
    b = np.ascontiguousarray(bonds.reshape(-1))
    call(lib, "espp_bonds_add", h, len(bonds), i64ptr(b))
    call(lib, "espp_fene_set", h, 30.0, 0.0, 1.5, math.inf, 0.0)
    call(lib, "espp_integrator_set", h, 0.01)
    call(lib, "espp_langevin_set", h, 1, 0.5, 1.0, 0, None)
    layout = _tune(lib, h, 10.0)
    ms = np.zeros(2)
    call(lib, "espp_run", h, cap_steps)
    call(lib, "espp_last_run_ms", h, dptr(ms))
    t_cap = float(ms[1])
    call(lib, "espp_lj_set", h, 0, 0, 1.0, 1.0, rc, shift, 0.0)
    call(lib, "espp_run", h, steps)
    call(lib, "espp_last_run_ms", h, dptr(ms))
    t_run = float(ms[1])
    v2 = ctypes.c_double()
    nn = ctypes.c_int64()
    call(lib, "espp_kinetic", h, ctypes.byref(v2), ctypes.byref(nn))
    e = ctypes.c_double()
    call(lib, "espp_energy", h, 1, ctypes.byref(e))
    mx = ctypes.c_double()
    call(lib, "espp_bonds_max_sqr", h, ctypes.byref(mx))
    lib.espp_system_destroy(h)
    n = len(ids)
    return {"value": n * (cap_steps + steps) / ((t_cap + t_run) * 1e-3),
            "ms_per_step": (t_cap + t_run) / (cap_steps + steps),
            "ms_per_step_capped": t_cap / cap_steps, "T_end": v2.value / (3 * n),
            "fene_energy_per_bond": e.value / len(bonds), "max_bond": math.sqrt(mx.value),
            "layout": layout}


def lj32k_config(lib, prec, steps=1000):
    """LJ fluid 32^3 = 32,768 particles (the reference's CPU-runnable case): rho 0.8442,
    rc 2.5, skin 0.3, dt 0.005, Langevin gamma 1 T 1, 1000 steps; the list layout is the
    autotuner's choice (before the timed steps)."""
    from espressopp_b200._abi import call, dptr
    h = make_system(lib, 32, prec)[0]
    call(lib, "espp_langevin_set", h, 1, 1.0, 1.0, 0, None)
    layout = _tune(lib, h, 6.0)
    call(lib, "espp_run", h, steps)
    ms = np.zeros(2)
    call(lib, "espp_last_run_ms", h, dptr(ms))
    lib.espp_system_destroy(h)
    return {"value": 32768 * steps / (ms[1] * 1e-3), "ms_per_step": float(ms[1]) / steps,
            "layout": layout}


def _tune(lib, h, steps_per_build):
    """espp_autotune_layout on the system as it stands; the chosen layout as a dict."""
    from espressopp_b200._abi import call, dptr, i32ptr
    best = np.zeros(5, np.int32)
    table = np.zeros((32, 8))
    n = ctypes.c_int32(0)
    call(lib, "espp_autotune_layout", h, steps_per_build, i32ptr(best), dptr(table), 32,
         ctypes.byref(n))
    names = {0: "global", 1: "brick", 2: "global-brick-build"}
    return {"form": names[int(best[0])], "threads_per_particle": int(best[1]),
            "brick": [int(x) for x in best[2:5]]}


def _plain(o):
    """JSON encoding of numpy scalars and arrays."""
    if isinstance(o, np.integer):
        return int(o)
    if isinstance(o, np.floating):
        return float(o)
    if isinstance(o, np.bool_):
        return bool(o)
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError("not JSON serialisable: %r" % type(o))


def emit(line):
    """Prints one JSON line."""
    print(json.dumps(line, default=_plain), flush=True)


def small_configs(lib, replica_steps=1000, cg_chains=200):
    from espressopp_b200 import _abi
    out = {}
    for name, prec in (("fp64", _abi.PREC_FP64), ("mixed", _abi.PREC_MIXED)):
        log("configs: Kremer-Grest melt, " + name)
        out["kg_melt_40k_" + name] = kg_melt_config(lib, prec)
        log("configs: 32k LJ, " + name)
        out["lj_32k_" + name] = lj32k_config(lib, prec)
    out["unit"] = "particle-steps/s (device-timed step loop)"
    if replica_steps > 0:
        log("configs: 64 PT replicas, %d steps" % replica_steps)
        rep, total, seg, segments, _ = run_replicas(lib, _abi.PREC_MIXED, replica_steps, 20)
        out["pt_replicas_64"] = {
            "workload": "64 LJ replicas, N ~ U{2000..64000} (seed 4), %d particles, mixed, "
                        "Langevin T 0.7..2.0, exchange every %d steps, %d steps (config: "
                        "20,000)" % (total, seg, seg * segments),
            "batched_value": rep["batched"]["value"],
            "sequential_value": rep["sequential"]["value"],
            "batched_over_sequential": rep["batched"]["value"] / rep["sequential"]["value"],
            "swaps": {"batched": rep["batched"]["swaps"],
                      "sequential": rep["sequential"]["swaps"]},
            "unit": "particle-steps/s (wall clock around run calls and exchanges)"}
    if cg_chains > 0:
        log("configs: learned-potential training gradient, 50,000 sites")
        out["mlp_training_gradient_50k"] = mlp_gradient_config(50000)
        log("configs: learned CG potential, %d chains" % cg_chains)
        t0 = time.perf_counter()
        line = cg_workflow(cg_chains, 100, 5, 20000, 5, 50)
        q = line["cg_quality"]
        out["cg_learned_potential"] = {
            "workload": "Kremer-Grest melt %d x 200 beads -> %d CG sites (4:1), 100 frames, "
                        "5 epochs, 5 IBI iterations, 20,000 CG steps (the full configuration: "
                        "1000 chains, 500 frames, 100,000 steps: --workload cg)"
                        % (cg_chains, cg_chains * 50),
            "force_matching_rel_err": q["force_matching_rel_err"],
            "rdf_l2": {k: v for k, v in q["rdf_l2"].items() if k != "curves"},
            "particle_steps_per_chain_motion_fg_over_cg":
                q["particle_steps_per_chain_motion_fg_over_cg"],
            "cg_ms_per_step": q["cg_ms_per_step"],
            "site_steps_per_s_learned": line["value"],
            "seconds": time.perf_counter() - t0}
    return out


# ---- learned coarse-grained potential ---------------------------------------------
def cg_arm(args, rank, world, local_rank):
    """Learned CG potential workload (cg_workflow at the sizes of the arguments)."""
    if rank != 0:
        return
    line = cg_workflow(args.cg_chains, args.cg_frames, args.cg_epochs, args.cg_steps,
                       args.cg_ibi, args.cg_window)
    emit(line)


def cg_workflow(nch, nfr, epochs, cg_steps, ibi_iters, window):
    """Learned CG potential: a fine-grained Kremer-Grest melt of nch x 200 beads mapped
    4 -> 1 (nch x 50 sites); nfr frames of mapped conservative forces averaged over
    `window` steps; CG bonds and angles from Boltzmann-inverted tables; an MLP 16-64-64-1
    trained by force matching on the GPU for `epochs` epochs; a force-matched pair table as
    the fallback; ibi_iters of iterative Boltzmann inversion; CG runs of cg_steps steps
    compared with the fine-grained melt by force-matching error, RDF and chain motion.
    Returns the result line."""
    from espressopp_b200 import cg
    from espressopp_b200._abi import call, dptr
    t0 = time.perf_counter()
    pos, frc, L, bonds = cg.fg_frames(nch, 200, nfr, 20, warm_capped=1000, warm=4000,
                                      window=window, log=log)
    t_fg = time.perf_counter() - t0
    log("fine-grained frames: %d x %d sites in %.1f s" % (nfr, pos.shape[1], t_fg))
    ntrain = int(0.8 * nfr)
    tab = cg.boltzmann_bond_table(cg.bond_lengths(pos, bonds))
    triples = cg.angle_triples(bonds)
    atab = cg.boltzmann_angle_table(cg.angles_of(pos[:ntrain], triples))
    # non-bonded target: mapped force minus the CG bond and angle forces
    bondsys = cg.CGSystem(pos[0], L, bonds, tab)
    bondsys.set_angle_table(triples, atab)
    fbond_test = np.zeros((nfr - ntrain,) + pos.shape[1:])
    for k in range(nfr):
        fb = bondsys.forces_at(pos[k])
        frc[k] -= fb
        if k >= ntrain:
            fbond_test[k - ntrain] = fb
    bondsys.close()
    target = frc
    t1 = time.perf_counter()
    # non-bonded terms act between sites that are not bonded to each other (excluding the
    # 1-3 pairs as well measured worse: RDF L2 0.034 against 0.024)
    excl = np.asarray(bonds, np.int64).reshape(-1, 2)
    ptab = cg.pair_fm_table(pos[:min(ntrain, 10)], target[:min(ntrain, 10)], L, exclude=excl)
    tabsys = cg.CGSystem(pos[0], L, bonds, tab, exclude=excl)
    tabsys.set_angle_table(triples, atab)
    tabsys.set_pair_table(ptab)
    err_table = cg.fm_error(tabsys, pos[ntrain:], target[ntrain:], fbond_test)
    t_tab = time.perf_counter() - t1
    # the learned potential corrects the force-matched pair table: trained on the residual
    pairsys = cg.CGSystem(pos[0], L, bonds, ([0.5, 1.0, 1.5, 2.0], [0.0] * 4, [0.0] * 4),
                          exclude=excl)
    pairsys.set_pair_table(ptab)
    resid = np.empty((ntrain,) + target.shape[1:])
    for k in range(ntrain):
        resid[k] = target[k] - pairsys.forces_at(pos[k])
    pairsys.close()
    s = cg.CGSystem(pos[0], L, bonds, tab, exclude=excl)
    s.set_angle_table(triples, atab)
    s.set_pair_table(ptab)
    model = cg.MLPModel(seed=3)
    s.attach(model)
    shift, scale = cg.descriptor_norm(s, pos)
    model.set_norm(shift, scale)
    t2 = time.perf_counter()
    hist = cg.train_mlp(s, model, pos[:ntrain], resid[:ntrain], epochs=epochs,
                        batch=4, lr=1e-3, log=log)
    t_train = time.perf_counter() - t2
    del resid
    err_mlp_fm = cg.fm_error(s, pos[ntrain:], target[ntrain:], fbond_test)
    err_zero = 1.0
    log("force-matching error: pair table + mlp %.4f, pair table %.4f" % (err_mlp_fm, err_table))
    # structure-based refinement (iterative Boltzmann inversion) of the pair table against
    # the RDF of the mapped fine-grained sites, for the learned model (network fixed) and
    # for the table-only fallback
    nb = 120
    g_fg = cg.rdf_of_frames(tabsys, pos[::max(1, nfr // 25)], nb)
    t3 = time.perf_counter()
    ibi = {}
    g_cg = {}
    blen = cg.bond_lengths(pos[:ntrain], bonds)
    for name, sysm in (("mlp", s), ("table", tabsys)):
        sysm.set_pos(sysm.ids, cg.wrap(pos[-1], L))
        call(sysm.lib, "espp_integrator_set", sysm.h, 0.01)
        sysm.thermostat(True)
        _, ibi[name], g_cg[name] = cg.ibi_refine(sysm, ptab, g_fg, nb, iters=ibi_iters,
                                                 log=log, bonded=(bonds, tab, blen))
    t_ibi = time.perf_counter() - t3
    err_mlp = cg.fm_error(s, pos[ntrain:], target[ntrain:], fbond_test)
    err_table_fm = err_table
    err_table = cg.fm_error(tabsys, pos[ntrain:], target[ntrain:], fbond_test)
    # chain motion of the FG frames
    sites_per_chain = 50
    msd_fg = cg.chain_com_msd(pos, sites_per_chain)
    # CG runs: learned potential and table fallback, both with the bond table
    out = {}
    for name, sysm in (("table", tabsys), ("mlp", s)):
        sysm.set_pos(sysm.ids, cg.wrap(pos[-1], L))
        call(sysm.lib, "espp_integrator_set", sysm.h, 0.01)
        sysm.thermostat(True)
        for k in range(20):
            try:
                sysm.run(100)
            except RuntimeError as e:
                p, v, f, img = sysm.state(sysm.ids)
                log("CG run (%s) failed after %d steps: %s; T %.3f, max |F| %.3g" %
                    (name, 100 * k, e, np.sum(4 * v * v) / (3 * len(v)),
                     np.max(np.abs(f))))
                raise
            if k % 5 == 4:
                p, v, f, img = sysm.state(sysm.ids)
                log("CG run (%s) step %d: T %.3f, max |F| %.3g" %
                    (name, 100 * (k + 1), np.sum(4 * v * v) / (3 * len(v)), np.max(np.abs(f))))
        traj = []
        window_steps = nfr * 20
        ms_total = 0.0
        g = np.zeros(nb)
        ng = 0
        for k in range(window_steps // 100):
            sysm.run(100)
            ms = np.zeros(2)
            call(sysm.lib, "espp_last_run_ms", sysm.h, dptr(ms))
            ms_total += ms[1]
            p, _, _, img = sysm.state(sysm.ids)
            traj.append(p + img * L)
            if k % 4 == 0:
                g += sysm.rdf(nb)
                ng += 1
        steps_rest = cg_steps - window_steps - 2000
        if steps_rest > 0:
            sysm.run(steps_rest)
            ms = np.zeros(2)
            call(sysm.lib, "espp_last_run_ms", sysm.h, dptr(ms))
            ms_total += ms[1]
        g /= ng
        traj = np.array(traj)
        msd_cg = cg.chain_com_msd(traj, sites_per_chain)
        dr = L / 2 / nb
        r = (np.arange(nb) + 0.5) * dr
        sel = r < 3.0 * 2
        l2 = float(np.sqrt(np.mean((g[sel] - g_fg[sel]) ** 2)))
        out[name] = {"rdf_l2": l2, "chain_msd_100tau": float(msd_cg[-1]),
                     "ms_per_step": ms_total / (window_steps // 100 * 100 + max(steps_rest, 0))}
        log("CG run (%s): RDF L2 %.4f, chain MSD %.3f (FG %.3f)" %
            (name, l2, msd_cg[-1], msd_fg[-1]))
    n_fg = nch * 200
    n_cg = nch * 50
    ratio = (n_fg / float(msd_fg[-1])) / (n_cg / out["mlp"]["chain_msd_100tau"])
    line = {
        "metric": "CG site-steps/s (learned potential)", "unit": "particle-steps/s",
        "value": n_cg / (out["mlp"]["ms_per_step"] * 1e-3), "n_gpus": 1,
        "higher_is_better": True, "data": "synthetic",
        "config": {"workload": "learned CG potential: Kremer-Grest melt %d x 200 beads -> "
                               "%d CG sites (4:1), %d frames, MLP 16-64-64-1 SiLU" %
                               (nch, n_cg, nfr)},
        "cg_quality": {
            "force_matching_rel_err": {
                "mlp_plus_ibi_table": err_mlp, "ibi_table": err_table,
                "mlp_plus_force_matched_table": err_mlp_fm,
                "force_matched_table": err_table_fm, "zero_model": err_zero},
            "rdf_l2": {"mlp_plus_ibi_table": out["mlp"]["rdf_l2"],
                       "ibi_table": out["table"]["rdf_l2"],
                       "ibi_iterations": {"mlp": ibi["mlp"], "table": ibi["table"]},
                       "curves": {"r": [round(float(x), 4) for x in (np.arange(nb) + 0.5) *
                                        (L / 2 / nb)],
                                  "fg": [round(float(x), 5) for x in g_fg],
                                  "mlp": [round(float(x), 5) for x in g_cg["mlp"]],
                                  "table": [round(float(x), 5) for x in g_cg["table"]]},
                       "definition": "sqrt(mean over bins r < 6 of (g_cg - g_fg)^2), "
                                     "120 bins up to L/2"},
            "particle_steps_per_chain_motion_fg_over_cg": ratio,
            "chain_com_msd_100tau": {"fg": float(msd_fg[-1]), "mlp": out["mlp"]["chain_msd_100tau"],
                                     "pair_table": out["table"]["chain_msd_100tau"]},
            "cg_ms_per_step": {"mlp": out["mlp"]["ms_per_step"],
                               "pair_table": out["table"]["ms_per_step"]},
            "training_loss_per_epoch": hist,
            "seconds": {"fg_frames": t_fg, "pair_table_fit": t_tab, "ibi": t_ibi,
                        "mlp_training": t_train},
            "force_target": "mapped conservative forces averaged over %d fine-grained "
                            "steps, minus the CG bond forces" % window,
            "note": "force-matching error on held-out frames (20 %) relative to the "
                    "window-averaged mapped forces; what remains of the fine-grained "
                    "fluctuation after the average is noise that no CG model can fit"},
    }
    model.close()
    return line


# ---- learned potential: force evaluation micro-benchmark --------------------------
def mlp_gradient_config(n_sites=50000, calls=20, warmup=3):
    """Force-matching gradient of the learned potential (espp_mlp_fm_grad: descriptor,
    site network forward, forward-mode tangent, weight-gradient products) on n_sites CG
    sites at density 0.2125 (jittered lattice), seeded weights and seeded reference forces,
    with the weight products on the tensor cores (BF16, FP32 accumulation) and on CUDA
    cores (FP32).  Wall clock around synchronous calls (each returns its loss), after
    `warmup` calls; the relative difference of the two gradients is reported."""
    from espressopp_b200 import cg
    from espressopp_b200._abi import call, dptr, i64ptr
    n_side = int(round(n_sites ** (1.0 / 3.0)))
    pos, L = lattice(n_side, 0.2125, 0.3, 7)
    n = len(pos)
    fref = np.random.Generator(np.random.PCG64(9)).normal(0.0, 3.0, size=(n, 3))
    zero = ([0.5, 1.0, 1.5, 2.0], [0.0] * 4, [0.0] * 4)
    out, grads = {}, {}
    for mode, name in ((1, "tensor_cores_bf16"), (0, "cuda_cores_fp32")):
        sysm = cg.CGSystem(pos, L, np.zeros((0, 2), np.int64), zero)
        model = cg.MLPModel(seed=5)
        call(model.lib, "espp_mlp_set_mode", model.m, mode)
        model.set_norm(np.full(16, 0.5), np.full(16, 1.0))
        sysm.attach(model)
        call(sysm.lib, "espp_integrator_set", sysm.h, 0.005)
        sysm.run(0)
        npar = ctypes.c_int64()
        call(sysm.lib, "espp_mlp_num_params", ctypes.byref(npar))
        g = np.zeros(npar.value)
        loss = ctypes.c_double()
        ids = np.ascontiguousarray(sysm.ids, np.int64)
        f = np.ascontiguousarray(fref.reshape(-1))

        def grad_call():
            call(sysm.lib, "espp_mlp_fm_grad", sysm.h, n, i64ptr(ids), dptr(f),
                 ctypes.byref(loss), dptr(g))
        for _ in range(warmup):
            grad_call()
        t0 = time.perf_counter()
        for _ in range(calls):
            grad_call()
        dt = time.perf_counter() - t0
        out[name] = {"ms_per_gradient": dt / calls * 1e3,
                     "site_gradients_per_s": n * calls / dt, "loss": loss.value}
        grads[name] = g.copy()
        sysm.close()
        model.close()
    a, b = grads["tensor_cores_bf16"], grads["cuda_cores_fp32"]
    out["gradient_rel_diff_bf16_vs_fp32"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["speedup_tensor_cores"] = (out["cuda_cores_fp32"]["ms_per_gradient"] /
                                   out["tensor_cores_bf16"]["ms_per_gradient"])
    out["workload"] = ("force-matching gradient, %d CG sites, rc 3.0, 16 basis functions, "
                       "MLP 16-64-64-1, %d calls" % (n, calls))
    out["unit"] = "wall clock around synchronous espp_mlp_fm_grad calls"
    return out


def mlp_arm(args, rank, world, local_rank):
    """Device time of the learned potential's force pass (descriptor, site network,
    pair forces) on a CG-like configuration: --mlp-sites sites at density 0.2125 on a
    jittered lattice, seeded random weights, NVE steps of a CG system that holds only the
    learned potential; site network on the tensor cores (BF16) and on CUDA cores (FP32)."""
    from espressopp_b200 import cg
    from espressopp_b200._abi import call, dptr
    if rank != 0:
        return
    n_side = int(round(args.mlp_sites ** (1.0 / 3.0)))
    pos, L = lattice(n_side, 0.2125, 0.3, 7)
    n = len(pos)
    zero = ([0.5, 1.0, 1.5, 2.0], [0.0] * 4, [0.0] * 4)
    out = {}
    for mode, name in ((1, "tensor_cores_bf16"), (0, "cuda_cores_fp32")):
        sysm = cg.CGSystem(pos, L, np.zeros((0, 2), np.int64), zero)
        model = cg.MLPModel(seed=5)
        call(model.lib, "espp_mlp_set_mode", model.m, mode)
        model.set_norm(np.full(16, 0.5), np.full(16, 1.0))
        sysm.attach(model)
        call(sysm.lib, "espp_integrator_set", sysm.h, 0.005)
        sysm.run(args.warmup)
        sysm.run(args.steps)
        ms = np.zeros(2)
        call(sysm.lib, "espp_last_run_ms", sysm.h, dptr(ms))
        out[name] = {"ms_per_step": ms[1] / args.steps,
                     "site_steps_per_s": n * args.steps / (ms[1] * 1e-3)}
        sysm.close()
        model.close()
    line = {"metric": "learned-potential site-steps/s", "unit": "particle-steps/s",
            "value": out["tensor_cores_bf16"]["site_steps_per_s"], "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "data": "synthetic",
            "config": {"workload": "learned CG potential force pass, %d sites, rc 3.0, "
                                   "16 basis functions, MLP 16-64-64-1" % n},
            "modes": out, "training_gradient": mlp_gradient_config(args.mlp_sites)}
    emit(line)


# ---- batched parallel-tempering replicas ------------------------------------------
def run_replicas(lib, prec, steps, warmup, R=64, dist=None):
    """R LJ replicas, N ~ U{2000..64000} (seed 4), rho 0.8442, rc 2.5, skin 0.3,
    T_r = 0.7 (2.0/0.7)^(r/(R-1)), Langevin gamma 1, dt 0.005, Metropolis exchange between
    neighbours every 100 steps (ParallelTempering.exchange rule).  Times `steps` steps of
    all replicas with one graph launch per 100-step segment (espp_batch_run) against the
    same steps run replica by replica (espp_run each), wall clock around the calls and
    exchanges.  Under torchrun the replicas are shared out among the ranks by particle
    count; the exchange gathers (E_pot, T, N) of every replica with one all-reduce and
    every rank applies the same decisions; the time is the max over ranks.
    Returns ({mode: result}, total particles, steps per segment, segments, this rank's
    replica count)."""
    from espressopp_b200._abi import call, dptr, i32ptr, i64ptr
    from espressopp_b200.parallel_tempering import (exchange_decisions, gather_replica_rows,
                                                    partition_replicas)
    rng = np.random.Generator(np.random.PCG64(4))
    sizes = rng.integers(2000, 64001, size=R)
    temps = [0.7 * (2.0 / 0.7) ** (r / (R - 1)) for r in range(R)]
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    group = dist.group.WORLD if dist is not None else None
    local = [r for r, o in enumerate(partition_replicas(sizes, world)) if o == rank]

    def make(r):
        N = int(sizes[r])
        L = (N / RHO) ** (1.0 / 3.0)
        a = int(math.ceil(N ** (1.0 / 3.0)))
        sp = L / a
        g = (np.arange(a) + 0.5) * sp
        grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:N]
        pr = np.random.Generator(np.random.PCG64(1000 + r))
        pos = grid + pr.uniform(-0.05, 0.05, size=grid.shape)
        vel = mb_velocities(N, temps[r], 2000 + r)
        h = ctypes.c_void_p()
        box = np.array([L, L, L])
        cg = np.array([int(L / (RC + SKIN))] * 3, np.int32)
        call(lib, "espp_system_create", dptr(box), SKIN, i32ptr(cg), prec, 77 + r, ctypes.byref(h))
        ids = np.arange(N, dtype=np.int64)
        call(lib, "espp_add_particles", h, N, i64ptr(ids), None, None,
             dptr(np.ascontiguousarray(pos.reshape(-1))), dptr(np.ascontiguousarray(vel.reshape(-1))))
        call(lib, "espp_decompose", h)
        call(lib, "espp_vl_create", h, RC, 0, None)
        call(lib, "espp_lj_set", h, 0, 0, 1.0, 1.0, RC, 4.0 * (RC ** -12 - RC ** -6), 0.0)
        call(lib, "espp_integrator_set", h, DT)
        call(lib, "espp_set_tpp", h, 1)
        return h

    T = list(temps)

    def set_T(hs):
        for r, h in zip(local, hs):
            call(lib, "espp_langevin_set", h, 1, 1.0, T[r], 0, None)

    def exchange(hs, oddeven, urng):
        rows = {}
        for r, h in zip(local, hs):
            v = ctypes.c_double()
            call(lib, "espp_energy", h, 0, ctypes.byref(v))
            k2 = ctypes.c_double()
            nn = ctypes.c_int64()
            call(lib, "espp_kinetic", h, ctypes.byref(k2), ctypes.byref(nn))
            rows[r] = (v.value, k2.value / (3.0 * nn.value), float(nn.value))
        allrows = gather_replica_rows(rows, R, group)
        dec = exchange_decisions(list(allrows[:, 0]), list(allrows[:, 1]),
                                 [int(x) for x in allrows[:, 2]], oddeven, urng.random)
        for m, n, _, _, ok in dec:
            if ok:
                T[m], T[n] = T[n], T[m]
        return sum(ok for *_, ok in dec)

    def barrier():
        if dist is not None:
            import torch
            t = torch.zeros(1, device="cuda")
            dist.all_reduce(t)
            torch.cuda.synchronize()

    import random
    total = int(sizes.sum())
    segments = max(1, steps // 100)
    seg = steps // segments
    out = {}
    for mode in ("sequential", "batched"):
        T[:] = temps
        hs = [make(r) for r in local]
        set_T(hs)
        b = None
        if mode == "batched" and hs:
            arr = (ctypes.c_void_p * len(hs))(*[h.value for h in hs])
            b = ctypes.c_void_p()
            call(lib, "espp_batch_create", arr, len(hs), ctypes.byref(b))
        urng = random.Random(335977)

        def step_all(n):
            if b is not None:
                call(lib, "espp_batch_run", b, n)
            else:
                for h in hs:
                    call(lib, "espp_run", h, n)

        step_all(warmup)
        swaps = 0
        barrier()
        t0 = time.perf_counter()
        for k in range(segments):
            step_all(seg)
            swaps += exchange(hs, k % 2, urng)
            set_T(hs)
        barrier()
        el = max_over_ranks(dist, time.perf_counter() - t0)
        out[mode] = {"seconds": el, "value": total * seg * segments / el, "swaps": swaps}
        if b is not None:
            lib.espp_batch_destroy(b)
        for h in hs:
            lib.espp_system_destroy(h)
    return out, total, seg, segments, len(local)


def replicas_arm(args, rank, world, local_rank):
    """The parallel-tempering workload alone: run_replicas at --steps steps, the replicas
    shared out among the ranks under torchrun (strong scaling: 64 replicas in total)."""
    import espressopp_b200
    from espressopp_b200 import _abi
    from espressopp_b200._abi import call
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(local_rank)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    lib = espressopp_b200.load_library()
    call(lib, "espp_select_device", local_rank)
    prec = _abi.PREC_MIXED if args.precision == "mixed" else _abi.PREC_FP64
    out, total, seg, segments, nlocal = run_replicas(lib, prec, args.steps, args.warmup,
                                                      dist=dist)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": "PT replica particle-steps/s, 64 LJ replicas on 1 B200",
                "value": out["batched"]["value"], "unit": "particle-steps/s", "n_gpus": world,
                "steps": seg * segments, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec else "f64",
                "data": "synthetic",
                "config": {"workload": "64 LJ replicas, N ~ U{2000..64000} (seed 4), total %d "
                                       "particles, rho 0.8442, rc 2.5, skin 0.3, Langevin gamma 1, "
                                       "T 0.7..2.0 geometric, dt 0.005, exchange every %d steps"
                                       % (total, seg),
                           "timing": "wall clock around the run calls and exchanges, max over "
                                     "ranks",
                           "parallelism": "replicas shared out over %d rank(s) by particle "
                                          "count; exchange rows all-reduced" % world,
                           "replicas_on_rank0": nlocal},
                "batched": out["batched"], "sequential": out["sequential"],
                "batched_over_sequential": out["batched"]["value"] / out["sequential"]["value"]}
        emit(line)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lj", choices=["lj", "replicas", "cg", "mlp"],
                    help="lj: the 4,096,000-particle fluid (default); replicas: 64 PT "
                         "replicas; cg: the learned coarse-grained potential; mlp: its "
                         "force pass alone")
    ap.add_argument("--mlp-sites", type=int, default=50000)
    ap.add_argument("--cg-chains", type=int, default=1000)
    ap.add_argument("--cg-frames", type=int, default=500)
    ap.add_argument("--cg-epochs", type=int, default=15)
    ap.add_argument("--cg-steps", type=int, default=100000)
    ap.add_argument("--cg-ibi", type=int, default=20, help="IBI iterations of the pair table")
    ap.add_argument("--cg-window", type=int, default=50,
                    help="steps over which the mapped forces of a frame are averaged")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--n-side", type=int, default=160)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--ref-budget", type=float, default=20.0)
    ap.add_argument("--steps-ref", type=int, default=1)
    ap.add_argument("--no-fp64", action="store_true", help="skip the all-FP64 comparison")
    ap.add_argument("--equil", type=int, default=1000,
                    help="Langevin steps (gamma 1, T 1) before the NVE segment")
    ap.add_argument("--drift-steps", type=int, default=2000,
                    help="NVE steps of the drift measurement (both precisions)")
    ap.add_argument("--cg-small", type=int, default=200,
                    help="chains of the reduced learned-CG run in the default line (0: skip)")
    ap.add_argument("--replica-steps", type=int, default=1000,
                    help="steps of the 64-replica measurement in the default line (0: skip)")
    ap.add_argument("--no-oracle", action="store_true",
                    help="skip the pair-set and force comparison with the FP64 oracle")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the Kremer-Grest melt and 32k LJ configurations")
    ap.add_argument("--tpp", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="threads per particle of the global-list force kernel")
    ap.add_argument("--layout", default="auto",
                    choices=["auto", "global", "brick", "global-brick-build"],
                    help="list layout: autotuned, global per-particle lists (per-cell build), "
                         "brick windows, global lists built by brick windows")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
    elif args.workload == "replicas":
        replicas_arm(args, rank, world, local_rank)
    elif args.workload == "cg":
        cg_arm(args, rank, world, local_rank)
    elif args.workload == "mlp":
        mlp_arm(args, rank, world, local_rank)
    else:
        gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
