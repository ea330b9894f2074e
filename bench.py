#!/usr/bin/env python
"""Throughput of the 2D electrostatic PIC step on B200.

Metric: particle-steps/s of bin + deposit + push (the particle phases of one
PIC step), with Poisson ms/step reported beside it.  One "step" is one full
PIC step of the workload: zero rho, deposit every species, Poisson to 1e-8
relative residual + E field, push every species.  `value` counts the device
time of the particle phases only (CUDA events on the library's stream, which
is torch's current stream), summed over the K timed steps, max over ranks.

Default workload: the 1024x1024 configuration with the 200 V internal
electrode and the drifting Gaussian blob (~2.3e8 particles, FP32 state,
64-bit fixed-point deposit).  The particle state (~9 GB) is far larger than
L2, so no flush is needed between steps.

Multi-GPU: a single instance does not shard (no domain decomposition), so N
ranks run N independent replicas with different seeds ("scaling": "weak").

--impl reference times the reference's algorithm on the host cores (the
hashmap port in oracle/, the reference's own CPU path being unbuildable here)
on the same full-size workload, every step a full step, and prints the same
JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "bmp-6th-sem_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "particle-steps/s (bin+deposit+push)"
UNIT = "particle-steps/s"
# Algorithmic HBM bytes per particle of the push pass (FP32 state, 20 B per
# particle: float4 {fx, fy, vx, vy} + float vz): read the state, write it to
# its slot in the other buffer.  Binning and the deposit ride on this pass.
BYTES_PUSH_PASS = 40
BYTES_STEP = 40           # whole particle phase of one step
BYTES_THREE_PASS_FP32 = 112   # separate push / deposit / bin passes: 48 + 12 + 52 bytes a particle-step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg3", choices=["cfg1", "cfg2", "cfg3", "cfg4"],
                    help="cfg4: the learned warm-start protocol on the cfg3 run (train on the "
                         "first --cfg4-train steps, evaluate on the next --cfg4-eval)")
    ap.add_argument("--cfg4-train", type=int, default=2000)
    ap.add_argument("--cfg4-eval", type=int, default=2000)
    ap.add_argument("--cfg4-epochs", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--solve-only", action="store_true",
                    help="profiling aid: W steps of the workload, then K Poisson solves from the same "
                         "state (phi of the previous step as the start); prints their statistics")
    ap.add_argument("--no-graph", action="store_true",
                    help="with --solve-only: PCG iterations as direct launches (for profilers)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-energy", action="store_true",
                    help="skip the energy-weighted mesh (deposit_energy = 0)")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned warm-start comparison")
    ap.add_argument("--ws-pairs", type=int, default=512,
                    help="pairs recorded for the learned warm start")
    ap.add_argument("--ws-epochs", type=int, default=12)
    ap.add_argument("--ws-lr", type=float, default=1e-3,
                    help="Adam step size, decaying along a half cosine to 1/100 of it")
    ap.add_argument("--ws-eval", type=int, default=24,
                    help="evaluation steps, each solved from both guesses")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 64-instance batched ensemble measurement")
    ap.add_argument("--ensemble-steps", type=int, default=10)
    ap.add_argument("--tile-shape", type=int, default=None, choices=[0, 1, 2, 3],
                    help="particle-kernel tile shape (0 64x4, 1 256x1, 2 128x2, 3 16x16); "
                         "default: the library's tuner picks it (under a profiler, fix it: "
                         "the tuner's timings change there)")
    return ap.parse_args()


def workload(name):
    import pic_configs as C
    return {"cfg1": C.cfg1, "cfg2": C.cfg2, "cfg3": C.cfg3}[name]()


def describe(w):
    el = [r for r in w.rects[4:]]
    return (f"{w.name}: {w.nx}x{w.ny} cells, dx={w.dx} m, dt={w.dt} s, Bz={w.b0} T, "
            f"{w.ppc} ppc/species background" +
            (f" + Gaussian blob peak {w.plasma[0].blob_peak_ppc:g} ppc sigma {w.plasma[0].blob_sigma:g} cells"
             if w.plasma[0].blob_peak_ppc else "") +
            (f", internal electrode {el}" if el else "") + ", electrons + Ar+")


# ---------------------------------------------------------------------------
# CPU side: the reference's algorithm (hashmap port) on a bounded sample
# ---------------------------------------------------------------------------

def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# The reference's hashmap gives every node key probing_length slots
# (prob_size * wg = 24 * 256 = 6144 by default, src/particles.cpp:181), with
# slot indices in int.  On the 1024^2 workload 6144 slots a node would take
# 62 GB per species and overflow int (1.05e6 nodes * 6144 * 1.2 > 2^31), so
# the port sizes the buckets to the data instead: the next power of two of
# 1.3 x the fullest bucket, capped where the slot index still fits an int.
def probing_length(peak: int, nodes: int) -> int:
    want = 1 << max(4, int(np.ceil(np.log2(1.3 * max(peak, 1)))))
    cap = int((2 ** 31 - 1) / (nodes * 1.2))
    return min(want, cap)


def cpu_reference_run(w, max_seconds=None, steps=None, min_steps=2):
    """Times the reference's step structure (src/main.cpp:130-230) on the
    host cores, on the full workload: per species the hashmap deposit, the
    Poisson solve (SuperLU, factored once beforehand), then per species the
    mover, compaction and map cleanup.  Runs `steps` steps, or steps until
    max_seconds of particle-phase time (at least min_steps).  Returns a dict:
    particle-steps/s of the particle phases, Poisson ms/step, per-step
    particle seconds, the sample description, threads, CPU model."""
    import oracle as O
    import pic_configs as C
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    t_setup = time.perf_counter()
    nx, ny = w.nx, w.ny
    dx = w.xmax / nx
    g = O.Grid(nx, ny, dx, dx, w.xmax, w.ymax)
    pts = []
    for s in range(2):
        ps = w.plasma[s]
        v_th = float(np.sqrt(C.QE * ps.temperature_ev / w.species[s][1]))
        pts.append(O.generate_plasma(nx, ny, dx, dx, ps.ppc, v_th, ps.blob_peak_ppc, ps.blob_cx,
                                     ps.blob_cy, ps.blob_sigma or 1.0, ps.drift_vx, ps.drift_vy,
                                     seed=900 + s))
    el = O.Electrodes(w.rects)
    t0 = time.perf_counter()
    D = O.DirectPoisson(w.GX, w.GY, dx, dx, el)
    factor_s = time.perf_counter() - t0
    species = [O.Species(str(s), *w.species[s]) for s in range(2)]
    weigh = [O.weighing_factor(sp, w.xmax * w.ymax, dx, dx) for sp in species]
    peak = max(int(O.bucket_counts(g, p).max()) for p in pts)
    probing = probing_length(peak, g.nodes)
    H = [O.RefHashmapSpecies(g, pts[s], probing_length=probing) for s in range(2)]
    bz = np.full(g.nodes, w.b0)
    n_particles = sum(len(p) for p in pts)
    setup_s = time.perf_counter() - t_setup
    part_t, pois_t = [], []
    t_start = time.perf_counter()
    it = 0
    while True:
        rho = np.zeros(g.nodes)
        t0 = time.perf_counter()
        for s in range(2):
            H[s].deposit(species[s], weigh[s], C.EPS0, rho)
        t1 = time.perf_counter()
        phi, ef = D.step(rho)
        t2 = time.perf_counter()
        for s in range(2):
            H[s].move(species[s].ctom, w.dt, ef, bz)
            H[s].compact()
            H[s].cleanup()
        t3 = time.perf_counter()
        part_t.append((t1 - t0) + (t3 - t2))
        pois_t.append(t2 - t1)
        it += 1
        if steps is not None:
            if it >= steps:
                break
        elif it >= min_steps and sum(part_t) > max_seconds:
            break
    value = n_particles * len(part_t) / sum(part_t)
    sample = (f"{w.name} at full size: {nx}x{ny} cells, {n_particles} particles, {len(part_t)} steps "
              f"of the reference hashmap algorithm (deposit, mover, compaction, cleanup) on "
              f"{threads} OpenMP threads, {probing} slots a bucket (fullest bucket {peak}); "
              f"Poisson by SuperLU on one thread (factored once in {factor_s:.1f} s)")
    return {"value": value, "poisson_ms": 1e3 * statistics.mean(pois_t), "part_t": part_t,
            "sample": sample, "threads": threads, "cpu": cpu_model(), "n": n_particles,
            "setup_s": setup_s, "factor_s": factor_s, "probing": probing}


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and f[1].replace(".", "").isdigit():
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows),
                "reasons": reasons}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic_per_particle():
    """Per-particle DRAM bytes of the scatter pass from the committed ncu
    summary (profiles/traffic.txt), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None, None
    kv = {}
    for line in open(p):
        if line.startswith("#") or not line.strip():
            continue
        k, _, v = line.strip().partition(" ")
        kv[k] = v
    v = kv.get("push_dram_bytes_per_particle")
    return (float(v) if v else None), kv.get("source")


def run_ours(args, rank, world, local_rank):
    import torch
    import pic_b200 as P
    import pic_configs as C
    torch.cuda.set_device(local_rank)
    w = workload(args.config)
    pic = P.Pic(C.library_config(w, device=local_rank, deposit_energy=not args.no_energy))
    # a dedicated (non-default) torch stream: the library runs on it and the
    # CUDA events below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    pic.set_stream(stream.cuda_stream)
    C.load_plasma(pic, w, seed=1234 + 7 * rank)
    counts = [pic.count(s) for s in range(2)]
    n_part = sum(counts)
    L = P.lib()
    import ctypes

    def launches():
        n = ctypes.c_int64(0)
        L.pic_launch_count(pic.h, ctypes.byref(n))
        return n.value

    it = 0
    # the library's tuner picks the particle kernels' tile shape for this
    # workload (it times the push on the loaded particles without keeping it)
    if args.tile_shape is None:
        tile_shape, tile_ms = pic.autotune(timings=True)
    else:
        tile_shape, tile_ms = args.tile_shape, None
        pic.set_tile_shape(tile_shape)
    for _ in range(args.warmup):
        pic.step(it)
        it += 1
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    l0 = launches()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]
    iters = []
    t_wall0 = time.perf_counter()
    for k in range(args.steps):
        e = ev[k]
        e[0].record(stream)
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        e[1].record(stream)
        pic.poisson_solve(it)
        e[2].record(stream)
        pic.move_particles(0, it)
        e[4].record(stream)
        pic.move_particles(1, it)
        e[3].record(stream)
        iters.append(pic.poisson_stats()[0])
        it += 1
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    gpu_launches = launches() - l0
    part_ms = sum(e[0].elapsed_time(e[1]) + e[2].elapsed_time(e[3]) for e in ev)
    pois_ms = [e[1].elapsed_time(e[2]) for e in ev]
    step_ms = sum(e[0].elapsed_time(e[3]) for e in ev)
    relres = pic.poisson_stats()[1]
    times = torch.tensor([part_ms, step_ms, sum(pois_ms)], dtype=torch.float64, device="cuda")
    nparts = torch.tensor([float(n_part)], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(times, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(nparts, op=torch.distributed.ReduceOp.SUM)
    part_ms, step_ms, pois_sum = times.tolist()
    total_particles = nparts.item()
    value = total_particles * args.steps / (part_ms * 1e-3)

    # per-kernel breakdown over 3 extra profiled steps (not part of `value`)
    L.pic_set_profiling(pic.h, 1)
    ms6 = (ctypes.c_double * P_PHASES)()
    calls6 = (ctypes.c_int64 * P_PHASES)()
    L.pic_profile_read(pic.h, ctypes.cast(ms6, ctypes.c_void_p), ctypes.cast(calls6, ctypes.c_void_p), 1)
    prof_steps = 3
    for _ in range(prof_steps):
        pic.step(it)
        it += 1
    L.pic_profile_read(pic.h, ctypes.cast(ms6, ctypes.c_void_p), ctypes.cast(calls6, ctypes.c_void_p), 1)
    L.pic_set_profiling(pic.h, 0)
    phase_names = ["push", "fixup", "relayout", "deposit", "flush", "poisson"]
    phases = {phase_names[i]: {"ms_per_step": ms6[i] / prof_steps, "calls_per_step": calls6[i] / prof_steps}
              for i in range(P_PHASES)}
    peak, peak_kind = measured_peaks()
    push_ms = ms6[0] / calls6[0] if calls6[0] else float("nan")
    avg_n = n_part / 2
    achieved = BYTES_PUSH_PASS * avg_n / (push_ms * 1e-3) / 1e9
    traffic_pp, traffic_src = ncu_traffic_per_particle()
    roofline = {"kernel": "k_cells<kPush> (gather + Boris + binning + fused deposit, one pass)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": f"{peak_kind} hbm_gbs",
                "bytes_per_particle": BYTES_PUSH_PASS,
                "traffic": (traffic_pp * avg_n) if traffic_pp else None,
                "traffic_source": traffic_src}
    step_particle_ms = (ms6[0] + ms6[1] + ms6[2] + ms6[4]) / prof_steps
    roofline_step = {"bytes_per_particle_step": BYTES_STEP,
                     "achieved_GBs": BYTES_STEP * n_part / (step_particle_ms * 1e-3) / 1e9,
                     "three_pass_112B_equivalent_GBs": BYTES_THREE_PASS_FP32 * n_part / (step_particle_ms * 1e-3) / 1e9}
    roofline_step["frac"] = roofline_step["achieved_GBs"] / peak
    roofline["kernels"] = kernel_rooflines(w, counts, ev, pois_ms, iters, phases, peak, peak_kind)

    learned = None
    if not args.no_learned:
        learned, it = run_learned(pic, args, it)
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(pic, args.steps, n_part, it)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": part_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": describe(w), "particles_per_gpu": n_part,
                   "tile_shape": ["64x4", "256x1", "128x2", "16x16"][tile_shape],
                   "ms_per_tile_shape": tile_ms,
                   "particles_per_species": counts, "grid_nodes": (w.nx + 1) * (w.ny + 1),
                   "l2": "inputs larger than L2 (particle state ~%.1f GB per GPU)" % (n_part * 40 / 1e9),
                   "parallelism": f"replicas x{world}",
                   "energy_mesh": not args.no_energy},
        "full_step": {"ms_per_step": step_ms / args.steps,
                      "particle_steps_per_s": total_particles * args.steps / (step_ms * 1e-3),
                      "wall_s": t_wall},
        "poisson": {"solver": "MG-PCG (FP32 V-cycle, FP64 CG)", "warm_start": "previous phi",
                    "ms_per_step_plain": pois_sum / args.steps,
                    "ms_per_step_learned": learned["ms_per_step_learned"] if learned else None,
                    "iters_per_step": statistics.mean(iters),
                    "relres": relres, "tol": 1e-8, "learned": learned},
        "roofline": roofline, "roofline_particle_phase": roofline_step,
        "phases": phases, "gpu_launches": gpu_launches, "clocks": clocks, "e2e": e2e,
    }
    return line, pic, w


P_PHASES = 6

# Algorithmic bytes of one MG-PCG iteration per fine node: the finest
# level's down kernel (read b, mask; write x and the coarse b: 10 B), up
# kernel (read x, b, mask, the coarse x, r; write z: 22 B), p/q update (read
# z, mask, p, q; write p, q: 37 B) and x/r update (read p, q, x, r, mask;
# write x, r, r32: 53 B), plus the coarser tiled levels (24 B a node at a
# quarter, a sixteenth ... of the nodes: about 8 B).
POISSON_BYTES_NODE_ITER = 130
# k_flush per node and species: read the two accumulators and rho, write
# them back (accumulators cleared) with final_mesh and energy_mesh.
FLUSH_BYTES_NODE = 64


def kernel_rooflines(w, counts, ev, pois_ms, iters, phases, peak, peak_kind):
    """HBM roofline of each kernel class of the step, from the timed steps'
    CUDA events (per-species push passes, the solve) and the profiled
    steps' phase timers (flush): algorithmic bytes / device time against
    the copy bandwidth.  The push passes include their side-list fix-up
    (~8 us); the solve's vectors (8 MB each at 1025^2) stay in L2, so it is
    latency-bound far below HBM, which the fraction shows."""
    steps = len(ev)
    nodes = (w.nx + 1) * (w.ny + 1)
    out = []
    for s, name in ((0, "electrons"), (1, "Ar+")):
        ms = sum((e[4].elapsed_time(e[3]) if s == 1 else e[2].elapsed_time(e[4])) for e in ev) / steps
        gbs = BYTES_PUSH_PASS * counts[s] / (ms * 1e-3) / 1e9
        out.append({"kernel": f"k_cells<kPush> {name} pass (+ k_fixup)", "ms": ms,
                    "bytes": BYTES_PUSH_PASS * counts[s], "achieved_GBs": gbs, "frac": gbs / peak})
    fl = phases["flush"]
    if fl["calls_per_step"]:
        ms = fl["ms_per_step"] / fl["calls_per_step"]
        gbs = FLUSH_BYTES_NODE * nodes / (ms * 1e-3) / 1e9
        out.append({"kernel": "k_flush (accumulators -> meshes, rho)", "ms": ms, "bytes": FLUSH_BYTES_NODE * nodes,
                    "achieved_GBs": gbs, "frac": gbs / peak})
    ms = statistics.mean(pois_ms)
    it = statistics.mean(iters)
    b = POISSON_BYTES_NODE_ITER * nodes * it
    gbs = b / (ms * 1e-3) / 1e9
    out.append({"kernel": "Poisson MG-PCG solve (k_mg_down, k_mg_fused, k_mg_up, k_pcg_pq, k_pcg_update per "
                "iteration; setup, true residual, E field)", "ms": ms, "iterations": it, "bytes": b,
                "bytes_per_node_iteration": POISSON_BYTES_NODE_ITER, "achieved_GBs": gbs, "frac": gbs / peak})
    for k in out:
        k["peak_GBs"] = peak
        k["peak_kind"] = f"{peak_kind} hbm_gbs"
    return out


def run_learned(pic, args, it):
    """The learned warm start on this workload (a short form of the
    train-then-evaluate protocol): record (input, RHS change) pairs from the
    running simulation, train the network on the GPU, then solve every
    evaluation step twice from the same state -- from the network's guess and
    from phi_{n-1} -- both to the same 1e-8 relative residual.  Poisson device
    milliseconds come from the library's own events around each solve."""
    import pic_b200 as P
    pic.ws_record(args.ws_pairs)
    for _ in range(args.ws_pairs + 1):
        pic.step(it)
        it += 1
    pic.ws_record(0)
    t0 = time.perf_counter()
    loss0 = pic.ws_train(1, args.ws_lr)
    loss = pic.ws_train_cosine(max(args.ws_epochs - 1, 1), args.ws_lr, args.ws_lr / 100)
    train_s = time.perf_counter() - t0
    ml, mp, il, ip, dphi, r0l, r0p = [], [], [], [], [], [], []
    for _ in range(args.ws_eval):
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        rho, phi_prev = pic.rho(), pic.phi()
        pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_LEARNED, 1e-8, 500)
        pic.poisson_solve(it)
        n_l, r_l, ms_l = pic.poisson_stats()
        r0l.append(pic.poisson_start_relres())
        phi_l = pic.phi()
        pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_PREVIOUS, 1e-8, 500)
        pic.set_phi(phi_prev)
        pic.set_rho(rho)
        pic.poisson_solve(it)
        n_p, r_p, ms_p = pic.poisson_stats()
        r0p.append(pic.poisson_start_relres())
        dphi.append(float(np.abs(phi_l - pic.phi()).max()))
        for s in range(2):
            pic.move_particles(s, it)
        it += 1
        ml.append(ms_l)
        mp.append(ms_p)
        il.append(n_l)
        ip.append(n_p)
    pic.ws_record(-1)
    # medians: a solve's event window spans host-issued launches and syncs, so
    # a host stall (another process, a driver query) lands in single steps
    return {"ms_per_step_learned": statistics.median(ml), "ms_per_step_plain_same_state": statistics.median(mp),
            "ms_mean_learned": statistics.mean(ml), "ms_mean_plain_same_state": statistics.mean(mp),
            "iters_learned": statistics.mean(il), "iters_plain_same_state": statistics.mean(ip),
            "start_relres_learned": statistics.mean(r0l), "start_relres_plain_same_state": statistics.mean(r0p),
            "max_abs_dphi_V": max(dphi), "train_pairs": args.ws_pairs, "train_epochs": args.ws_epochs,
            "train_s": train_s, "loss_first_epoch": loss0, "loss_last_epoch": loss,
            "eval_steps": args.ws_eval, "scales": list(pic.ws_scales()),
            "what": "residual loss |db - A guess|^2 (scaled); network: 3-level conv encoder-decoder, "
                    "32 channels, 32->32 convolutions (forward, data and weight gradients) on tcgen05 (TMEM accumulators), the 3->32 / 32->1 layers on mma.sync and FP32 cores; bf16 operands, FP32 accumulation"}, it


def run_ensemble(args, rank, world, local_rank):
    """The 64-instance ensemble (grids 128^2..384^2, left electrode 50-300 V,
    Bz 0-0.02 T, 32 particles/cell/species, 5e14-2e15 m^-3, seeded per
    instance): one launch per phase over all instances, the Poisson solves
    in one persistent launch, the step replayed as a CUDA graph, tile shape
    autotuned.  With N ranks the 64 instances are placed whole on the GPUs by
    the greedy longest-first rule on their cell counts (sharding.py): the
    total work is fixed ("strong" scaling), no data-path collective; times
    from each rank's ensemble CUDA events, max over ranks; per-instance
    results gathered to rank 0."""
    import pic_b200 as P
    import pic_configs as C
    import sharding as S
    ws = C.cfg5_instances()
    cells = [w.nx * w.ny for w in ws]
    mine = S.local(cells, world, rank)
    t0 = time.perf_counter()
    E = P.Ensemble([C.library_config(ws[k], device=local_rank) for k in mine]) if mine else None
    for j, k in enumerate(mine):
        C.load_plasma(E[j], ws[k], seed=5000 + 97 * k)
    setup_s = time.perf_counter() - t0
    n_local = sum(E[j].count(s) for j in range(len(mine)) for s in range(2)) if E else 0
    shape, ms_shapes = E.autotune() if E else (0, [])
    for it in range(args.warmup):
        if E:
            E.step(it)
    dep, pois, push, iters = [], [], [], []
    for it in range(args.warmup, args.warmup + args.ensemble_steps):
        if E:
            E.step(it)
            d, p, q = E.timing()
        else:
            d = p = q = 0.0
        dep.append(d)
        pois.append(p)
        push.append(q)
    metrics = {}
    if E:
        info = E.info()
        for j, k in enumerate(mine):
            it_k, rel_k, _ = E[j].poisson_stats()
            metrics[k] = {"rank": rank, "cells": cells[k], "iters": it_k, "relres": rel_k,
                          "particles": [E[j].count(s) for s in range(2)]}
        E.close()
    else:
        info = {"graph": False, "solver_blocks": 0}
    every = S.gather_metrics(metrics)
    part_ms = S.max_over_ranks(statistics.mean(d + q for d, q in zip(dep, push)))
    push_ms = S.max_over_ranks(statistics.mean(push))
    pois_ms = S.max_over_ranks(statistics.mean(pois))
    total_ms = S.max_over_ranks(statistics.mean(a + b + c for a, b, c in zip(dep, pois, push)))
    n_part = S.sum_over_ranks(n_local)
    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    return {"workload": f"{len(ws)} instances, grids {min(w.nx for w in ws)}^2..{max(w.nx for w in ws)}^2, "
                        "left electrode 50-300 V, Bz 0-0.02 T, 32 ppc/species, 5e14-2e15 m^-3",
            "instances": len(ws), "particles": int(n_part),
            "particle_steps_per_s": n_part / (part_ms * 1e-3),
            "ms_per_step_particles": part_ms, "ms_per_step_poisson_all": pois_ms,
            "ms_per_step_total": total_ms,
            "poisson_iters_mean": statistics.mean(m["iters"] for m in every.values()),
            "worst_relres": max(m["relres"] for m in every.values()),
            "push_roofline_frac": BYTES_PUSH_PASS * n_part / world / (push_ms * 1e-3) / 1e9 / peak,
            "tile_shape": ["64x4", "256x1", "128x2", "16x16"][shape], "ms_per_shape": ms_shapes,
            "graph": info["graph"], "solver_blocks": info["solver_blocks"], "steps": args.ensemble_steps,
            "setup_s": setup_s, "scaling": "strong", "n_gpus": world,
            "placement": "whole instances, greedy longest-first on cell counts; rank loads (cells) "
                         + str([int(x) for x in S.loads(cells, world)])}


def run_cfg4(args):
    """Learned vs plain warm start on the 1024^2 run: (input, RHS change)
    pairs recorded over steps 0..T-1, the network trained on the GPU, then
    every step of T..T+E-1 solved from the network's guess and, from the same
    state, from phi_{n-1}; both to 1e-8.  Prints its own JSON line."""
    import torch
    import pic_b200 as P
    import pic_configs as C
    torch.cuda.set_device(0)
    w = C.cfg3()
    pic = P.Pic(C.library_config(w))
    C.load_plasma(pic, w, seed=1234)
    T, E = args.cfg4_train, args.cfg4_eval
    t0 = time.perf_counter()
    pic.ws_record(T)
    plain_ms_rec, plain_it_rec = [], []
    for it in range(T + 1):
        pic.step(it)
        n_it, _, ms = pic.poisson_stats()
        plain_it_rec.append(n_it)
        plain_ms_rec.append(ms)
    pic.ws_record(0)
    rec_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    losses = [pic.ws_train(1, args.ws_lr)]
    losses.append(pic.ws_train_cosine(max(args.cfg4_epochs - 1, 1), args.ws_lr, args.ws_lr / 100))
    train_s = time.perf_counter() - t0
    pic.ws_record(-1)
    ml, mp, il, ip, dphi, r0l, r0p = [], [], [], [], [], [], []
    it = T + 1
    for _ in range(E):
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        rho, phi_prev = pic.rho(), pic.phi()
        pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_LEARNED, 1e-8, 500)
        pic.poisson_solve(it)
        n_l, r_l, ms_l = pic.poisson_stats()
        r0l.append(pic.poisson_start_relres())
        phi_l = pic.phi()
        pic.set_poisson(P.SOLVER_MG_PCG, P.WARM_PREVIOUS, 1e-8, 500)
        pic.set_phi(phi_prev)
        pic.set_rho(rho)
        pic.poisson_solve(it)
        n_p, r_p, ms_p = pic.poisson_stats()
        r0p.append(pic.poisson_start_relres())
        dphi.append(float(np.abs(phi_l - pic.phi()).max()))
        for s in range(2):
            pic.move_particles(s, it)
        it += 1
        ml.append(ms_l)
        mp.append(ms_p)
        il.append(n_l)
        ip.append(n_p)
    pic.close()
    line = {"metric": "Poisson ms/step, learned warm start, relres 1e-8", "value": statistics.mean(ml),
            "unit": "ms", "higher_is_better": False, "n_gpus": 1, "impl": "ours", "data": "synthetic",
            "config": {"workload": describe(w) + f"; train on steps 0-{T - 1}, evaluate on {T + 1}-{T + E}",
                       "epochs": args.cfg4_epochs},
            "plain_ms_per_step_same_state": statistics.mean(mp),
            "iters_learned": statistics.mean(il), "iters_plain_same_state": statistics.mean(ip),
            "start_relres_learned": statistics.mean(r0l), "start_relres_plain_same_state": statistics.mean(r0p),
            "iters_learned_hist": {str(k): il.count(k) for k in sorted(set(il))},
            "iters_plain_hist": {str(k): ip.count(k) for k in sorted(set(ip))},
            "max_abs_dphi_V": max(dphi), "loss_per_epoch": losses,
            "record_s": rec_s, "train_s": train_s,
            "plain_ms_during_recording": statistics.mean(plain_ms_rec)}
    print(json.dumps(line))
    return 0


def run_e2e(pic, steps, n_part, it0):
    """Same metric through the public C ABI with host buffers: import both
    species from host Points, K x (zero rho, deposit, read rho to host, push),
    export both species back.  Wall clock around the whole sequence."""
    import pic_b200 as P
    host = [pic.export_points(s) for s in range(2)]   # untimed: the inputs on the host
    # the caller's output buffers exist (and are paged in) before the run
    outbuf = [np.empty_like(h) for h in host]
    for o in outbuf:
        o.view(np.uint8).fill(0)
    rho_host = np.zeros(pic.nodes)
    t0 = time.perf_counter()
    for s in range(2):
        pic.import_points(s, host[s])
    pic.synchronize()
    t1 = time.perf_counter()
    for k in range(steps):
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        rho_host[:] = pic.rho()
        for s in range(2):
            pic.move_particles(s, it0 + k)
    pic.synchronize()
    t2 = time.perf_counter()
    out = [pic.export_points(s, outbuf[s]) for s in range(2)]
    pic.synchronize()
    t = time.perf_counter() - t0
    split = {"import_s": t1 - t0, "steps_s": t2 - t1, "export_s": t0 + t - t2}
    # bytes on the host link: the library moves 24-byte records (cell,
    # FP32 offsets and velocities); the caller's arrays hold 56-byte Points
    rec = 24
    h2d = sum(len(h) for h in host) * rec
    d2h = sum(len(o) for o in out) * rec
    return {"value": n_part * steps / t, "unit": UNIT,
            "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps + pic.nodes * 8,
            "link_bytes_per_particle": rec,
            "api_bytes_per_particle": P.POINT_DTYPE.itemsize,
            "wall_s": t, "split": split,
            "what": "pic_import_points (both species) + K x (zero_rho, charge_deposition x2, "
                    "pic_get_rho to host, move_particles x2) + pic_export_points; E held "
                    "from the last solve (Poisson excluded, as in the metric)"}


def run_solve_only(args):
    """K solves of the workload's Poisson problem from one state, for a
    kernel launch list; not a bench line."""
    import pic_b200 as P
    import pic_configs as C
    w = workload(args.config)
    with P.Pic(C.library_config(w, deposit_energy=not args.no_energy)) as pic:
        C.load_plasma(pic, w)
        for it in range(args.warmup):
            pic.step(it)
        phi_prev = pic.phi()
        pic.zero_rho()
        for s in range(2):
            pic.charge_deposition(s)
        rho = pic.rho()
        P._check(P.lib().pic_set_poisson_graph(pic.h, 0 if args.no_graph else 1))
        st = []
        for _ in range(args.steps):
            pic.set_rho(rho)
            pic.set_phi(phi_prev)
            pic.poisson_solve(args.warmup)
            st.append(pic.poisson_stats())
    print(json.dumps({"solve_only": describe(w), "graph": not args.no_graph, "iters": [x[0] for x in st],
                      "relres": st[-1][1], "ms_median": statistics.median([x[2] for x in st])}))
    return 0


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        w = workload(args.config)
        # every step is one full step of the workload
        r = cpu_reference_run(w, steps=args.steps + args.warmup)
        timed = r["part_t"][args.warmup:]
        value = r["n"] * len(timed) / sum(timed)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * sum(timed) / len(timed), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": describe(w), "particles": r["n"],
                           "parallelism": "host cores"},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["threads"], "kind": "port",
                                 "cpu": r["cpu"], "sample": r["sample"]},
                "poisson": {"ms_per_step": r["poisson_ms"], "solver": "SuperLU (PARDISO restatement)",
                            "factor_s": r["factor_s"]},
                "setup_s": r["setup_s"],
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if args.config == "cfg4":
        return run_cfg4(args) if rank == 0 else 0
    if args.solve_only:
        return run_solve_only(args) if rank == 0 else 0
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device(f"cuda:{local_rank}"))
    line, pic, w = run_ours(args, rank, world, local_rank)
    pic.close()
    if not args.no_ensemble and args.config == "cfg3":
        ens = run_ensemble(args, rank, world, local_rank)
        if rank == 0:
            line["ensemble"] = ens
    if rank == 0 and not args.no_cpu_baseline:
        r = cpu_reference_run(w, max_seconds=args.cpu_seconds)
        line["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": r["threads"],
                                "kind": "port", "cpu": r["cpu"], "sample": r["sample"],
                                "poisson_ms_per_step": r["poisson_ms"]}
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
